"""Writes tests/golden/algobytes.json: the algorithmic bytes a ray pass moves per item, counted on the
reference's own BVH2 walk by the oracle (oracle/trace_ref.cpp, trace.wgsl:83-130) on a fixed 1 % sample of
the workload's items (every 100th), for the bench's roofline numerator. The definition, per item:

    32 B per BVH2 node record fetched (the root, then both children of every inner node visited)
  + 48 B per triangle tested + 16 B per material read (an accepted candidate's opacity)
  + 64 B texel record in + 16 B result out
  + for a gather ray that meets a surface: 32 B chart + 16 B light atlas texel

This counts the reference walk's work, independent of how the product's kernels walk (leaf lists, ray order,
register caps), so achieved = these bytes / the kernel's time compares kernels on the same work.

    python tests/golden/make_algobytes.py [workload ...]
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from bench import load_workload  # noqa: E402


def counts(name: str, every: int = 100) -> dict:
    scene, P, direct, gather, probes, light = load_workload(name, 0)
    sc = oracle.Scene.of(P)
    out = {}
    for kernel, pass_, items in (("direct_warp", 0, direct), ("gather_warp", 1, gather)):
        sample = np.ascontiguousarray(items[::every])
        t0 = time.perf_counter()
        _, c = oracle.run(pass_, sc, P.params, sample, light if pass_ else None)
        surface = 0
        if pass_ == 1:
            rec = oracle.gather_records(sc, P.params, sample, len(light))
            surface = int((rec[:, :, 0] == 2).sum())
        n = len(sample)
        walk = 32 * c["nodes"] + 48 * c["tris"] + 16 * c["mats"]
        out[kernel] = {"items_sampled": n, "items_total": int(len(items)), "every": every, "rays": c["rays"],
                       "nodes": c["nodes"], "tris": c["tris"], "mats": c["mats"], "surface_hits": surface,
                       "bytes_per_item": (walk + 48 * surface) / n + 80.0,
                       "oracle_seconds": round(time.perf_counter() - t0, 2)}
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or ["map_100m"]
    path = HERE / "algobytes.json"
    data = json.loads(path.read_text()) if path.exists() else {}
    for name in names:
        data[name] = counts(name)
    path.write_text(json.dumps(data, indent=1) + "\n")
    print(json.dumps(data, indent=1))
