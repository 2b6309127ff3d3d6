"""Writes tests/golden/bvh_hashes.json: the BLAKE3 of the BVH2 (nodes, then triangles, as the host
builds them for the device) of each synthetic workload. Run once with a build known to follow
crates/lightbaker/src/bvh.rs:50-106 step by step (the serial builder); the tests then hold every later
build, parallel or not, to the same bytes."""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import lightbaker_b200 as lb  # noqa: E402
from lightbaker_b200 import scenes  # noqa: E402


def digest(name: str) -> dict:
    P = lb.prepare(scenes.WORKLOADS[name]())
    return {"nodes": len(P.nodes), "tris": len(P.tris),
            "blake3": lb.blake3(P.nodes.tobytes() + P.tris.tobytes()).hex()}


if __name__ == "__main__":
    out = {name: digest(name) for name in ("reference_test", "small_map", "map_100m")}
    (HERE / "bvh_hashes.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))
