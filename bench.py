"""Benchmark: rays traced per second (Grays/s) baking the 100 x 100 m map, and the bake's seconds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload map_100m]

A step is one bake's ray work over the whole map: the direct pass over every covered texel (inside
test, 2 x 16 sun rays, 256 occlusion rays), three gather passes (128 rays a texel) and the volume pass
(50 x 50 x 16 probes, 128 sphere rays + 16 sun rays). `value` times those passes with their inputs
already in device memory (CUDA events on the library's stream, L2 flushed between steps by writing a
256 MB buffer); `e2e` times the drop-in bake through the C ABI from the scene file's bytes in host
memory to the atlases back in host memory (layout, BVH, texels, the passes, the texel passes, the
volume, the atlas). Under torchrun each rank bakes its own map (seed = rank): weak scaling, no
collective on the data path; the time is the max over ranks.

--impl reference times the CPU restatement of the same passes (the oracle, OpenMP on every host core)
on a bounded sample of the same item lists, reported in the same unit.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """Samples nvidia-smi during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def gather_items(P, covered_by_tile):
    """Gather texels as the bake picks them before knowing which texels lie inside solids: covered texels
    on the indirect grid, plus the first texel of each (smaller texel, chart) pair (bake.rs:286-298)."""
    ds = P.info.indirect_downscale
    out = []
    for t, tex in covered_by_tile:
        h, w = tex.shape
        cov = tex["pos"][:, :, 3] > 0.5
        chart = tex["normal"][:, :, 3].view(np.uint32)
        yy, xx = np.mgrid[0:h, 0:w]
        grid = cov & (yy % ds == 0) & (xx % ds == 0)
        block = (yy // ds) * ((w + ds - 1) // ds) + xx // ds
        key = block.astype(np.uint64) << np.uint64(32) | chart.astype(np.uint64)
        flat_cov = np.flatnonzero(cov)
        keys = key.reshape(-1)[flat_cov]
        uniq, first = np.unique(keys, return_index=True)
        extra = flat_cov[first[~np.isin(uniq, key[grid])]]
        g = grid.reshape(-1).copy()
        g[extra] = True
        out.append(tex.reshape(-1)[g])
    return np.concatenate(out)


def probe_items(P, scene_header):
    v = scene_header["volume"]
    n = [max(int(round((v["max"][a] - v["min"][a]) / v["step"])) + 1, 2) for a in range(3)]
    nx, ny, nz = n
    k = np.arange(nx * ny * nz, dtype=np.uint32)
    items = np.zeros(len(k), dtype=__import__("lightbaker_b200").TEXEL)
    items["pos"][:, 0] = np.float32(v["min"][0]) + (k % nx).astype(np.float32) * np.float32(v["step"])
    items["pos"][:, 1] = np.float32(v["min"][1]) + (k // (nx * nz)).astype(np.float32) * np.float32(v["step"])
    items["pos"][:, 2] = np.float32(v["min"][2]) + ((k // nx) % nz).astype(np.float32) * np.float32(v["step"])
    items["pos"][:, 3] = 1.0
    items["normal"][:, 1] = 1.0
    items["normal"][:, 3] = k.view(np.float32)
    return items


def scene_header(scene: bytes) -> dict:
    import struct
    hl = struct.unpack("<I", scene[8:12])[0]
    return json.loads(scene[12:12 + hl])


def load_workload(name: str, seed: int):
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    scene = scenes.WORKLOADS[name](seed=seed) if name != "reference_test" else scenes.reference_test()
    P = lb.prepare(scene)
    by_tile = [(t, P.rasterize(t)) for t in range(len(P.tiles))]
    direct = np.concatenate([tex.reshape(-1)[tex.reshape(-1)["pos"][:, 3] > 0.5] for _, tex in by_tile])
    gather = gather_items(P, by_tile)
    probes = probe_items(P, scene_header(scene))
    light = np.zeros((P.info.atlas_width * P.info.atlas_height, 4), np.float32)
    for t, tex in by_tile:
        tl = P.tiles[t]
        cov = tex["pos"][:, :, 3] > 0.5
        blk = light.reshape(P.info.atlas_height, P.info.atlas_width, 4)[tl["y"]:tl["y"] + tl["h"], tl["x"]:tl["x"] + tl["w"]]
        blk[cov] = (1.0, 1.0, 1.0, 1.0)
    return scene, P, direct, gather, probes, light


def cpu_baseline(P, direct, gather, probes, light, budget_s: float, threads: int = 0):
    """The oracle on a bounded sample of the workload's items: rays per second on the host's cores."""
    import oracle
    sc = oracle.Scene.of(P)
    rng = np.random.default_rng(7)
    rays, secs, n_items = 0, 0.0, {"direct": 0, "gather": 0, "volume": 0}
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end:
        for pass_, items, chunk, key in ((0, direct, 2048, "direct"), (1, gather, 1024, "gather"),
                                         (2, probes, 256, "volume")):
            start = int(rng.integers(0, max(1, len(items) - chunk)))
            sample = items[start:start + chunk]
            t0 = time.perf_counter()
            _, cnt = oracle.run(pass_, sc, P.params, sample, light if pass_ else None, threads)
            secs += time.perf_counter() - t0
            rays += cnt["rays"]
            n_items[key] += len(sample)
    return rays / secs / 1e9, rays, secs, n_items


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="map_100m")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    world, rank, local = dist_env()

    if args.impl == "reference":
        # the CPU restatement on this host's cores: rank 0 alone
        if rank != 0:
            return
        import oracle  # noqa: F401
        scene, P, direct, gather, probes, light = load_workload(args.workload, 0)
        samples = []
        for i in range(args.warmup + args.steps):
            g, rays, secs, n_items = cpu_baseline(P, direct, gather, probes, light,
                                                  min(args.cpu_seconds, 20.0) / max(1, args.steps))
            if i >= args.warmup:
                samples.append((g, rays, secs))
        value = sum(s[1] for s in samples) / sum(s[2] for s in samples) / 1e9
        cores = os.cpu_count()
        line = {"metric": "Grays/s", "value": value, "unit": "Grays/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * sum(s[2] for s in samples) / len(samples), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload, "seed": 0, "triangles": int(P.info.n_triangles),
                           "direct_texels": int(len(direct)), "gather_texels": int(len(gather)),
                           "probes": int(len(probes))},
                "cpu_baseline": {"value": value, "unit": "Grays/s", "cores": cores, "kind": "port",
                                 "sample": f"oracle passes on contiguous slices of the {args.workload} item lists "
                                           f"(2048 direct, 1024 gather, 256 probes a round), about "
                                           f"{min(args.cpu_seconds, 20.0) / max(1, args.steps):.1f} s a step"},
                "e2e": {"value": value, "unit": "Grays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    import lightbaker_b200 as lb
    scene, P, direct, gather, probes, light = load_workload(args.workload, rank)
    gpu = lb.Gpu.new(local)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(gpu.stream, device=dev)

    def to_dev(a):
        return torch.from_numpy(a.view(np.uint8).reshape(-1)).to(dev)

    d_direct, d_gather, d_probes, d_light = to_dev(direct), to_dev(gather), to_dev(probes), to_dev(light)
    out_direct = torch.empty(len(direct) * 16, dtype=torch.uint8, device=dev)
    out_gather = torch.empty(len(gather) * 16, dtype=torch.uint8, device=dev)
    out_probes = torch.empty(len(probes) * 64, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    params = P.params
    params_vol = params.copy()
    params_vol.counts[2] = scene_header(scene)["volume"]["rays"]
    bounces = P.info.gi_bounces
    n_light = len(light)

    def step(ev=None):
        with torch.cuda.stream(stream):
            if ev is not None:
                ev[0].record(stream)
            gpu.run_async(lb.Pass.DIRECT, buffers, params, d_direct.data_ptr(), len(direct), 0,
                          d_light.data_ptr(), n_light, out_direct.data_ptr())
            if ev is not None:
                ev[1].record(stream)
            for _ in range(bounces):
                gpu.run_async(lb.Pass.GATHER, buffers, params, d_gather.data_ptr(), len(gather), 0,
                              d_light.data_ptr(), n_light, out_gather.data_ptr())
            gpu.run_async(lb.Pass.VOLUME, buffers, params_vol, d_probes.data_ptr(), len(probes), 0,
                          d_light.data_ptr(), n_light, out_probes.data_ptr())

    # rays a step, counted on the device, and the direct pass's walk for the roofline
    gpu.set_counting(True)
    with torch.cuda.stream(stream):
        gpu.run_async(lb.Pass.DIRECT, buffers, params, d_direct.data_ptr(), len(direct), 0, d_light.data_ptr(),
                      n_light, out_direct.data_ptr())
    gpu.sync()
    walk = gpu.counters()
    gpu.set_counting(False)
    rays_step = walk["rays"]
    with torch.cuda.stream(stream):
        gpu.run_async(lb.Pass.GATHER, buffers, params, d_gather.data_ptr(), len(gather), 0, d_light.data_ptr(),
                      n_light, out_gather.data_ptr())
    gpu.sync()
    rays_step += bounces * gpu.counters()["rays"]
    with torch.cuda.stream(stream):
        gpu.run_async(lb.Pass.VOLUME, buffers, params_vol, d_probes.data_ptr(), len(probes), 0, d_light.data_ptr(),
                      n_light, out_probes.data_ptr())
    gpu.sync()
    rays_step += gpu.counters()["rays"]

    for _ in range(args.warmup):
        step()
    gpu.sync()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = Clocks(local)
    clocks.start()
    total_ms, direct_ms = 0.0, []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        step(ev)
        with torch.cuda.stream(stream):
            ev[2].record(stream)
        gpu.sync()
        total_ms += ev[0].elapsed_time(ev[2])
        direct_ms.append(ev[0].elapsed_time(ev[1]))
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    elapsed = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(elapsed, op=torch.distributed.ReduceOp.MAX)
    ms_per_step = elapsed.item() / args.steps
    value = rays_step * world / (ms_per_step / 1e3) / 1e9

    # end to end through the C ABI: scene bytes in host memory to atlases in host memory
    gpu.transfer(reset=True)
    e2e_ms = []
    e2e_rays = 0
    for i in range(args.e2e_steps + 1):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
        b = lb.bake(scene, gpu)
        with torch.cuda.stream(stream):
            ev1.record(stream)
        gpu.sync()
        if i == 0:  # warm-up bake
            gpu.transfer(reset=True)
            continue
        e2e_ms.append(ev0.elapsed_time(ev1))
        e2e_rays = b.stats.rays
        bake_stats = b.stats
        b.close()
    h2d, d2h = gpu.transfer()
    e2e_t = torch.tensor([sum(e2e_ms) / len(e2e_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = e2e_rays * world / (e2e_t.item() / 1e3) / 1e9

    if rank == 0:
        peaks = {}
        try:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs")
        peak_note = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        alg_bytes = walk["nodes"] * 32 + walk["tris"] * 48 + walk["mats"] * 16 + len(direct) * (64 + 16)
        dms = statistics.median(direct_ms)
        achieved = alg_bytes / (dms / 1e3) / 1e9
        traffic = None
        tfile = ROOT / "profiles" / "traffic.json"
        if tfile.exists():
            try:
                traffic = json.loads(tfile.read_text()).get(args.workload, {}).get("direct_bytes_per_launch")
            except Exception:
                traffic = None
        cpu_g, cpu_rays, cpu_secs, cpu_items = cpu_baseline(P, direct, gather, probes, light, args.cpu_seconds)
        line = {
            "metric": "Grays/s", "value": value, "unit": "Grays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "seed": "rank", "triangles": int(P.info.n_triangles),
                       "bvh_nodes": int(P.info.n_nodes), "direct_texels": int(len(direct)),
                       "gather_texels": int(len(gather)), "bounces": int(bounces), "probes": int(len(probes)),
                       "rays_per_step": int(rays_step), "l2": "flushed between steps (256 MB write)",
                       "path": "BVH2 passes, one thread an item", "parallelism": f"replicas x{world}"},
            "bake_seconds": e2e_t.item() / 1e3,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "kernel": "direct_kernel", "peak_source": peak_note,
                         "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": dms},
            "cpu_baseline": {"value": cpu_g, "unit": "Grays/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"oracle on {cpu_items['direct']} direct, {cpu_items['gather']} gather texels "
                                       f"and {cpu_items['volume']} probes of this workload ({cpu_rays} rays, "
                                       f"{cpu_secs:.1f} s)"},
            "e2e": {"value": e2e_value, "unit": "Grays/s", "h2d_bytes_per_step": h2d // max(1, args.e2e_steps),
                    "d2h_bytes_per_step": d2h // max(1, args.e2e_steps), "bake_seconds": e2e_t.item() / 1e3,
                    "stages_s": {"layout_bvh": bake_stats.t_layout, "direct": bake_stats.t_direct,
                                 "bounces": bake_stats.t_bounces, "volume": bake_stats.t_volume}},
            "gpu_launches": args.steps * (2 + bounces),
            "clocks": clock_info,
        }
        print(json.dumps(line))
    buffers.close()
    gpu.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
