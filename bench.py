"""Benchmark: rays traced per second (Grays/s) baking the 100 x 100 m map, and the bake's seconds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload map_100m]

A step is one whole bake of the map on the device: the direct pass over every covered texel (inside
test, 16 hard + 16 soft sun rays, 256 occlusion rays), the texel passes (occlusion curve, smoothing,
the sun's distance field, fills, the atlas), three bounces (gather pass of 128 rays a texel, smoothing,
fill, the atlas rewritten), the volume (50 x 50 x 16 probes, 128 sphere rays + 16 sun rays), its fill,
the fallback and the atlas composite: the device-resident bake's CUDA graph, inputs already in device
memory. `value` = the rays of a step (counted on the device) / the step's time (CUDA events on the
library's stream; L2 flushed before every step by writing 256 MB). `e2e` times the same bake through
the C ABI from the scene file's bytes in host memory to the atlases in host memory (the host's layout,
BVH and texels included; the median of three calls after an untimed first, each call's time listed).
`plain` is the drop-in bake (the reference's structure: a pass, a host round trip, the host's texel
passes) for the batched-vs-plain ratio. Under torchrun each rank bakes its own
map (seed = rank): weak scaling, no collective on the data path; times are the max over ranks.

--impl reference times the CPU restatement of the same passes (the oracle, OpenMP on every host core)
on a bounded sample of the same item lists, in the same unit.
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
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """Samples nvidia-smi during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
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

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in self.rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in self.rows) if v is not None]
        pw = [v for v in (num(r[3]) for r in self.rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(self.rows)}


def gather_items(P, by_tile):
    """Gather texels as the bake picks them, taking every covered texel as valid: the first covered
    texel of each chart in each smaller (ds x ds) texel, row order (bake.rs:286-298)."""
    ds = P.info.indirect_downscale
    out = []
    for t, tex in by_tile:
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


def rank_seed(rank: int) -> int:
    """Each rank bakes its own map of the workload (weak scaling): the map's seed is the rank."""
    return rank


def reduce_max(x: float, dist, device) -> float:
    """x's maximum over the ranks (every rank gets it); x itself with one process."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def sum_over_ranks(x: int, dist, device) -> int:
    """x summed over the ranks (every rank gets it); x itself with one process."""
    import torch
    t = torch.tensor([int(x)], dtype=torch.int64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def job_value(rays_all_ranks: int, ms_max: float) -> float:
    """Whole-job Grays/s: the rays every rank traced (summed: each rank bakes its own map) over the slowest
    rank's time."""
    return rays_all_ranks / (ms_max / 1e3) / 1e9


def algorithmic_bytes(workload: str, kernel: str):
    """The reference walk's bytes per item for a pass (tests/golden/algobytes.json, counted by the oracle on a
    1 % sample of the workload's items), or None."""
    try:
        d = json.loads((ROOT / "tests" / "golden" / "algobytes.json").read_text())
        return float(d[workload][kernel]["bytes_per_item"])
    except Exception:
        return None


def parse_tuning(tuning: str) -> dict:
    """The autotuner's report ("direct: bvh 2, refill 0, near 1, order 0, register cap 0, 2 blocks/SM (...);
    gather: ...") as {"direct": {"bvh": 2, ...}, "gather": {...}}."""
    import re
    out = {}
    for part in tuning.split(";"):
        if ":" not in part:
            continue
        name, rest = part.split(":", 1)
        out[name.strip()] = {k.strip(): int(v) for k, v in re.findall(r"([a-z ]+?) (\d+)(?:,|$| blocks)", rest)}
    return out


def scene_header(scene: bytes) -> dict:
    import struct
    hl = struct.unpack("<I", scene[8:12])[0]
    return json.loads(scene[12:12 + hl])


def probe_items(scene: bytes):
    import lightbaker_b200 as lb
    v = scene_header(scene).get("volume")
    if not v:  # a scene without an irradiance volume
        return np.zeros(0, dtype=lb.TEXEL)
    nx, ny, nz = [max(int(round((v["max"][a] - v["min"][a]) / v["step"])) + 1, 2) for a in range(3)]
    k = np.arange(nx * ny * nz, dtype=np.uint32)
    items = np.zeros(len(k), dtype=lb.TEXEL)
    st = np.float32(v["step"])
    items["pos"][:, 0] = np.float32(v["min"][0]) + (k % nx).astype(np.float32) * st
    items["pos"][:, 1] = np.float32(v["min"][1]) + (k // (nx * nz)).astype(np.float32) * st
    items["pos"][:, 2] = np.float32(v["min"][2]) + ((k // nx) % nz).astype(np.float32) * st
    items["pos"][:, 3] = 1.0
    items["normal"][:, 1] = 1.0
    items["normal"][:, 3] = k.view(np.float32)
    return items


def load_workload(name: str, seed: int):
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    scene = scenes.WORKLOADS[name](seed=seed) if name != "reference_test" else scenes.reference_test()
    P = lb.prepare(scene)
    by_tile = [(t, P.rasterize(t)) for t in range(len(P.tiles))]
    direct = np.concatenate([tex.reshape(-1)[tex.reshape(-1)["pos"][:, 3] > 0.5] for _, tex in by_tile])
    gather = gather_items(P, by_tile)
    light = np.zeros((P.info.atlas_width * P.info.atlas_height, 4), np.float32)
    for t, tex in by_tile:
        tl = P.tiles[t]
        cov = tex["pos"][:, :, 3] > 0.5
        blk = light.reshape(P.info.atlas_height, P.info.atlas_width, 4)[tl["y"]:tl["y"] + tl["h"], tl["x"]:tl["x"] + tl["w"]]
        blk[cov] = (1.0, 1.0, 1.0, 1.0)
    return scene, P, direct, gather, probe_items(scene), light


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
            if len(items) == 0:
                continue
            start = int(rng.integers(0, max(1, len(items) - chunk)))
            sample = items[start:start + chunk]
            t0 = time.perf_counter()
            _, cnt = oracle.run(pass_, sc, P.params, sample, light if pass_ else None, threads)
            secs += time.perf_counter() - t0
            rays += cnt["rays"]
            n_items[key] += len(sample)
    return rays / secs / 1e9, rays, secs, n_items


def reference_arm(args):
    _, rank, _ = dist_env()
    if rank != 0:
        return
    scene, P, direct, gather, probes, light = load_workload(args.workload, 0)
    per_step = min(args.cpu_seconds, 20.0) / max(1, args.steps)
    samples = []
    for i in range(args.warmup + args.steps):
        g, rays, secs, n_items = cpu_baseline(P, direct, gather, probes, light, per_step if i >= args.warmup else 1.0)
        if i >= args.warmup:
            samples.append((rays, secs))
    value = sum(s[0] for s in samples) / sum(s[1] for s in samples) / 1e9
    cores = os.cpu_count()
    sample = (f"oracle passes on contiguous slices of the {args.workload} item lists (2048 direct texels, "
              f"1024 gather texels, 256 probes a round), about {per_step:.1f} s a step, {cores} threads")
    print(json.dumps({
        "metric": "Grays/s", "value": value, "unit": "Grays/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(s[1] for s in samples) / len(samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "seed": 0, "triangles": int(P.info.n_triangles),
                   "direct_texels": int(len(direct)), "gather_texels": int(len(gather)), "probes": int(len(probes))},
        "cpu_baseline": {"value": value, "unit": "Grays/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Grays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def adjoint_only(args):
    """The transport's forward and backward alone on the workload, for a profiler: no flush."""
    import torch
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    scene = scenes.WORKLOADS[args.workload]()
    gpu = lb.Gpu.new(0)
    tr = lb.Transport(scene, gpu)
    dev = torch.device("cuda", 0)
    th = torch.from_numpy(tr.theta0()).to(dev)
    out = torch.empty((tr.ih, tr.iw, 4), dtype=torch.float32, device=dev)
    g_in = torch.rand((tr.ih, tr.iw, 4), dtype=torch.float32, device=dev)
    g_th = torch.empty(tr.n_params, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(gpu.stream, device=dev)
    torch.cuda.synchronize()
    res = {}
    for name, fn in (("forward", lambda: tr.forward_async(th.data_ptr(), out.data_ptr())),
                     ("backward", lambda: tr.backward_async(g_in.data_ptr(), g_th.data_ptr()))):
        times = []
        for i in range(args.warmup + args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            gpu.sync()
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1))
        res[name + "_ms"] = statistics.median(times)
    print(json.dumps({"kernel": "adjoint", "workload": args.workload, **res,
                      "backward_over_forward": res["backward_ms"] / res["forward_ms"]}))
    tr.close()
    gpu.close()


def kernel_only(args):
    """One pass kind alone over a slice of the workload's items, for a profiler: no flush, no bake."""
    import torch
    import lightbaker_b200 as lb
    if args.kernel_only == "adjoint":
        return adjoint_only(args)
    scene, P, direct, gather, probes, light = load_workload(args.workload, 0)
    items = (direct if args.kernel_only == "direct" else gather)[: args.items]
    gpu = lb.Gpu.new(0)
    gpu.set_pass_kernel(1)
    walk = [int(x) for x in args.walk.split(",")]
    bvh, refill, near, order = walk[:4]
    gpu.set_register_cap(walk[4] if len(walk) > 4 else 0)
    gpu.set_fetch(walk[5] if len(walk) > 5 else 0)
    gpu.set_warp_walk(walk[6] if len(walk) > 6 else 0)
    gpu.set_bvh(bvh)
    gpu.set_refill(refill)
    gpu.set_near(near)
    gpu.set_ray_order(order, order)
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)
    dev = torch.device("cuda", 0)
    d_items = torch.from_numpy(items.view(np.uint8).reshape(-1)).to(dev)
    d_light = torch.from_numpy(light.view(np.uint8).reshape(-1)).to(dev)
    out = torch.empty(len(items) * 16, dtype=torch.uint8, device=dev)
    pass_ = lb.Pass.DIRECT if args.kernel_only == "direct" else lb.Pass.GATHER
    stream = torch.cuda.ExternalStream(gpu.stream, device=dev)
    times = []
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        gpu.run_async(pass_, buffers, P.params, d_items.data_ptr(), len(items), 0, d_light.data_ptr(), len(light),
                      out.data_ptr())
        with torch.cuda.stream(stream):
            e1.record(stream)
        gpu.sync()
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1))
    rays = gpu.counters()["rays"]
    print(json.dumps({"kernel": f"{args.kernel_only}_warp", "walk": args.walk, "workload": args.workload, "items": int(len(items)),
                      "rays": int(rays), "ms": statistics.median(times), "grays": rays / statistics.median(times) / 1e6}))
    buffers.close()
    gpu.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="map_100m")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--device-only", action="store_true",
                    help="time the device bake's steps and stop (for a profiler's launch list)")
    ap.add_argument("--kernel-only", choices=["direct", "gather", "adjoint"], default=None,
                    help="run one warp-per-item pass over --items texels of the workload, warmup + steps times "
                         "(for profiler captures; prints its own line)")
    ap.add_argument("--items", type=int, default=262144)
    ap.add_argument("--walk", default="2,0,1,8",
                    help="kernel-only: bvh,refill,near,order[,register cap[,fetch[,warp walk]]]")
    ap.add_argument("--split", action="store_true",
                    help="N > 1: one map (seed 0) split over the ranks (lb_bake_options.exchange: each rank traces "
                         "its share of every pass, the outputs summed over NCCL), strong scaling; prints the "
                         "device bake's line and stops")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.kernel_only:
        return kernel_only(args)
    world, rank, local = dist_env()

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    import lightbaker_b200 as lb
    scene, P, direct, gather, probes, light = load_workload(args.workload, 0 if args.split else rank_seed(rank))
    gpu = lb.Gpu.new(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.ExternalStream(gpu.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, dev)

    # ---- the device-resident bake: graph replays, inputs resident ----
    exchange = lb.Exchange() if args.split and world > 1 else None
    plan = lb.Plan(scene, gpu, autotune=True, exchange=exchange)
    tuning = (lb._native.lib().lb_plan_tuning(plan._h) or b"").decode()
    plan.launch()
    gpu.sync()
    rays3 = plan.rays()
    rays_step = sum(rays3)
    kernels = lb._native.lib().lb_plan_kernels(plan._h)
    for _ in range(args.warmup):
        plan.launch()
    gpu.sync()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0.record(stream)
        plan.launch()
        with torch.cuda.stream(stream):
            e1.record(stream)
        gpu.sync()
        ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    ms_per_step = max_over_ranks(sum(ms) / len(ms))
    rays_job = sum_over_ranks(rays_step, dist, dev)
    value = job_value(rays_job, ms_per_step)
    baked = plan.result()
    plan.close()
    if args.device_only or args.split:
        # for a profiler's launch list: the device bake's steps alone; or one map split over the ranks (each
        # step's time includes the sums between the graph's pieces)
        if rank == 0:
            print(json.dumps({"metric": "Grays/s", "value": value, "unit": "Grays/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                              "device_only": True, "autotune": tuning, "graph_kernels": kernels,
                              "scaling": "strong" if args.split else "weak", "split": bool(args.split),
                              "config": {"workload": args.workload, "seed": 0 if args.split else "rank"},
                              "clocks": clock_info}))
        gpu.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- the dominant kernels alone: the warp-per-item passes over the same items ----
    buffers = gpu.scene(P.nodes, P.tris, P.materials, P.charts)

    def to_dev(a):
        return torch.from_numpy(a.view(np.uint8).reshape(-1)).to(dev)
    d_direct, d_gather, d_light = to_dev(direct), to_dev(gather), to_dev(light)
    out = torch.empty(max(len(direct), len(gather)) * 16, dtype=torch.uint8, device=dev)
    gpu.set_pass_kernel(1)
    kernel_stats = {}
    shapes = parse_tuning(tuning)
    for name, pass_, items, d_items in (("direct_warp", lb.Pass.DIRECT, direct, d_direct),
                                        ("gather_warp", lb.Pass.GATHER, gather, d_gather)):
        # the shape the plan's autotuner chose for this pass
        sh = shapes.get("direct" if pass_ == lb.Pass.DIRECT else "gather", {})
        gpu.set_bvh(sh.get("bvh", 2))
        gpu.set_refill(sh.get("refill", 0))
        gpu.set_near(sh.get("near", 1))
        gpu.set_register_cap(sh.get("register cap", 0))
        gpu.set_ray_order(sh.get("order", 8), sh.get("order", 8))
        gpu.set_fetch(sh.get("fetch", 0))
        gpu.set_warp_walk(sh.get("warp walk", 0))
        gpu.set_counting(True)
        gpu.run_async(pass_, buffers, P.params, d_items.data_ptr(), len(items), 0, d_light.data_ptr(), len(light),
                      out.data_ptr())
        gpu.sync()
        walk = gpu.counters()
        gpu.set_counting(False)
        times = []
        for i in range(max(3, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.fill_(1)
                e0.record(stream)
            gpu.run_async(pass_, buffers, P.params, d_items.data_ptr(), len(items), 0, d_light.data_ptr(), len(light),
                          out.data_ptr())
            with torch.cuda.stream(stream):
                e1.record(stream)
            gpu.sync()
            if i > 0:
                times.append(e0.elapsed_time(e1))
        kms = statistics.median(times)
        # the kernel's own fetches (its leaf lists and walks), counted on the device
        fetched = walk["nodes"] * 32 + walk["tris"] * 48 + walk["mats"] * 16 + len(items) * 80
        per_item = algorithmic_bytes(args.workload, name)
        kernel_stats[name] = {"ms": kms, "rays": walk["rays"], "kernel_fetch_bytes": fetched,
                              "alg_bytes": per_item * len(items) if per_item else None, "nodes": walk["nodes"],
                              "tris": walk["tris"], "mats": walk["mats"], "items": int(len(items))}
    gpu.set_pass_kernel(0)
    gpu.set_register_cap(0)
    gpu.set_ray_order(8, 8)
    gpu.set_near(1)
    gpu.set_fetch(True)
    gpu.set_warp_walk(True)
    buffers.close()
    del d_direct, d_gather, d_light, out

    # ---- end to end through the C ABI: scene bytes in host memory to atlases in host memory ----
    # (one call, as a user bakes a map once: no autotuning, the library's default shapes)
    gpu.transfer(reset=True)
    e2e_ms, bake_seconds, e2e_parts = [], [], []
    e2e_log = []
    for i in range(args.e2e_steps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        t0 = time.perf_counter()
        e2e_log.clear()
        b = lb.bake_device(scene, gpu, log=e2e_log.append)
        with torch.cuda.stream(stream):
            e1.record(stream)
        gpu.sync()
        wall = time.perf_counter() - t0
        if i == 0:
            gpu.transfer(reset=True)
            continue
        e2e_ms.append(e0.elapsed_time(e1))
        bake_seconds.append(wall)
        e2e_stats = b.stats
        # where each call's time went: the library's host build and its collection (device and results)
        e2e_parts.append([round(wall, 4), round(b.stats.t_layout, 4), round(b.stats.t_composite, 4)])
        b.close()
    h2d, d2h = gpu.transfer()
    # the median call (a call a step, after an untimed first one): the bake's host side shares the box's
    # cores, and one call in a few has met a stall of a fraction of a second there
    e2e_t = max_over_ranks(statistics.median(e2e_ms))
    e2e_value = job_value(sum_over_ranks(e2e_stats.rays, dist, dev), e2e_t)

    # ---- the plain drop-in bake (the reference's structure), once ----
    plain = None
    if not args.no_plain:
        t0 = time.perf_counter()
        pb = lb.bake(scene, gpu)
        pw = max_over_ranks(time.perf_counter() - t0)
        st = pb.stats
        plain = {"bake_seconds": pw, "grays_e2e": sum_over_ranks(st.rays, dist, dev) / pw / 1e9,
                 "grays_passes": st.rays / (st.t_direct + st.t_bounces + st.t_volume) / 1e9,
                 "pass_seconds": st.t_direct + st.t_bounces + st.t_volume, "rays": int(st.rays),
                 "stages_s": {"layout_bvh": st.t_layout, "direct": st.t_direct, "bounces": st.t_bounces,
                              "volume": st.t_volume}}
        pb.close()

    # ---- the bounce transport and its adjoint: gradients of the indirect atlas wrt albedos, sky, sun ----
    adjoint = None
    if not args.no_adjoint:
        def timed(fn, reps):
            out_ms = []
            for i in range(reps + 1):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                    e0.record(stream)
                fn()
                with torch.cuda.stream(stream):
                    e1.record(stream)
                gpu.sync()
                if i > 0:
                    out_ms.append(e0.elapsed_time(e1))
            return statistics.median(out_ms)

        t0 = time.perf_counter()
        tr = lb.Transport(scene, gpu)
        create_s = time.perf_counter() - t0
        th = torch.from_numpy(tr.theta0()).to(dev)
        out_t = torch.empty((tr.ih, tr.iw, 4), dtype=torch.float32, device=dev)
        g_in = torch.rand((tr.ih, tr.iw, 4), dtype=torch.float32, device=dev)
        g_th = torch.empty(tr.n_params, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        reps = max(3, args.steps)
        fwd_ms = timed(lambda: tr.forward_async(th.data_ptr(), out_t.data_ptr()), reps)
        bwd_ms = timed(lambda: tr.backward_async(g_in.data_ptr(), g_th.data_ptr()), reps)
        shape = tr.shape
        # the L2 loss against a target baked at theta0 + N(0, 0.05), its gradient at theta0, and central
        # differences (h = 1e-3) of the loss on a few parameters: albedos, the sky's colours, the sun
        rng = np.random.default_rng(100 + rank)
        theta0 = tr.theta0()
        target = tr.forward(theta0 + rng.normal(0.0, 0.05, theta0.shape).astype(np.float32)).astype(np.float64)

        def loss(t):
            return float(((tr.forward(t).astype(np.float64) - target) ** 2).sum())
        y0 = tr.forward(theta0)
        grad = tr.backward(2.0 * (y0.astype(np.float64) - target))
        M = tr.n_materials
        h = 1e-3
        checks = []
        for j in sorted({0, 1, 2, 3 * (M // 2) + 1, 3 * (M - 1) + 2, 3 * M, 3 * M + 4, 3 * M + 8, 3 * M + 9}):
            tp, tm = theta0.copy(), theta0.copy()
            tp[j] += h
            tm[j] -= h
            fd = (loss(tp) - loss(tm)) / (2 * h)
            gj = float(grad[j])
            checks.append({"param": j, "adjoint": gj, "central_difference": float(fd),
                           "rel_err": float(abs(fd - gj) / max(abs(gj), 1e-30))})
        # texels the volume's fallback lit (validity 5): the transport carries them through the probes, whose
        # rays it recorded at create
        fallback_texels = int((tr.export("state") == 5).sum())
        volume_records = int(len(tr.export("volume_records")))
        tr.close()
        one = lb.Transport(scene, gpu, max_checkpoints=1)
        one.forward_async(th.data_ptr(), out_t.data_ptr())
        bwd1_ms = timed(lambda: one.backward_async(g_in.data_ptr(), g_th.data_ptr()), reps)
        one_bytes = one.shape.checkpoint_bytes
        one.close()
        adjoint = {"forward_ms": max_over_ranks(fwd_ms), "backward_ms": max_over_ranks(bwd_ms),
                   "backward_over_forward": bwd_ms / fwd_ms, "create_s": create_s,
                   "backward_ms_one_checkpoint": max_over_ranks(bwd1_ms),
                   "checkpoint_bytes": {"every_bounce": int(shape.checkpoint_bytes), "one": int(one_bytes)},
                   "bounces": int(shape.bounces), "params": int(shape.n_params), "records": int(shape.records),
                   "lit_records": int(shape.lit_records),
                   "fallback_texels": fallback_texels,
                   "volume_records": volume_records,
                   "gradient_check": {"loss": "L2 to a target baked at theta0 + N(0, 0.05)", "h": h,
                                      "max_rel_err": max(c["rel_err"] for c in checks), "params": checks},
                   "note": "device time of one forward (theta on the device to the indirect atlas) and one "
                           "backward (atlas gradient to theta's gradient), CUDA graphs, L2 flushed before each"}
        del th, out_t, g_in, g_th

    if rank == 0:
        peaks = {}
        try:
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs")
        peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if hbm else "fallback 6650 GB/s"
        hbm = hbm or 6650.0
        # each pass runs once a step (the gathers of later bounces are evaluated from records)
        dom = max(kernel_stats, key=lambda k: kernel_stats[k]["ms"])
        ks = kernel_stats[dom]
        alg_src = "tests/golden/algobytes.json (the reference BVH2 walk's bytes per item, oracle, 1 % sample)"
        if ks["alg_bytes"] is None:
            ks["alg_bytes"], alg_src = ks["kernel_fetch_bytes"], "the kernel's own fetches (no frozen count)"
        achieved = ks["alg_bytes"] / (ks["ms"] / 1e3) / 1e9
        # DRAM and L2 bytes a launch from an ncu capture (profiles/traffic.txt: workload kernel dram_bytes
        # l2_bytes simt_efficiency source, a full launch each)
        traffic, traffic_src, l2_bytes, simt = None, None, None, None
        tfile = ROOT / "profiles" / "traffic.txt"
        if tfile.exists():
            for row in tfile.read_text().splitlines():
                f = row.split()
                if len(f) >= 6 and not row.startswith("#") and f[0] == args.workload and f[1] == dom:
                    traffic, l2_bytes, simt, traffic_src = int(f[2]), int(f[3]), float(f[4]), f[5]
        cpu_g, cpu_rays, cpu_secs, cpu_items = cpu_baseline(P, direct, gather, probes, light, args.cpu_seconds)
        line = {
            "metric": "Grays/s", "value": value, "unit": "Grays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "seed": "rank", "triangles": int(P.info.n_triangles),
                       "bvh_nodes": int(P.info.n_nodes), "direct_texels": int(baked.stats.texels_baked),
                       "bounces": int(P.info.gi_bounces), "probes": int(len(probes)),
                       "rays_per_step": int(rays_step), "rays_direct_gather_volume": [int(r) for r in rays3],
                       "rays_counted": "traced on the device; the gather rays of the first bounce only (later "
                                       "bounces evaluate its recorded outcomes: same rays, same bits)",
                       "l2": "flushed before every step (256 MB write)",
                       "path": "device-resident bake, one CUDA graph, warp-per-item BVH2 passes",
                       "autotune": tuning,
                       "parallelism": f"independent maps x{world}"},
            "bake_seconds": e2e_t / 1e3,
            "roofline": {"bound": "issue", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic,
                         "dram_frac": (traffic / (ks["ms"] / 1e3) / 1e9 / hbm) if traffic else None,
                         "l2_gbs": (l2_bytes / (ks["ms"] / 1e3) / 1e9) if l2_bytes else None,
                         "simt_efficiency": simt,
                         "traffic_source": traffic_src and f"profiles/{traffic_src}, scaled by texels",
                         "kernel": dom, "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": ks["alg_bytes"], "algorithmic_bytes_source": alg_src,
                         "kernel_fetch_bytes_per_launch": ks["kernel_fetch_bytes"], "kernel_ms": ks["ms"],
                         "note": "achieved = the reference BVH2 walk's bytes (32 B a node record, 48 B a triangle "
                                 "tested, 16 B a material, 80 B an item) for the launch's items over its time; "
                                 "they come from L1/L2 (the BVH fits in L2), so frac compares work rates, not "
                                 "HBM use: dram_frac is the DRAM bytes ncu measured over the same time. The "
                                 "kernel is bound by instruction issue and dependent-arithmetic latency "
                                 "(profiles/direct_warp_*.md)"},
            "kernels": kernel_stats,
            "cpu_baseline": {"value": cpu_g, "unit": "Grays/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"oracle on {cpu_items['direct']} direct, {cpu_items['gather']} gather texels "
                                       f"and {cpu_items['volume']} probes of this workload ({cpu_rays} rays, "
                                       f"{cpu_secs:.1f} s)"},
            "e2e": {"value": e2e_value, "unit": "Grays/s", "h2d_bytes_per_step": h2d // max(1, args.e2e_steps),
                    "d2h_bytes_per_step": d2h // max(1, args.e2e_steps), "bake_seconds": e2e_t / 1e3,
                    "calls_s": [round(t / 1e3, 4) for t in e2e_ms], "of_calls": "median",
                    "calls_wall_build_collect_s": e2e_parts,
                    "host_prepare_s": e2e_stats.t_layout, "collect_s": e2e_stats.t_composite,
                    "stages": [l for l in e2e_log if l.startswith("timing")],
                    "path": "lb_bake_device: scene bytes in, atlases out, one call, default shapes (no autotune)"},
            "plain": plain,
            "adjoint": adjoint,
            # the same bake (same outputs): the drop-in's pass seconds over the device step's seconds
            "batched_vs_plain": (plain["pass_seconds"] / (ms_per_step / 1e3)) if plain else None,
            # the same comparison in the metric's unit: each path's traced rays over its own seconds (the device
            # traces the first bounce's gather rays only; the drop-in traces every bounce's)
            "batched_vs_plain_grays": (value / world / plain["grays_passes"]) if plain else None,
            "gpu_launches": kernels * args.steps,
            "clocks": clock_info,
        }
        print(json.dumps(line))
    gpu.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
