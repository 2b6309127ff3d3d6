"""The bench's multi-GPU path on the CPU: two gloo ranks, each baking its own map (seed = rank, no
collective on the data path), the step time taken as the maximum over ranks and the job's value as the
sum of every rank's rays over it. The bake itself runs on the oracle's tracer here (no GPU)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import time

    import torch.distributed as dist

    import bench
    import lightbaker_b200 as lb
    import oracle
    from lightbaker_b200 import scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=300))
    try:
        # small_map's seeds 0 and 3 both fit its 256-wide atlas
        scene = scenes.small_map(seed=3 * bench.rank_seed(rank))
        tracer, keep = oracle.tracer(threads=2)
        t0 = time.perf_counter()
        baked = lb.bake_with(scene, tracer)
        ms = (time.perf_counter() - t0) * 1e3
        ms_max = bench.reduce_max(ms, dist, "cpu")
        rays = baked.stats.rays
        out.put((rank, ms, ms_max, rays, bench.job_value(bench.sum_over_ranks(rays, dist, "cpu"), ms_max),
                 float(np.asarray(baked.indirect, np.float64).sum())))
        dist.barrier()
        del keep
    except Exception as e:
        out.put((rank, "error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_two_ranks_bake_their_own_maps_and_time_as_the_slowest():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=600) for _ in procs)
    assert all(r[1] != "error" for r in res), res
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (_, ms0, max0, rays0, v0, ind0), (_, ms1, max1, rays1, v1, ind1) = res
    assert max0 == max1 == pytest.approx(max(ms0, ms1))
    # weak scaling: each rank its own map
    assert ind0 != ind1
    # the job's rays are both ranks' own counts summed (the maps differ, so do their ray counts)
    assert rays0 != rays1
    assert v0 == v1 == pytest.approx((rays0 + rays1) / (max0 / 1e3) / 1e9)
