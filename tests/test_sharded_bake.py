"""One bake split over ranks (lb_exchange): each rank bakes a contiguous share of the dirty tiles and of the probe
chunks, and the light atlas after every bounce, the probes and the atlases' pieces travel as sums of 32-bit words
(one writer a word). Run as gloo ranks on the CPU with the oracle's tracer: every rank's atlases, validity and
volume must equal the one-process bake's bit for bit, with a cold cache and with a cache that holds some tiles."""
import os
import shutil
import socket
import tempfile

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _digest(b):
    import hashlib
    h = hashlib.sha256()
    for a in (b.direct, b.validity, b.indirect, b.volume):
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _rank(rank, world, port, name, cache_src, out):
    import torch.distributed as dist

    import lightbaker_b200 as lb
    import oracle
    from lightbaker_b200 import scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=300))
    cache = None
    try:
        if cache_src:
            # every rank reads the same cache state (a copy of its own: each rank writes its tiles)
            cache = tempfile.mkdtemp(prefix=f"lb-shard{rank}-")
            shutil.copytree(cache_src, cache, dirs_exist_ok=True)
        scene = scenes.reference_test(6.0) if name == "reference_moved" else scenes.WORKLOADS[name]()
        tracer, keep = oracle.tracer(threads=2)
        logs = []
        baked = lb.bake_with(scene, tracer, cache=cache, log=logs.append, exchange=lb.Exchange())
        out.put((rank, _digest(baked), baked.stats.tiles_baked, baked.stats.rays, [l for l in logs if "rank" in l]))
        dist.barrier()
        del keep
    except Exception as e:
        out.put((rank, "error", repr(e), 0, []))
        raise
    finally:
        if cache:
            shutil.rmtree(cache, ignore_errors=True)
        dist.destroy_process_group()


def _run(world, name, cache_src=None):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, cache_src, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=900) for _ in procs)
    for p in procs:
        p.join(timeout=120)
    assert all(r[1] != "error" for r in res), res
    assert all(p.exitcode == 0 for p in procs)
    return res


def _one_process(name, cache_src=None):
    import lightbaker_b200 as lb
    import oracle
    from lightbaker_b200 import scenes
    scene = scenes.reference_test(6.0) if name == "reference_moved" else scenes.WORKLOADS[name]()
    cache = None
    if cache_src:
        cache = tempfile.mkdtemp(prefix="lb-one-")
        shutil.copytree(cache_src, cache, dirs_exist_ok=True)
    try:
        tracer, keep = oracle.tracer()
        b = lb.bake_with(scene, tracer, cache=cache)
        return _digest(b), b.stats.tiles_baked, b.stats.rays
    finally:
        if cache:
            shutil.rmtree(cache, ignore_errors=True)


@pytest.mark.parametrize("world,name", [(2, "small_map"), (3, "reference_test")])
def test_sharded_bake_equals_one_process(world, name):
    want, tiles, rays = _one_process(name)
    res = _run(world, name)
    assert all(r[1] == want for r in res), "a rank's bake differs from the one-process bake"
    assert all(r[2] == tiles for r in res)
    # the ranks' rays add up to the one process's (each traced its own share)
    assert sum(r[3] for r in res) == rays
    assert all(r[4] for r in res)  # each rank logged its share


def test_sharded_bake_with_some_tiles_cached():
    """A cache holding the tiles of the box at x = 8: after the box moves to x = 6, only the tiles it reaches
    are baked again, split over the ranks; the cached tiles' light enters on every rank."""
    import lightbaker_b200 as lb
    import oracle
    from lightbaker_b200 import scenes
    src = tempfile.mkdtemp(prefix="lb-src-")
    try:
        tracer, keep = oracle.tracer()
        lb.bake_with(scenes.reference_test(8.0), tracer, cache=src)
        want, tiles, rays = _one_process("reference_moved", src)
        assert 0 < tiles < 16
        res = _run(2, "reference_moved", src)
        assert all(r[1] == want for r in res)
        assert all(r[2] == tiles for r in res)
    finally:
        shutil.rmtree(src, ignore_errors=True)
