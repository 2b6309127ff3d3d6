"""The bake split over ranks with its passes on the GPU (lb_bake_run with an lb_exchange): two ranks run as two
threads of this process, each with its own handle (its own stream) on the one GPU, their sums made on the host
(the ranks meet only between passes, on the host: no kernel waits for another). Each rank's passes key their items
from the rank's base (lb_run's params.atlas[2]), so both ranks must return the one-process bake bit for bit."""
import ctypes as C
import threading

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import _native as N
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


class HostGroup:
    """An element-wise sum of 32-bit words over `world` threads: every call of every rank adds its words to
    that call's accumulator, waits for the others, then takes the sum."""

    def __init__(self, world):
        self.world = world
        self.barrier = threading.Barrier(world, timeout=600)
        self.lock = threading.Lock()
        self.acc = {}

    def exchange(self, rank):
        calls = [0]

        def _sum(ctx, data, count, device):
            try:
                assert device == 0
                a = np.ctypeslib.as_array(C.cast(data, C.POINTER(C.c_uint32)), shape=(count,))
                k = calls[0]
                calls[0] += 1
                with self.lock:
                    acc = self.acc.setdefault(k, np.zeros(count, np.uint32))
                    acc += a
                self.barrier.wait()
                a[:] = self.acc[k]
                self.barrier.wait()
                return 0
            except Exception:
                self.barrier.abort()
                return 1

        cb = N.SUM_CB(_sum)
        ex = lb.Exchange.__new__(lb.Exchange)
        ex.rank, ex.world, ex._cb = rank, self.world, cb
        ex.struct = N.Exchange(None, rank, self.world, cb)
        return ex


def digest(b):
    return [np.ascontiguousarray(a).tobytes() for a in (b.direct, b.validity, b.indirect, b.volume) if a is not None]


@pytest.mark.parametrize("name", ["reference_test", "small_map"])
def test_two_ranks_on_one_gpu_equal_one_process(gpu, name):
    s = scenes.WORKLOADS[name]()
    want = digest(lb.bake(s, gpu))
    group = HostGroup(2)
    out, errors = [None, None], []

    def rank(r):
        g = lb.Gpu.new(0)
        try:
            b = lb.bake(s, g, exchange=group.exchange(r))
            out[r] = (digest(b), b.stats.rays)
            b.close()
        except Exception as e:  # reported below
            errors.append(repr(e))
            group.barrier.abort()
        finally:
            g.close()

    threads = [threading.Thread(target=rank, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=900)
    assert not errors, errors
    assert out[0][0] == want and out[1][0] == want


class DeviceGroup(HostGroup):
    """The same sums for device words (the device-resident bake's exchanges): each rank's words come to the
    host through torch, are added there, and go back."""

    def exchange(self, rank):
        import torch
        calls = [0]

        def _sum(ctx, data, count, device):
            try:
                assert device == 1
                t = torch.as_tensor(lb._DeviceWords(data, count), device="cuda")
                a = t.cpu().numpy().view(np.uint32)
                k = calls[0]
                calls[0] += 1
                with self.lock:
                    acc = self.acc.setdefault(k, np.zeros(count, np.uint32))
                    acc += a
                self.barrier.wait()
                t.copy_(torch.from_numpy(self.acc[k].view(np.int32)).cuda())
                torch.cuda.synchronize()
                self.barrier.wait()
                return 0
            except Exception:
                self.barrier.abort()
                return 1

        cb = N.SUM_CB(_sum)
        ex = lb.Exchange.__new__(lb.Exchange)
        ex.rank, ex.world, ex._cb = rank, self.world, cb
        ex.struct = N.Exchange(None, rank, self.world, cb)
        return ex


def _device_ranks(s, world, cache_src=None):
    """`world` ranks as threads, each its own handle (stream) on the one GPU, each a device-resident bake of
    its shares; their digests, rays and logs."""
    import shutil
    import tempfile
    group = DeviceGroup(world)
    out, errors = [None] * world, []

    def rank(r):
        g = lb.Gpu.new(0)
        cache = None
        try:
            if cache_src:
                cache = tempfile.mkdtemp(prefix=f"lb-dshard{r}-")
                shutil.copytree(cache_src, cache, dirs_exist_ok=True)
            logs = []
            b = lb.bake_device(s, g, cache=cache, log=logs.append, exchange=group.exchange(r))
            out[r] = (digest(b), b.stats.rays, [l for l in logs if "rank" in l], b.stats.tiles_baked)
            b.close()
        except Exception as e:  # reported below
            errors.append(repr(e))
            group.barrier.abort()
        finally:
            g.close()
            if cache:
                shutil.rmtree(cache, ignore_errors=True)

    threads = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=900)
    assert not errors, errors
    return out


@pytest.mark.parametrize("world,name", [(2, "reference_test"), (2, "small_map"), (3, "small_map")])
def test_device_bake_split_over_ranks_equals_one_process(gpu, world, name):
    """The device-resident bake split over ranks (lb_bake_device with an exchange): every pass traces the
    rank's share of its items, the graph is cut after each pass and the ranks sum its outputs; every rank
    returns the one-process bake bit for bit, and the ranks' rays add up to its rays."""
    s = scenes.WORKLOADS[name]()
    one = lb.bake_device(s, gpu)
    want, rays = digest(one), one.stats.rays
    one.close()
    out = _device_ranks(s, world)
    assert all(o[0] == want for o in out), "a rank's bake differs from the one-process bake"
    assert sum(o[1] for o in out) == rays
    assert all(o[2] for o in out)  # each rank logged its share


def test_device_bake_split_with_some_tiles_cached(gpu):
    """A cache holding the tiles of the box at x = 8; after it moves to x = 6 the two ranks rebake the tiles
    it reaches on the device, the cached tiles' light entering on both."""
    import shutil
    import tempfile
    src = tempfile.mkdtemp(prefix="lb-dsrc-")
    one_cache = tempfile.mkdtemp(prefix="lb-done-")
    try:
        lb.bake_device(scenes.reference_test(8.0), gpu, cache=src).close()
        shutil.copytree(src, one_cache, dirs_exist_ok=True)
        s = scenes.reference_test(6.0)
        one = lb.bake_device(s, gpu, cache=one_cache)
        want, tiles = digest(one), one.stats.tiles_baked
        one.close()
        assert 0 < tiles < 16
        out = _device_ranks(s, 2, src)
        assert all(o[0] == want for o in out)
        assert all(o[3] == tiles for o in out)
    finally:
        shutil.rmtree(src, ignore_errors=True)
        shutil.rmtree(one_cache, ignore_errors=True)
