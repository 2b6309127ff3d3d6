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
