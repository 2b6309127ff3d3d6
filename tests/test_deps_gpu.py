"""The tiles' and probe chunks' dependency hashes computed on the device (csrc/deps.cu: the swept-box test
and BLAKE3 of every tile's message at once; deps.rs:70-121) against the host's (csrc/host/deps.cpp): a
device bake with a cache directory writes exactly the cache entries the drop-in bake writes (their names
are the hashes), and each bake finds the other's entries."""
import os
import shutil
import tempfile

import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["reference_test", "small_map", "map_100m"])
def test_device_hashes_equal_host_hashes(gpu, name):
    s = scenes.WORKLOADS[name]() if name != "reference_test" else scenes.reference_test(8.0)
    d_host, d_dev = tempfile.mkdtemp(prefix="lb-host-"), tempfile.mkdtemp(prefix="lb-dev-")
    try:
        host = lb.bake(s, gpu, cache=d_host)
        dev = lb.bake_device(s, gpu, cache=d_dev)
        names_host, names_dev = sorted(os.listdir(d_host)), sorted(os.listdir(d_dev))
        assert names_host == names_dev
        assert sum(n.startswith("tile-") for n in names_dev) == dev.stats.tiles
        assert sum(n.startswith("probes-") for n in names_dev) == dev.stats.chunks
        # the device bake reads the host's cache whole, and the host bake the device's
        again = lb.bake_device(s, gpu, cache=d_host)
        assert again.stats.tiles_baked == 0 and again.stats.chunks_baked == 0
        back = lb.bake(s, gpu, cache=d_dev)
        assert back.stats.tiles_baked == 0 and back.stats.chunks_baked == 0
    finally:
        shutil.rmtree(d_host, ignore_errors=True)
        shutil.rmtree(d_dev, ignore_errors=True)


def test_moved_box_changes_only_the_tiles_it_reaches(gpu):
    d = tempfile.mkdtemp(prefix="lb-move-")
    try:
        lb.bake(scenes.reference_test(8.0), gpu, cache=d)
        moved = lb.bake_device(scenes.reference_test(6.0), gpu, cache=d)
        d2 = tempfile.mkdtemp(prefix="lb-move2-")
        try:
            lb.bake(scenes.reference_test(8.0), gpu, cache=d2)
            moved_host = lb.bake(scenes.reference_test(6.0), gpu, cache=d2)
            assert 0 < moved.stats.tiles_baked == moved_host.stats.tiles_baked < moved.stats.tiles
            assert moved.stats.chunks_baked == moved_host.stats.chunks_baked
        finally:
            shutil.rmtree(d2, ignore_errors=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)
