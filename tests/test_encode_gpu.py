"""The file encodings made on the device (csrc/encode.cu: BC5 of the direct atlas, RGB9E5 of the indirect
atlas, the probes' bytes; encode.rs:7-70, output.rs:97-181) against the host's encoders: the same bits, so
the .lbake written from a device bake equals, chunk for chunk, the one written by the drop-in bake (which
encodes on the host) from the same atlases."""
import ctypes as C
import json
import struct

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import _native as N
from lightbaker_b200 import scenes

pytestmark = pytest.mark.gpu


def chunks(data: bytes) -> dict:
    assert data[:4] == b"LBAK"
    n = struct.unpack_from("<I", data, 8)[0]
    head = json.loads(data[12:12 + n])
    base = (12 + n + 7) // 8 * 8
    return {c["name"]: data[base + c["offset"]:base + c["offset"] + c["length"]] for c in head["chunks"]}, head


def test_rgb9e5_device_equals_host_at_every_exponent_edge(gpu):
    """The exponent is floor(log2 m) as the C library's log2f rounds it: for a few floats just below each power
    of two that is the next exponent. Every float within 64 ulps of each power of two from 2^-27 to 2^16, the
    clamps, zero and random colours."""
    import torch
    vals = []
    for e in range(-27, 17):
        b = np.float32(2.0 ** e).view(np.uint32)
        vals.extend((np.arange(int(b) - 64, int(b) + 65, dtype=np.uint32)).view(np.float32).tolist())
    vals += [0.0, -1.0, 65408.0, 65407.99, 70000.0, 1e30, 5.960464477539063e-08]
    rng = np.random.default_rng(3)
    v = np.array(vals, np.float32)
    rgb = np.zeros((len(v) + 4000, 4), np.float32)
    rgb[:len(v), 0] = v
    rgb[:len(v), 1] = v * np.float32(0.5)
    rgb[:len(v), 2] = np.roll(v, 7)
    rgb[len(v):, :3] = (rng.lognormal(0, 3, (4000, 3))).astype(np.float32)
    d_in = torch.from_numpy(rgb).cuda()
    d_out = torch.zeros(len(rgb), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().lb_rgb9e5_device(gpu.handle, d_in.data_ptr(), len(rgb), d_out.data_ptr()), "lb_rgb9e5_device")
    gpu.sync()
    dev = d_out.cpu().numpy().view(np.uint32)
    host = np.array([lb.rgb9e5(c[:3]) for c in rgb], np.uint32)
    bad = np.nonzero(dev != host)[0]
    assert len(bad) == 0, [(rgb[i, :3].tolist(), hex(dev[i]), hex(host[i])) for i in bad[:5]]


@pytest.mark.parametrize("name", ["small_map", "map_100m"])
def test_device_encoded_file_equals_host_encoded(gpu, name):
    s = scenes.WORKLOADS[name]()
    dev = lb.bake_device(s, gpu)
    plain = lb.bake(s, gpu)
    assert dev.device_encoded and not plain.device_encoded
    a, ha = chunks(dev.write())
    b, hb = chunks(plain.write())
    assert sorted(a) == sorted(b) and "volume" in a
    for k in a:
        assert a[k] == b[k], f"chunk {k} differs"
    assert ha["volume"] == hb["volume"] and ha["atlas"] == hb["atlas"]
