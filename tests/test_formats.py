"""Formats: the reference's encode known-answer tests (crates/lightbaker/src/encode.rs:150-180),
BLAKE3 against the published implementation, scene validation (scene.rs:140-201) and the .lbake
layout (output.rs:95-154, docs/FORMAT.md)."""
import json
import struct
import zlib

import numpy as np
import pytest

import lightbaker_b200 as lb
from lightbaker_b200 import scenes


def test_bc4_keeps_values_within_a_seventh():
    v = [(i * 13) % 256 for i in range(16)]
    b = lb.bc4_block(v)
    bits = int.from_bytes(b[2:8] + b"\0\0", "little")
    hi, lo = float(b[0]), float(b[1])
    for k, x in enumerate(v):
        i = (bits >> (3 * k)) & 7
        p = hi if i == 0 else lo if i == 1 else ((8 - i) * hi + (i - 1) * lo) / 7.0
        assert abs(p - x) <= (hi - lo) / 14.0 + 0.5


def test_rgb9e5_round_trips():
    for c in [[0.0, 0.0, 0.0], [1.0, 0.5, 0.25], [3.2, 0.01, 7.5], [0.001, 0.002, 0.0005]]:
        d = lb.rgb9e5_decode(lb.rgb9e5(c))
        m = max(c)
        for i in range(3):
            assert abs(d[i] - c[i]) <= m / 256.0 + 1e-6, (c, d)


def _blake3_py(data: bytes) -> bytes:
    """BLAKE3 (O'Connor, Aumasson, Neves, Wilcox-O'Hearn, 2020) from its specification, the incremental way:
    chunk chaining values pushed on a stack and merged as each subtree completes. Slow; for tests."""
    IV = [0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A, 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19]
    PERM = [2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8]
    M32 = 0xFFFFFFFF
    CHUNK_START, CHUNK_END, PARENT, ROOT = 1, 2, 4, 8

    def rotr(x, n):
        return ((x >> n) | (x << (32 - n))) & M32

    def g(v, a, b, c, d, x, y):
        v[a] = (v[a] + v[b] + x) & M32
        v[d] = rotr(v[d] ^ v[a], 16)
        v[c] = (v[c] + v[d]) & M32
        v[b] = rotr(v[b] ^ v[c], 12)
        v[a] = (v[a] + v[b] + y) & M32
        v[d] = rotr(v[d] ^ v[a], 8)
        v[c] = (v[c] + v[d]) & M32
        v[b] = rotr(v[b] ^ v[c], 7)

    def compress(cv, block, counter, blen, flags):
        m = list(struct.unpack("<16I", block.ljust(64, b"\0")))
        v = cv[:] + IV[:4] + [counter & M32, (counter >> 32) & M32, blen, flags]
        for r in range(7):
            g(v, 0, 4, 8, 12, m[0], m[1]); g(v, 1, 5, 9, 13, m[2], m[3])
            g(v, 2, 6, 10, 14, m[4], m[5]); g(v, 3, 7, 11, 15, m[6], m[7])
            g(v, 0, 5, 10, 15, m[8], m[9]); g(v, 1, 6, 11, 12, m[10], m[11])
            g(v, 2, 7, 8, 13, m[12], m[13]); g(v, 3, 4, 9, 14, m[14], m[15])
            m = [m[i] for i in PERM]
        return [v[i] ^ v[i + 8] for i in range(8)] + [v[i + 8] ^ cv[i] for i in range(8)]

    def chunk_output(chunk, counter):
        # (cv, last block, its length, flags) of a chunk, for the caller to finish
        cv = IV[:]
        blocks = [chunk[i:i + 64] for i in range(0, max(len(chunk), 1), 64)] or [b""]
        for i, blk in enumerate(blocks[:-1]):
            cv = compress(cv, blk, counter, 64, CHUNK_START if i == 0 else 0)[:8]
        last = blocks[-1]
        return cv, last, len(last), (CHUNK_START if len(blocks) == 1 else 0) | CHUNK_END, counter

    chunks = [data[i:i + 1024] for i in range(0, len(data), 1024)] or [b""]
    stack = []
    for k, ch in enumerate(chunks[:-1]):
        cv, last, blen, flags, ctr = chunk_output(ch, k)
        cur = compress(cv, last, ctr, blen, flags)[:8]
        total = k + 1
        while total & 1 == 0:
            cur = compress(IV, struct.pack("<16I", *(stack.pop() + cur)), 0, 64, PARENT)[:8]
            total >>= 1
        stack.append(cur)
    cv, block, blen, flags, ctr = chunk_output(chunks[-1], len(chunks) - 1)
    while stack:
        child = compress(cv, block, ctr, blen, flags)[:8]
        cv, block, ctr, blen, flags = IV, struct.pack("<16I", *(stack.pop() + child)), 0, 64, PARENT
    return struct.pack("<8I", *compress(cv, block, ctr, blen, flags | ROOT)[:8])


def test_blake3_matches_the_specification():
    """The library's one-call hash (its chunks in parallel and merged level by level from 64 KiB on) against
    the specification's incremental tree, across chunk and subtree boundaries."""
    assert _blake3_py(b"").hex().startswith("af1349b9f5f9a1a6a0404dea36dcc949")  # the published empty hash
    for n in [0, 1, 64, 1023, 1024, 1025, 3073, 65535, 65536, 65537, 65536 + 1024, 131072, 200003]:
        data = bytes((i * 31 + 7) % 256 for i in range(n))
        assert lb.blake3(data) == _blake3_py(data), n


def test_blake3_matches_published_implementation():
    blake3 = pytest.importorskip("blake3")
    for n in [0, 1, 63, 64, 65, 1023, 1024, 1025, 2048, 3073, 65537, 300001]:
        data = bytes((i * 31 + 7) % 256 for i in range(n))
        assert lb.blake3(data) == blake3.blake3(data).digest()


def _header():
    return json.loads(scenes.reference_test()[12:12 + struct.unpack("<I", scenes.reference_test()[8:12])[0]])


@pytest.mark.parametrize("mutate,message", [
    (lambda b: b"XXXX" + b[4:], "not a lightbaker scene"),
    (lambda b: b[:4] + struct.pack("<I", 2) + b[8:], "scene format 2"),
    (lambda b: b[:-8], "cut short"),
    (lambda b: b + b"\0\0\0\0", "bytes after the last mesh"),
])
def test_scene_read_errors(mutate, message):
    with pytest.raises(lb.LightbakerError, match=message):
        lb.prepare(mutate(scenes.reference_test()))


@pytest.mark.parametrize("patch,message", [
    (lambda h: h["lightmap"].update(atlasWidth=66), "atlasWidth"),
    (lambda h: h["lightmap"].update(indirectDownscale=3), "indirectDownscale"),
    (lambda h: h["bake"].update(sunSamples=15), "square"),
    (lambda h: h["bake"].update(aoRays=0), "aoRays"),
    (lambda h: h["bake"].update(bogus=1), "unknown field"),
    (lambda h: h["meshes"][0].update(material=9), "no material"),
    (lambda h: h["volume"].update(step=0.0), "volume"),
])
def test_scene_validation(patch, message):
    h = _header()
    patch(h)
    pos = []
    raw = scenes.reference_test()
    hl = struct.unpack("<I", raw[8:12])[0]
    at = (12 + hl + 3) & ~3
    for m in _header()["meshes"]:
        n = m["triangles"] * 9
        pos.append(np.frombuffer(raw[at:at + n * 4], np.float32))
        at = (at + n * 4 + 3) & ~3
    with pytest.raises(lb.LightbakerError, match=message):
        lb.encode_scene(h, pos)


def test_lbake_layout():
    import oracle
    t, keep = oracle.tracer()
    b = lb.bake_with(scenes.reference_test(), t)
    f = b.write()
    assert f[:4] == b"LBAK" and struct.unpack("<I", f[4:8])[0] == 1
    hl = struct.unpack("<I", f[8:12])[0]
    head = json.loads(f[12:12 + hl])
    base = (12 + hl + 7) // 8 * 8
    names = [c["name"] for c in head["chunks"]]
    assert names == ["direct", "indirect", "charts", "triangleCharts", "validity", "volume"]
    chunk = {c["name"]: f[base + c["offset"]: base + c["offset"] + c["length"]] for c in head["chunks"]}
    for c in head["chunks"]:
        assert c["offset"] % 8 == 0
    w, h = head["atlas"]["width"], head["atlas"]["height"]
    assert zlib.decompress(chunk["validity"], -15) == b.validity.tobytes()
    charts = np.frombuffer(zlib.decompress(chunk["charts"], -15), np.float32).reshape(-1, 8)
    assert np.array_equal(charts, b.charts)
    tri = np.frombuffer(zlib.decompress(chunk["triangleCharts"], -15), np.uint32)
    assert np.array_equal(tri, b.tri_charts)
    vol = zlib.decompress(chunk["volume"], -15)
    assert len(vol) == 16 * b.volume.shape[0]
    for name, vk, size in [("direct", 141, w * h), ("indirect", 123, 4 * b.indirect_size[0] * b.indirect_size[1])]:
        k = chunk[name]
        assert k[:12] == bytes([0xAB, 0x4B, 0x54, 0x58, 0x20, 0x32, 0x30, 0xBB, 0x0D, 0x0A, 0x1A, 0x0A])
        assert struct.unpack("<I", k[12:16])[0] == vk
        data_at, packed, raw = struct.unpack("<QQQ", k[80:104])
        assert raw == size
        pa = pytest.importorskip("pyarrow")
        got = pa.decompress(k[data_at:data_at + packed], decompressed_size=raw, codec="zstd")
        assert len(got) == raw
    assert head["baker"].startswith("lightbaker")
    assert head["stats"]["tilesBaked"] == b.stats.tiles_baked
