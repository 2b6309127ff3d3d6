"""The C ABI library: it loads without a GPU and exports every function include/lightbaker.h declares;
without a device it fails loudly, never substituting a CPU path."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "lightbaker.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(lb_[a-z0-9_]+)\s*\(", text))
    types = set(re.findall(r"typedef\s+struct\s+(lb_[a-z0-9_]+)", text))
    return sorted(names - types)


def test_exports_every_declared_symbol():
    from lightbaker_b200 import _native
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python declarations cover them
    assert not [n for n in names if n not in _native.SIGNATURES], [n for n in names if n not in _native.SIGNATURES]


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import lightbaker_b200 as lb
    with pytest.raises(lb.LightbakerError, match="no GPU"):
        lb.Gpu.new(0)


def _nodes(rows):
    from lightbaker_b200 import _native
    import numpy as np
    a = np.zeros(len(rows), _native.NODE)
    for i, (first, count) in enumerate(rows):
        a[i]["first"], a[i]["count"] = first, count
    return a


def _check(nodes, n_tris):
    from lightbaker_b200 import _native
    return _native.lib().lb_bvh_check(nodes.ctypes.data, len(nodes), n_tris), _native.last_error()


def test_bvh_check_accepts_the_reference_shapes():
    # an inner root and two leaves; the reference's empty BVH (one inner node, children past the array)
    assert _check(_nodes([(1, 0), (0, 2), (2, 2)]), 4)[0] == 0
    assert _check(_nodes([(0, 0)]), 1)[0] == 0
    # real builds
    import lightbaker_b200 as lb
    from lightbaker_b200 import scenes
    P = lb.prepare(scenes.reference_test())
    assert _check(P.nodes, len(P.tris))[0] == 0


def test_bvh_check_refuses_what_a_walk_could_loop_in():
    # a child pointing back at its parent (a cycle), a child before its parent, a node with two parents
    for rows, why in (([(1, 0), (0, 0), (3, 1)], "not a tree node"),
                      ([(3, 0), (0, 1), (1, 1), (1, 0), (2, 1)], "not a tree node"),
                      ([(1, 0), (3, 0), (3, 0), (0, 1), (1, 1)], "not a tree node"),
                      ([(1, 0), (0, 2), (2, 3)], "past the triangle array")):
        rc, msg = _check(_nodes(rows), 4)
        assert rc == -1 and why in msg, (rows, msg)
