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
