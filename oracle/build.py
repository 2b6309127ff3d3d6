"""ORACLE build recipe — test infrastructure only.

Compiles the CPU restatement (trace_ref.cpp, filter_ref.cpp, bake_ref.cpp, bvh_ref.cpp) into oracle/liboracle.so with g++
-O2 -ffp-contract=off -fopenmp: no fused multiply-add, so every float operation rounds in the order the
shader's source gives it. The reference itself (Rust + wgpu) cannot be built here: there is no Rust
toolchain and no graphics stack, so there is no oracle/_ref.

    python oracle/build.py
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "liboracle.so"
SRCS = [HERE / "trace_ref.cpp", HERE / "filter_ref.cpp", HERE / "bake_ref.cpp", HERE / "bvh_ref.cpp"]
DEPS = SRCS + [HERE / "oracle.h", HERE.parent / "include" / "lightbaker.h"]


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= max(p.stat().st_mtime for p in DEPS):
        return OUT
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-Wall",
           *map(str, SRCS), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
