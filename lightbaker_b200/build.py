"""Builds the package's native library in-tree: lightbaker_b200/liblightbaker_b200.so.

CUDA sources (csrc/*.cu) are compiled by nvcc for sm_100a only, with -fmad=false so every float
operation rounds as the shader's source orders it; host sources (csrc/host/*.cpp) by g++ with
-ffp-contract=off for the same reason (the reference's Rust host code never contracts). The library
links the CUDA runtime statically; zlib is linked and zstd opened at run time.

    python -m lightbaker_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "liblightbaker_b200.so"
BUILD = HERE / "_build"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fopenmp", "--expt-relaxed-constexpr"]
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
CUDA_HOME = Path(NVCC).resolve().parent.parent
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
             f"-I{CUDA_HOME / 'include'}"]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    headers = sorted(CSRC.rglob("*.h")) + sorted(CSRC.rglob("*.cuh")) + [HERE.parent / "include" / "lightbaker.h"]
    return cu, cpp, headers


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    cu, cpp, headers = _sources()
    newest_header = max((h.stat().st_mtime for h in headers if h.exists()), default=0)
    BUILD.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for src in cu + cpp:
        obj = BUILD / (src.stem + (".cu.o" if src.suffix == ".cu" else ".o"))
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if not stale:
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        else:
            cmd = [CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
        jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if force or jobs or not OUT.exists() or OUT.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = OUT.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              "-Xcompiler", "-fopenmp", "-lz", "-ldl", "-lpthread", "-lrt"])
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
