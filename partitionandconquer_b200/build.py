"""Builds libpc.so in-tree: CUDA sources for sm_100a with nvcc, host C++ with g++.

The shared library is written next to this file so that it travels with the
source tree; object files go to ``_build/`` (not committed).  The build is
incremental: a translation unit is recompiled when it or any header of the
package (or ``include/``) is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libpc.so"
BIN = PKG / "bin"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-O3,-Wall,-Wno-unused-function",
    "-I", str(ROOT / "include"),
]
CXX = os.environ.get("PC_CXX", "g++")  # the system g++ (CXX may name a toolchain without libgomp)
CXX_FLAGS = ["-O3", "-fPIC", "-fopenmp", "-std=c++17", "-Wall", "-I", str(ROOT / "include")]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    return cu, cpp


def _headers():
    hs = list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.hpp"))
    hs += list((ROOT / "include").glob("*.h")) + list((ROOT / "include").glob("*.hpp"))
    return hs


def _stale(src: Path, obj: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles every CUDA and host source and links ``libpc.so``; returns its path."""
    BUILD.mkdir(exist_ok=True)
    cu, cpp = _sources()
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or ptxas_info or _stale(src, obj, newest_header):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + CUDA_FLAGS + extra + ["-c", str(src), "-o", str(obj)])
    for src in cpp:
        obj = BUILD / (src.stem + ".cpp.o")
        objs.append(obj)
        if force or _stale(src, obj, newest_header):
            jobs.append([CXX] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)])
    outputs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for out in ex.map(_run, jobs):
                outputs.append(out)
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-Xcompiler", "-fopenmp", "-lgomp"])
        os.replace(tmp, LIB)
    # command-line tools linked against the library (rpath to the package dir)
    BIN.mkdir(exist_ok=True)
    for src in sorted((CSRC / "tools").glob("*.cpp")):
        exe = BIN / src.stem
        if force or jobs or not exe.exists() or src.stat().st_mtime > exe.stat().st_mtime:
            _run([CXX, "-O3", "-std=c++17", "-Wall", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                  "-L", str(PKG), "-lpc", "-Wl,-rpath,$ORIGIN/.."])
    if verbose:
        for o in outputs:
            if o.strip():
                print(o)
    return LIB


if __name__ == "__main__":
    p = build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(p)
