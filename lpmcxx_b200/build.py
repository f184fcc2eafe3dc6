"""Build recipe for liblpm_b200.so (sm_100a) -- compiled in-tree with nvcc / g++.

    python -m lpmcxx_b200.build          # or: from lpmcxx_b200.build import build_library

CUDA sources are compiled for sm_100a only; host C++ (the mesh generator) is compiled with
-ffp-contract=off so that its floating-point results match the reference's bit for bit.
Objects go to lpmcxx_b200/_build/ and the library to lpmcxx_b200/liblpm_b200.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblpm_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-Xptxas", "-warn-spills"] + ARCH
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall"]


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    if proc.stdout.strip():
        sys.stderr.write(proc.stdout)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted((PKG.parent / "include").glob("*.h"))
    objs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC, *NVFLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    for src in sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, [src] + headers):
            cmd = [CXX, *CXXFLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    print(build_library(verbose=True, force="--force" in sys.argv))
