"""Build the CUDA shared library of the B200 MPM path, in tree.

Compiles every ``csrc/*.cu`` for sm_100a with nvcc into
``molla_b200/libmolla_mpm.so`` (static CUDA runtime, C ABI of
``include/molla_mpm.h``).  Object files go to ``molla_b200/_build/``;
unchanged sources are not recompiled.

Usage:  python -m molla_b200.build
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmolla_mpm.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    f"-I{ROOT / 'include'}",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build molla_b200")
    return cand


def _host_compiler() -> list[str]:
    # nvcc's host compiler: prefer the system g++ (matching libstdc++).
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if Path(gxx).exists() else []


def _needs(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    objs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _needs(obj, [src, *headers]):
            cmd = [nvcc, *_host_compiler(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _needs(LIB, objs):
        cmd = [nvcc, *_host_compiler(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt",
               "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-q" not in sys.argv)
    print(LIB)
