"""Build recipe for the in-tree CUDA library ``libkennett_b200.so`` (sm_100a only).

``python -m seismicinversion_b200.build`` compiles every ``csrc/*.cu`` with nvcc for
``compute_100a/sm_100a`` into a single shared library next to this file.  nvcc
cross-compiles without a GPU.  The library links cuFFT dynamically and the CUDA runtime
statically.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libkennett_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libkennett_b200")
    return exe


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    cuda_lib = "/usr/local/cuda/lib64"
    cmd = [
        nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17",
        "-Xcompiler", "-fPIC", "-shared", "-I", str(INCLUDE),
        "-o", str(LIB), *map(str, sources()),
        "-L", cuda_lib, "-lcufft", "-Xlinker", f"-rpath,{cuda_lib}",
    ]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
