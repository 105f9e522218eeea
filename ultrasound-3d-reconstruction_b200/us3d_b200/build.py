"""Build of the us3d_b200 CUDA library (sm_100a) with nvcc, in-tree.

The library is a plain C-ABI shared object (``lib/libus3d_b200.so``) loaded with ctypes;
no PyTorch headers are involved, so it builds in seconds without a GPU.
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT_DIR = PKG_DIR.parent  # ultrasound-3d-reconstruction_b200/
CSRC_DIR = ROOT_DIR / "csrc"
INCLUDE_DIR = ROOT_DIR.parent / "include"
LIB_PATH = PKG_DIR / "lib" / "libus3d_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3",
    "--use_fast_math",  # same floating-point mode as the reference kernels
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-shared",
]


def sources() -> list[Path]:
    return sorted(CSRC_DIR.glob("*.cu"))


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    deps = list(sources()) + list(CSRC_DIR.glob("*.cuh")) + list(INCLUDE_DIR.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every .cu under csrc/ into one shared library; returns its path."""
    if not force and not needs_build():
        return LIB_PATH
    LIB_PATH.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE_DIR), *map(str, sources()), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
