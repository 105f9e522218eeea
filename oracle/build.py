"""TEST INFRASTRUCTURE: builds the C oracle (``oracle/liboracle_us3d.so``) with gcc.

Plain IEEE arithmetic (-O2, no -ffast-math, -ffp-contract=off) and OpenMP for the
multi-core CPU baseline. Usage: python oracle/build.py
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_us3d.so"
SOURCES = sorted(HERE.glob("*_oracle.c"))


def build(force: bool = False) -> Path:
    deps = SOURCES + sorted(HERE.glob("*_oracle_impl.h"))
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           *map(str, SOURCES), "-lm", "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
