"""Generates tests/golden/ultrags_*.npz from the reference's own UltraGS-baseline CUDA build
(oracle/_ref/ultrags_ref_C*.so, built by oracle/build_ref.py).

Inputs are seeded camera scenes (tests/gs_helpers.make_scene); outputs are what the
reference's rasterize_gaussians / rasterize_gaussians_backward return, plus its internal
binning and compositing state decoded from the geometry / binning / image byte buffers it
returns. Usage on a GPU machine from the repository root:
    python tests/golden/make_ultrags_golden.py [--out tests/golden]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests"), str(ROOT / "ultrasound-3d-reconstruction_b200"),
                str(ROOT / "oracle" / "_ref")]

import ultrags_ref_C as REF  # noqa: E402
from gs_helpers import CASES, build_case  # noqa: E402


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    dev = torch.device("cuda")
    for name in CASES:
        scene, ref = build_case(REF, name, dev)
        d = dict(scene)
        d.update(ref)
        np.savez_compressed(a.out / f"ultrags_{name}.npz", **d)
        print(name, int(ref["ref_num"]), {k: v.shape for k, v in ref.items() if not k.startswith("ref_state")})


if __name__ == "__main__":
    main()
