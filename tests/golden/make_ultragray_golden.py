"""Generates tests/golden/ultragray_*.npz from the reference's own UltraGray CUDA build
(oracle/_ref/ultragray_ref_C*.so, built by oracle/build_ref.py; the reference tree lacks the
covariance header its shader includes, so that build uses oracle/ref_shim/covariance.cuh).

Inputs are seeded probe scenes (tests/ugr_helpers.make_scene); outputs are what the
reference's MapperForwardCUDA, ShaderForwardCUDA and ShaderBackwardCUDA return for them,
with explicit ray perturbations (the values the reference's autograd function draws per
call). Usage on a GPU machine from the repository root:
    python tests/golden/make_ultragray_golden.py [--out tests/golden]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests"), str(ROOT / "ultrasound-3d-reconstruction_b200"),
                str(ROOT / "oracle" / "_ref")]

import ultragray_ref_C as REF  # noqa: E402
from ugr_helpers import make_scene, run_reference_ugr  # noqa: E402

# name: (G, W, H, seed, extra make_scene arguments)
CASES = {
    "small": (600, 48, 40, 0, {}),
    "tilted": (900, 40, 56, 1, dict(tilted=True, elev_cut=0.5, wr=1.5)),
    "local": (1200, 52, 60, 2, dict(local=True, maxwin=6.0, depth_mm=50.0)),
    "nowindow": (500, 33, 37, 3, dict(wr=0.0, ops_max_offset_mm=1.0)),
}


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=Path(__file__).resolve().parent)
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    dev = torch.device("cuda")
    for name, (G, W, H, seed, kw) in CASES.items():
        scene = make_scene(G, W, H, seed, **kw)
        ref = run_reference_ugr(REF, scene, dev)
        d = {k: v for k, v in scene.items()}
        d.update(ref)
        np.savez_compressed(a.out / f"ultragray_{name}.npz", **d)
        print(name, int(ref["ref_counts"].sum()), {k: v.shape for k, v in ref.items()})


if __name__ == "__main__":
    main()
