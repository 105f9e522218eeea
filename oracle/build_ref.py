"""TEST INFRASTRUCTURE: compiles the reference's own renderer CUDA extensions, unmodified,
from the reference tree for sm_100a, into ``oracle/_ref/`` (git-ignored; they travel to the
GPU machine with the repository snapshot and are used only by tests as parity checkers).

Recipe: nvcc on each renderer's .cu files and g++ on its bindings, with the reference's own
nvcc flags (its setup.py files: -O3 --use_fast_math -lineinfo
-DTHRUST_IGNORE_CUB_VERSION_CHECK; the UltraGS rasteriser adds its vendored GLM include
directory and needs ``-include cstdint``), plus ``oracle/ref_shim`` for the helper headers
the reference tree does not contain (math_utils.cuh, load_utils.cuh, and UltraGray's
covariance.cuh, whose four functions are defined there from the mathematics their call
sites imply). Two harnesses in ``oracle/ref_harness`` expose internal binning results.
The reference's setup.py files are not run.

Usage: python oracle/build_ref.py [--reference /path/to/reference]  (default: $US3D_REFERENCE)
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
SHIM = HERE / "ref_shim"
# The reference checkout: $US3D_REFERENCE, else the path this machine keeps it at.
DEFAULT_REFERENCE = Path(os.environ.get("US3D_REFERENCE") or "/root/reference")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# module name -> (renderer directory, sources relative to it, extra nvcc flags)
MODULES = {
    "ultragauss_ref_C": (
        "ops/ultragauss_renderer",
        ["src/mapper/wrapper_mapper.cu", "src/mapper/core.cu", "src/shader/wrapper_shader.cu",
         "src/shader/forward.cu", "src/shader/backward.cu", "src/bindings.cpp"],
        ["-O3", "--use_fast_math", "-lineinfo", "-DTHRUST_IGNORE_CUB_VERSION_CHECK"],
    ),
    "gaussianplie_ref_C": (
        "ops/gaussianplie_renderer",
        ["src/bindings.cpp", "src/mapper/core_tile.cu", "src/mapper/core_pixel.cu", "src/shader/forward.cu",
         "src/shader/backward.cu", "src/shader/plane_cond2d.cu", "src/shader/us_focus.cu",
         "src/shader/wrapper_shader.cu"],
        ["-O3", "--use_fast_math", "-lineinfo", "-DTHRUST_IGNORE_CUB_VERSION_CHECK"],
    ),
    "ultragray_ref_C": (
        "ops/ultragray_renderer",
        ["src/bindings.cpp", "src/mapper/wrapper_mapper.cu", "src/mapper/core.cu", "src/shader/wrapper_shader.cu",
         "src/shader/forward.cu", "src/shader/backward.cu"],
        ["-O3", "--use_fast_math", "-lineinfo", "-DTHRUST_IGNORE_CUB_VERSION_CHECK"],
    ),
    "ultrags_ref_C": (
        "ops/ultrags_baseline_renderer",
        ["cuda_rasterizer/rasterizer_impl.cu", "cuda_rasterizer/forward.cu", "cuda_rasterizer/backward.cu",
         "rasterize_points.cu", "ext.cpp"],
        ["-O3", "--use_fast_math", "-lineinfo", "-DTHRUST_IGNORE_CUB_VERSION_CHECK", "-include", "cstdint",
         "-I{root}/third_party/glm"],
    ),
    "slice_adapted_ref_C": (
        "ops/slice_adapted_3dgs_renderer",
        ["src/bindings.cpp", "src/render.cu"],
        ["-O3", "--use_fast_math", "-lineinfo"],
    ),
    # The reference's render.cu included by oracle/ref_harness/slice_adapted_bins.cu, which
    # exposes its internal tile binning.
    "slice_adapted_ref_bins": (
        "ops/slice_adapted_3dgs_renderer",
        ["HARNESS:slice_adapted_bins.cu"],
        ["-O3", "--use_fast_math", "-lineinfo"],
    ),
    # The reference's mapper kernels plus oracle/ref_harness/ultragauss_keys.cu, which runs
    # them the way MapperForwardCUDA does and returns its private sorted keys and ranges.
    "ultragauss_ref_keys": (
        "ops/ultragauss_renderer",
        ["src/mapper/core.cu", "HARNESS:ultragauss_keys.cu"],
        ["-O3", "--use_fast_math", "-lineinfo", "-DTHRUST_IGNORE_CUB_VERSION_CHECK"],
    ),
}


def _torch_flags():
    import torch
    from torch.utils import cpp_extension as ce

    inc = ce.include_paths(device_type="cuda") + [sysconfig.get_paths()["include"]]
    libdirs = ce.library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return inc, libdirs, abi


def _plan(name: str, reference: Path):
    """Compile commands (source -> object) and the link command of one module."""
    rdir, srcs, nvflags = MODULES[name]
    root = reference / rdir
    nvflags = [f.replace("{root}", str(root)) for f in nvflags]
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = OUT_DIR / f"{name}{suffix}"
    obj_dir = OUT_DIR / f"obj_{name}"
    inc, libdirs, abi = _torch_flags()
    defs = [f"-DTORCH_EXTENSION_NAME={name}", "-DTORCH_API_INCLUDE_EXTENSION_H", f"-D_GLIBCXX_USE_CXX11_ABI={abi}"]
    incs = ["-I", str(root / "include"), "-I", str(root / "src"), "-I", str(SHIM)] + [x for p in inc for x in ("-I", p)]
    compiles, objs = [], []
    for s in srcs:
        src = (HERE / "ref_harness" / s.split(":", 1)[1]) if s.startswith("HARNESS:") else root / s
        obj = obj_dir / (s.replace("/", "_").replace(":", "_") + ".o")
        if s.endswith(".cu"):
            cmd = ["nvcc", "-c", str(src), "-o", str(obj), *ARCH, *nvflags, "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", *defs, *incs]
        else:
            cmd = ["g++", "-c", str(src), "-o", str(obj), "-O3", "-std=c++17", "-fPIC", "-include", "cstdint", *defs,
                   *incs, *[f for f in nvflags if f.startswith("-I")]]
        compiles.append(cmd)
        objs.append(str(obj))
    link = ["g++", "-shared", "-o", str(out), *objs]
    for d in libdirs:
        link += ["-L", d, f"-Wl,-rpath,{d}"]
    link += ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python", "-lcudart"]
    return out, obj_dir, compiles, objs, link


def _run_plans(plans, jobs: int) -> None:
    from concurrent.futures import ThreadPoolExecutor

    for _, obj_dir, _, _, _ in plans:
        obj_dir.mkdir(parents=True, exist_ok=True)
    cmds = [c for plan in plans for c in plan[2]]
    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for f in [ex.submit(subprocess.run, c, check=True) for c in cmds]:
            f.result()
    for out, obj_dir, _, objs, link in plans:
        subprocess.run(link, check=True)
        for o in objs:
            os.remove(o)
        obj_dir.rmdir()


def build_module(name: str, reference: Path, force: bool = False, jobs: int = 0) -> Path:
    plan = _plan(name, reference)
    if plan[0].exists() and not force:
        return plan[0]
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    _run_plans([plan], jobs or os.cpu_count() or 1)
    return plan[0]


def build_all(reference: Path = DEFAULT_REFERENCE, force: bool = False, jobs: int = 0) -> list[Path]:
    """Builds every module; the translation units of all modules compile in parallel."""
    if not reference.exists():
        return []
    plans = [_plan(n, reference) for n in MODULES]
    todo = [p for p in plans if force or not p[0].exists()]
    if todo:
        OUT_DIR.mkdir(parents=True, exist_ok=True)
        _run_plans(todo, jobs or os.cpu_count() or 1)
    return [p[0] for p in plans]


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for p in build_all(a.reference, a.force):
        print(p)
