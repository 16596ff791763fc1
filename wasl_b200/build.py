"""Build libwasl_b200.so in the package directory (sm_100a, in-tree).

    python -m wasl_b200.build            # incremental
    python -m wasl_b200.build --clean
    python -m wasl_b200.build --checked  # libwasl_b200_checked.so: device index
                                         # checks on (WASL_DEVICE_CHECKS)

The checked build records an out-of-range element index read from mesh data
in the handle's error word instead of faulting (euler_device.cuh,
checked_index); load it with WASL_B200_LIBRARY=<path> in place of the
ordinary one.

Kernels whose results must match the reference bit for bit are compiled with
--fmad=false (no fused multiply-add contraction); host code with
-ffp-contract=off for the same reason.  The mixed-precision kernels keep FMA.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwasl_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++20", "-lineinfo", f"-I{INCLUDE}", f"-I{CSRC}",
          "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"]

# file -> extra flags
SOURCES = {
    "euler_tri_f64.cu": ["--fmad=false"],
    # FP32 here carries only perturbations around FP64 means: approximate
    # division/square root and flushed denormals cost nothing in accuracy.
    "euler_tri_mixed.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "euler_tri_solver.cu": [],
    "line_f64.cu": ["--fmad=false"],
    "scalar_tri_f64.cu": ["--fmad=false"],
    "line_solver.cu": [],
    "scalar_tri_solver.cu": [],
    "mesh.cpp": [],
    "tables.cpp": [],
    "capi.cpp": [],
    "profiling.cpp": [],
    "cfl_static.cu": [],
    "autotune.cpp": [],
    "tri_setup.cpp": [],
    "batch_solver.cu": [],
    "capi_batch.cpp": [],
    "mlp.cu": [],
    "mlp_trainer.cpp": [],
    "setup_device.cu": ["--fmad=false"],
    "halo.cu": [],
}
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]


def _newest_header() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "wasl_b200.h")]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, flags: list[str], build_dir: str = BUILD) -> str:
    obj = os.path.join(build_dir, src + ".o")
    path = os.path.join(CSRC, src)
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
            and os.path.getmtime(obj) >= _newest_header()):
        return obj
    lang = [] if src.endswith(".cu") else ["-x", "cu"]
    cmd = [NVCC, *ARCH, *COMMON, *flags, *lang, "-c", path, "-o", obj]
    subprocess.run(cmd, check=True)
    return obj


def build(clean: bool = False, verbose: bool = False, checked: bool = False) -> str:
    build_dir = BUILD + ("_checked" if checked else "")
    lib = LIB.replace(".so", "_checked.so") if checked else LIB
    extra = ["-DWASL_DEVICE_CHECKS"] if checked else []
    if clean and os.path.isdir(build_dir):
        shutil.rmtree(build_dir)
    os.makedirs(build_dir, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        futures = [pool.submit(_compile, s, f + extra, build_dir) for s, f in SOURCES.items()]
        objs = [f.result() for f in futures]
    if (not os.path.exists(lib) or
            max(os.path.getmtime(o) for o in objs) > os.path.getmtime(lib)):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", lib, *objs, "-ldl"], check=True)
    if verbose:
        print(lib)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--checked", action="store_true", help="device index checks on")
    args = ap.parse_args()
    build(clean=args.clean, verbose=True, checked=args.checked)
    sys.exit(0)
