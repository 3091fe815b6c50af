"""Build libacfd_gpu.so in-tree with nvcc for sm_100a.

Usage: python -m artracfd_b200.build [--verbose]

Each translation unit gets its own floating-point contraction setting:
the units that must reproduce the reference bit for bit (exact FP64 sweeps,
boundary fill and CFL, immersed-boundary geometry) are compiled with
--fmad=false; the fast FP64 and FP32 sweeps with FMA contraction, the FP32
sweeps also with approximate FP32 square root and division.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libacfd_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                 "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# unit -> extra flags
UNITS = {
    "acfd_api.cu": [],
    "boundary.cu": ["--fmad=false"],
    "cfl_noalloc.cu": ["--fmad=false"],
    "ib.cu": ["--fmad=false"],
    "sweep_exact.cu": ["--fmad=false"],
    "sweep_fast.cu": [],
    # FP32 bulk and hybrid forms: no bitwise bar (their error against the FP64
    # form is measured), so FP32 square roots and divisions use the hardware
    # approximations and denormals flush to zero (issue-bound kernels)
    "sweep_fp32.cu": ["-prec-sqrt=false", "-prec-div=false", "-ftz=true"],
    "sensor.cu": [],
}


def _deps_newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "acfd.h"))
    jobs = []
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        objs.append(obj)
        if _deps_newer(obj, [src, __file__] + headers) or ptxas_info:
            cmd = [NVCC] + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=min(8, len(jobs) or 1)) as ex:
        outs = list(ex.map(run, jobs))
    if ptxas_info:
        for o in outs:
            sys.stdout.write(o)
    if jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        run(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
