"""Builds the drnum_b200 shared library (CUDA, sm_100a) in-tree.

    python -m drnum_b200.build            # -> drnum_b200/libdrnum_b200.so

Every CUDA translation unit is compiled for sm_100a only; the FP64 stage
kernel gets -fmad=false (bitwise parity with the reference CPU iterator), the
FP32 (fixed-point storage) kernel gets fast-math intrinsics without implicit
FMA contraction (duplicated border faces must round identically); the donor
copy, the host overlap set-up and the generic flux-functor schemes are built
without contraction too (weights, interpolated values and fluxes round like
the reference's).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdrnum_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
          "--expt-relaxed-constexpr"]

# translation unit -> extra flags
UNITS = {
    "dn_api.cu": ["-Xcompiler", "-ffp-contract=off"],
    "fv_fp64.cu": ["-fmad=false"],
    "fv_fx32.cu": ["-use_fast_math", "-fmad=false"],
    "dn_noalloc.cu": [],
    "dn_donor.cu": ["-fmad=false"],
    "dn_overlap.cpp": ["-Xcompiler", "-ffp-contract=off"],
    "dn_levelset.cpp": ["-Xcompiler", "-ffp-contract=off"],
    "dn_lsbc.cu": ["-fmad=false"],
    "fv_schemes.cu": ["-fmad=false"],
    "dn_gridio.cpp": [],
    "dn_exchange.cpp": [],
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _sources_newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "drnum_b200.h"))
    hs.append(os.path.join(INCLUDE, "drnum_b200_functor.cuh"))
    return hs


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    headers = _headers()

    def compile_one(unit: str) -> str:
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJDIR, os.path.splitext(unit)[0] + ".o")
        if _sources_newer(obj, [src, *headers]) or ptxas_info:
            cmd = [cc, *ARCH, *COMMON, *UNITS[unit], "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed for {unit}:\n{res.stdout}\n{res.stderr}")
            if ptxas_info:
                print(res.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(compile_one, UNITS))
    if _sources_newer(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    build_example()
    return LIB


EXAMPLE_SRC = os.path.join(HERE, "examples", "rusanov_stage.cu")
EXAMPLE_LIB = os.path.join(HERE, "examples", "libdn_example_stage.so")


def build_example(verbose: bool = False) -> str:
    """The example user stage function (a caller-written flux functor on
    include/drnum_b200_functor.cuh), as its own shared library."""
    deps = [EXAMPLE_SRC, os.path.join(INCLUDE, "drnum_b200.h"), os.path.join(INCLUDE, "drnum_b200_functor.cuh")]
    if _sources_newer(EXAMPLE_LIB, deps):
        cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-shared", "-Xcompiler", "-fPIC",
               "-I", INCLUDE, EXAMPLE_SRC, "-o", EXAMPLE_LIB]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"example build failed:\n{res.stdout}\n{res.stderr}")
    return EXAMPLE_LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
