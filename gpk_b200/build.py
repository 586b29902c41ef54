"""Builds gpk_b200/libgpk_b200.so in-tree with nvcc for sm_100a.

The CUDA sources are compiled with -fmad=false so that no multiply-add is
contracted into an FMA: with IEEE division/square root (nvcc's defaults) and
no flush-to-zero, float arithmetic written in the reference's operand order
rounds exactly like the reference's x86-64 SSE build.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpk_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-ftz=false", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp,-O2"]
SOURCES = ["gpk_capi.cu", "gpk_step.cu", "gpk_geometry.cu", "gpk_local.cu", "gpk_topology.cu", "gpk_spectral.cu",
           "gpk_batch.cu", "gpk_adjoint.cu", "gpk_init_dev.cu", "gpk_alcu.cu", "gpk_init.cpp", "gpk_core_shim.cpp"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _obj(src: str) -> str:
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _deps() -> list:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(HERE, "..", "include")
    files += [os.path.join(inc, f) for f in os.listdir(inc)]
    return files


def _stale(target: str, deps: list) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, extra: list) -> str:
    out = _obj(src)
    cmd = [_nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return out


def build(force: bool = False, verbose: bool = False, extra: list | None = None) -> str:
    """Compile every CUDA source for sm_100a and link the shared library."""
    extra = list(extra or [])
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), SOURCES))
    cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lgomp", "-lcufft", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
