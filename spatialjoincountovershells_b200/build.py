"""Build the native parts of the package in-tree.

    lib/libsjcs.so        CUDA kernels + the C ABI of include/sjcs.h (sm_100a only)
    lib/libsjcs_host.so   host formats and generators of include/sjcs_host.h
    bin/sjcs_rcount       the astr_rcount-compatible driver

Run ``python -m spatialjoincountovershells_b200.build`` (or call ``build()``).
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
LIB = PKG / "lib"
BIN = PKG / "bin"
INCLUDE = ROOT / "include"

CUDA_SOURCES = [
    "sjcs_abi.cu", "index_build.cu", "learned_index.cu", "query_prep.cu", "shell_count.cu", "morton_count.cu",
    "scan.cu", "serve.cu", "decode.cu", "noalloc.cu",
]
HOST_SOURCES = ["sjcs_io.c", "sjcs_gen.c"]

# Exact fp32 semantics: no fast-math, no FMA contraction anywhere (the
# parity-critical arithmetic also uses __fmul_rn/__fadd_rn/__fsub_rn).
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "-shared",
]
CC_FLAGS = ["-std=gnu11", "-O2", "-ffp-contract=off", "-fPIC", "-Wall", "-Wno-unused-parameter"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libsjcs.so")


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose: bool) -> None:
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, force: bool = False) -> dict:
    LIB.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    out = {}
    cu = [CSRC / s for s in CUDA_SOURCES]
    cu_deps = cu + list(CSRC.glob("*.cuh")) + [INCLUDE / "sjcs.h"]
    libsjcs = LIB / "libsjcs.so"
    if force or _stale(libsjcs, cu_deps):
        tmp = libsjcs.with_suffix(".so.tmp")
        _run([_nvcc(), *NVCC_FLAGS, "-o", tmp, *cu], verbose)
        os.replace(tmp, libsjcs)
    out["libsjcs"] = libsjcs

    hs = [HOST / s for s in HOST_SOURCES]
    host_deps = hs + [INCLUDE / "sjcs_host.h"]
    libhost = LIB / "libsjcs_host.so"
    if force or _stale(libhost, host_deps):
        tmp = libhost.with_suffix(".so.tmp")
        _run(["gcc", *CC_FLAGS, "-shared", "-o", tmp, *hs, "-lm", "-pthread"], verbose)
        os.replace(tmp, libhost)
    out["libsjcs_host"] = libhost

    drv = BIN / "sjcs_rcount"
    drv_src = [HOST / "sjcs_rcount.c", *hs]
    if force or _stale(drv, drv_src + [libsjcs, INCLUDE / "sjcs.h", INCLUDE / "sjcs_host.h"]):
        tmp = BIN / "sjcs_rcount.tmp"
        _run(["gcc", *[f for f in CC_FLAGS if f != "-fPIC"], "-o", tmp, *drv_src,
              f"-L{LIB}", "-lsjcs", "-Wl,-rpath,$ORIGIN/../lib", "-lm", "-pthread"], verbose)
        os.replace(tmp, drv)
    out["sjcs_rcount"] = drv
    return out


if __name__ == "__main__":
    res = build(verbose=True, force="--force" in sys.argv)
    for k, v in res.items():
        print(f"{k}: {v}")
