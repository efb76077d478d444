"""Builds the engine's shared library in-tree: rovaca_b200/libphmm_b200.so.

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``) with
flush-to-zero single precision (the reference runs with MXCSR.FTZ set) and IEEE division; host
sources with g++.  Objects go to rovaca_b200/_build/ and are rebuilt only when a source or header
is newer.  Usage: ``python -m rovaca_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libphmm_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-ftz=true", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
             f"-I{CUDA_HOME / 'include'}"]

CU_SOURCES = ["phmm_kernels.cu", "phmm_fwd32_m0.cu", "phmm_fwd32_m1.cu", "phmm_fwd32_m2.cu", "phmm_engine.cu",
              "phmm_noalloc.cu", "phmm_regionk.cu", "phmm_sw.cu"]
CPP_SOURCES = ["phmm_tables.cpp", "phmm_plan.cpp", "phmm_capi.cpp", "phmm_serve.cpp", "phmm_region.cpp",
               "phmm_tune.cpp", "phmm_multi.cpp"]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *headers])


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles (incrementally) and links libphmm_b200.so; returns its path."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append([NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    for s in CPP_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"], verbose)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
