"""Build libacgpu.so (sm_100a) in-tree: laplacians.jl_b200/acgpu/libacgpu.so.

    python laplacians.jl_b200/build.py [--force]

Host C++ (the elimination, the Julia-compatible random stream, the C ABI) and
the CUDA kernels are compiled by nvcc into one shared library that exports
the symbols declared in include/acgpu.h.  The host part alone (the "host"
sections of include/acgpu.h: random stream, elimination, LDLinv files) is
also linked into libacghost.so, which needs no CUDA runtime: a CPU-only
caller (the benchmark's reference arm) builds factors with it without
mapping the GPU library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "acgpu" / "libacgpu.so"
HOST_OUT = PKG / "acgpu" / "libacghost.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["acg_solver.cu"]
CPP_SOURCES = ["acg_rng.cpp", "acg_factor.cpp", "acg_factor_par.cpp", "acg_host_api.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.cpp")) + list(CSRC.glob("*.h"))
    deps.append(ROOT / "include" / "acgpu.h")
    deps.append(Path(__file__))
    return deps


def up_to_date() -> bool:
    if not OUT.exists() or not HOST_OUT.exists():
        return False
    t = min(OUT.stat().st_mtime, HOST_OUT.stat().st_mtime)
    return all(p.stat().st_mtime <= t for p in _sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
    for src in CPP_SOURCES:
        obj = objdir / (src + ".o")
        cmd = [NVCC, *common, "-Xcompiler", "-ffp-contract=off", "-x", "c++", "-c", str(CSRC / src), "-o", str(obj)]
        _run(cmd, verbose)
        objs.append(obj)
    host_tmp = HOST_OUT.with_suffix(".so.tmp")
    _run([NVCC, "-shared", "-o", str(host_tmp), *map(str, objs)], verbose)
    os.replace(host_tmp, HOST_OUT)
    for src in CU_SOURCES:
        obj = objdir / (src + ".o")
        cmd = [NVCC, *common, *GENCODE, "-lineinfo", "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v", "-Wno-deprecated-gpu-targets"]
        _run(cmd, verbose)
        objs.append(obj)
    tmp = OUT.with_suffix(".so.tmp")
    _run([NVCC, "-shared", *GENCODE, "-o", str(tmp), *map(str, objs), "-lcudart"], verbose)
    os.replace(tmp, OUT)
    return OUT


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose="-v" in sys.argv))
