"""Builds the native library libslimtracer_b200.so in-tree (sm_100a).

The CUDA kernels are compiled for B200 only (``-gencode
arch=compute_100a,code=sm_100a``) with ``-fmad=false``: the trace path
keeps the reference's floating-point operation order and fuses multiply-adds
only where the reference's sources call fast_mul_add (written as fmaf).
Host code is compiled with ``-ffp-contract=off`` for the same reason.

Usage: ``python -m slimtracincpp_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OUT_DIR = PKG / "_native"
LIB = OUT_DIR / "libslimtracer_b200.so"
BUILD_DIR = ROOT / "_build" / "slimtracer"

CUDA_SOURCES = ["api.cu", "kernels_fused.cu", "kernels_wavefront.cu", "kernels_refit.cu", "kernels_nrc.cu",
                "kernels_bake.cu"]
HOST_SOURCES = ["host_assets.cpp", "texture_baker.cpp"]
HEADERS = ["device_scene.h", "host_common.h", "kernels.h", "tracer_core.cuh", "nrc.h", "umma.cuh", "launch_count.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "--prec-div=true", "--prec-sqrt=true",
              "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", str(INCLUDE), "-I", str(CSRC)]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-I", str(INCLUDE),
             "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libslimtracer_b200")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}):\n{' '.join(map(str, cmd))}\n{res.stdout}\n{res.stderr}")
    if verbose and (res.stdout or res.stderr):
        print(res.stdout, res.stderr, flush=True)
    return res


def _source_digest() -> str:
    h = hashlib.sha256()
    for p in sorted([CSRC / f for f in CUDA_SOURCES + HOST_SOURCES + HEADERS] + [INCLUDE / "slimtracer_b200.h"]):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(ARCH + NVCC_FLAGS + CXX_FLAGS).encode())
    return h.hexdigest()


STAMP = OUT_DIR / "build.stamp"


def up_to_date() -> bool:
    """True when the library was built from exactly the current sources
    (content hash, so copies of the tree with fresh mtimes stay valid)."""
    return LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == _source_digest()


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    if not force and not ptxas_verbose and up_to_date():
        return LIB
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    common = [CSRC / h for h in HEADERS] + [INCLUDE / "slimtracer_b200.h", Path(__file__)]
    objects = []
    for src in CUDA_SOURCES:
        obj = BUILD_DIR / (src + ".o")
        objects.append(obj)
        if force or ptxas_verbose or _stale(obj, [CSRC / src] + common):
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", CSRC / src, "-o", obj], verbose or ptxas_verbose)
    for src in HOST_SOURCES:
        obj = BUILD_DIR / (src + ".o")
        objects.append(obj)
        if force or _stale(obj, [CSRC / src] + common):
            _run(["g++", *CXX_FLAGS, "-c", CSRC / src, "-o", obj], verbose)
    if force or _stale(LIB, objects):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objects, "-Xcompiler", "-fPIC"], verbose)
        os.replace(tmp, LIB)
    STAMP.write_text(_source_digest() + "\n")
    return LIB


def build_oracle(verbose: bool = False) -> Path:
    """Compiles the CPU oracle (test infrastructure) with its Makefile."""
    _run(["make", "-s", "-C", ROOT / "oracle"], verbose)
    return ROOT / "oracle" / "liboracle.so"


def build_reference(verbose: bool = False):
    """Compiles the reference's CPU path into oracle/_ref when its sources are
    present (they are only on the development machine); returns the library
    path or None."""
    script = ROOT / "oracle" / "build_ref.sh"
    src = Path(os.environ.get("SLIM_REFERENCE_SRC", "/root/reference/src"))
    if not (src / "slim").is_dir():
        lib = ROOT / "oracle" / "_ref" / "libslimref.so"
        return lib if lib.exists() else None
    _run(["bash", script], verbose)
    return ROOT / "oracle" / "_ref" / "libslimref.so"


if __name__ == "__main__":
    args = set(sys.argv[1:])
    lib = build(force="--force" in args, verbose="--verbose" in args, ptxas_verbose="--ptxas" in args)
    print(lib)
