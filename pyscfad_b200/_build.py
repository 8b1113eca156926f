"""Builds the in-tree CUDA library pyscfad_b200/lib/libpyscfad_b200.so for sm_100a.

    python -m pyscfad_b200._build [--verbose]
    python -m pyscfad_b200._build --ffi <jaxlib include dir>   # XLA FFI handlers

Every .cu under pyscfad_b200/csrc is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared library exposing the C-ABI declared in include/pyscfad_b200.h.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpyscfad_b200.so")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = subprocess.run(cmd, capture_output=True, text=True)
            if verbose or r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}")
    need_link = force or not os.path.exists(LIB) or any(
        os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)
    if need_link:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        os.replace(tmp, LIB)
    return LIB


FFI_SRC = os.path.join(HERE, "ffi", "ct_xla_ffi.cc")
FFI_LIB = os.path.join(LIBDIR, "libpyscfad_b200_xla_ffi.so")


def build_ffi(xla_include: str) -> str:
    """Builds the XLA FFI handlers (ffi/ct_xla_ffi.cc) against jaxlib's headers
    (the directory holding xla/ffi/api/ffi.h), linked to the main library."""
    if not os.path.exists(os.path.join(xla_include, "xla", "ffi", "api", "ffi.h")):
        raise RuntimeError(f"xla/ffi/api/ffi.h not found under {xla_include}")
    lib = build()
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", xla_include, "-I", cuda_inc,
           "-I", os.path.join(ROOT, "include"), FFI_SRC, "-o", FFI_LIB, "-L", LIBDIR, "-lpyscfad_b200",
           "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("FFI build failed")
    return FFI_LIB


if __name__ == "__main__":
    if "--ffi" in sys.argv:
        print(build_ffi(sys.argv[sys.argv.index("--ffi") + 1]))
    else:
        build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
        print(LIB)
