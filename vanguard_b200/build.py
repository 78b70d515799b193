"""Build the in-tree CUDA library vanguard_b200/libvanguard_slic.so for sm_100a.

Each translation unit is compiled by nvcc with its own floating-point contract:
  slic_fp64*.cu -fmad=false  (exact FP64: no FMA contraction, bitwise parity with the reference; one unit per
                             model family so that ptxas runs on them in parallel)
  slic_mixed.cu -fmad=true   (mixed FP32/FP64 form)
  adjoint.cu    -fmad=true   (derivatives; the operands of the forward's branches use explicit __d*_rn operations)
  source_batch.cu -fmad=false (the HPR source batch: its forward equals the reference's forcing step)
  source_adjoint.cu -fmad=true (its reverse pass)
  *.cu (rest)   host code and helpers
The objects are linked into one shared library with the CUDA runtime linked statically, so the library
only depends on the driver.  Run `python -m vanguard_b200.build` or call build().
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libvanguard_slic.so")
OBJDIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math", "-ccbin", "g++"]

# (source, extra flags)
UNITS = [
    ("slic_fp64.cu", ["-fmad=false"]),
    ("slic_fp64_euler.cu", ["-fmad=false"]),
    ("slic_fp64_mhd.cu", ["-fmad=false"]),
    ("slic_fp64_hpr.cu", ["-fmad=false"]),
    ("slic_fp64_hpr_solid.cu", ["-fmad=false"]),
    ("slic_fp64_hpr_two.cu", ["-fmad=false"]),
    ("slic_mixed.cu", ["-fmad=true"]),
    ("vg_api.cu", []),
    ("vg_noalloc.cu", ["-fmad=false"]),
    ("batch.cu", ["-fmad=false"]),
    ("adjoint.cu", ["-fmad=true"]),
    ("source_batch.cu", ["-fmad=false"]),
    ("source_adjoint.cu", ["-fmad=true"]),
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "vanguard_slic.h"))
    return [h for h in hs if os.path.exists(h)]


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every CUDA unit for sm_100a and link libvanguard_slic.so; returns its path."""
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    headers = _headers()
    objs, jobs = [], []
    for src, flags in UNITS:  # the units are independent: compile the stale ones concurrently
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            jobs.append((cmd, o, subprocess.Popen(cmd, env=env)))
    failed = [cmd for cmd, o, p in jobs if p.wait() != 0]
    if failed:
        for cmd, o, p in jobs:  # a failed unit must not leave a stale object that looks current
            if p.returncode != 0 and os.path.exists(o):
                os.remove(o)
        raise subprocess.CalledProcessError(1, failed[0])
    if force or _stale(OUT, objs):
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-ccbin", "g++", "-o", OUT, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
    build_shim(verbose=verbose, force=force)
    return OUT


SHIM_DIR = os.path.join(HERE, "shim")
SHIM_OUT = os.path.join(HERE, "libvanguard_shim.so")
DRIVER_SRC = os.path.join(os.path.dirname(HERE), "tests", "shim", "shim_driver.cpp")
DRIVER_OUT = os.path.join(os.path.dirname(HERE), "tests", "shim", "shim_driver")


def build_shim(verbose: bool = False, force: bool = False) -> str:
    """The drop-in C++ surface (libvanguard_shim.so, the reference's class names over the C ABI) and the
    Vanguard-style test caller tests/shim/shim_driver, both with g++ and an $ORIGIN-relative rpath."""
    env = dict(os.environ)
    env.pop("CXX", None)
    src = os.path.join(SHIM_DIR, "vanguard_shim.cpp")
    hdrs = [os.path.join(SHIM_DIR, "vanguard_shim.h"), os.path.join(os.path.dirname(HERE), "include", "vanguard_slic.h")]
    if force or _stale(SHIM_OUT, [src, OUT] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-o", SHIM_OUT, src, "-L" + HERE,
               "-lvanguard_slic", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
    if os.path.exists(DRIVER_SRC) and (force or _stale(DRIVER_OUT, [DRIVER_SRC, SHIM_OUT] + hdrs)):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I" + SHIM_DIR, "-o", DRIVER_OUT, DRIVER_SRC, "-L" + HERE,
               "-lvanguard_shim", "-lvanguard_slic", "-Wl,-rpath," + "$ORIGIN/../../vanguard_b200"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True, env=env)
    return SHIM_OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
