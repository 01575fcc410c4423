"""Builds libvhlle_b200.so in-tree with nvcc for sm_100a.

    python -m vhlle_b200.build          # library only
    python -m vhlle_b200.build --check  # plus `-Xptxas -v` resource report

The kernels are FP64 and are compiled with -fmad=false: the reference is
compiled without FMA contraction, and keeping every multiply and add
separately rounded is what makes the device results bit-identical.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvhlle_b200.so")
SOURCES = ["vh_step.cu", "vh_capi.cu", "vh_noalloc.cu", "vh_surface.cu", "vh_vorticity.cu", "vh_mlp.cu",
           "vh_batch.cu", "vh_ic.cu", "vh_ic_ref.cu"]
HEADERS = ["vh_physics.cuh", "vh_step.cuh", "vh_surface.cuh", "vh_cornelius.cuh", "vh_mlp.cuh",
           "vh_ctx.cuh"]
DRIVER_SRC = os.path.join(HERE, "driver", "vhlle_run.cpp")
DRIVER = os.path.join(HERE, "driver", "vhlle_run")


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the system g++ (a wrapper on PATH may link libstdc++ statically)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def nvcc_flags(extra=()):
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
            "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
            "-I", os.path.join(ROOT, "include"), *extra]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "vhlle_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and not _stale() and not ptxas_v:
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        extra = ["-Xptxas", "-v"] if ptxas_v else []
        cmd = [nvcc, *nvcc_flags(extra), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        if ptxas_v:
            sys.stdout.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-ccbin", host_cxx(), *objs, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


def build_driver(force: bool = False) -> str:
    """Compiles the C++ driver program (vhlle_run) against the library."""
    build()
    hpp = os.path.join(ROOT, "include", "vhlle_b200.hpp")
    if (not force and os.path.exists(DRIVER)
            and os.path.getmtime(DRIVER) >= max(os.path.getmtime(p) for p in (DRIVER_SRC, hpp, LIB))):
        return DRIVER
    cmd = [host_cxx(), "-O2", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           DRIVER_SRC, "-L", HERE, "-lvhlle_b200", "-Wl,-rpath,$ORIGIN/..", "-o", DRIVER + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("driver build failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


if __name__ == "__main__":
    out = build(force=True, verbose=True, ptxas_v="--check" in sys.argv)
    print(out)
    print(build_driver(force=True))
