"""Builds libhighreg_b200.so in-tree (sm_100a only).

CUDA sources are compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``; the host
planner (host/*.cpp) with g++ and OpenMP; the library links the CUDA runtime
(static) and OpenMP. Objects go to ``_build/`` next to this file; the shared library sits
next to this file so that it travels with the working tree.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhighreg_b200.so")
REFAPI = os.path.join(HERE, "libhighreg_refapi.so")
FFTWAPI = os.path.join(HERE, "libhighreg_fftw.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                  "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-I", os.path.join(ROOT, "include")]


def _sources():
    cu = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    cpp = sorted(f for f in glob.glob(os.path.join(HERE, "host", "*.cpp"))
                 if not f.endswith(("hr_ref_api.cpp", "hr_fftw_shim.cpp")))
    hdr = sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))
                 + glob.glob(os.path.join(HERE, "host", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
                 + glob.glob(os.path.join(ROOT, "include", "fftw_shim", "*.h")))
    return cu, cpp, hdr


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp, hdr = _sources()
    hdr_t = max([os.path.getmtime(h) for h in hdr] + [os.path.getmtime(__file__)])
    objs = []
    logs = []
    for src in cu + cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_t and not ptxas_info):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC] + NVFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", obj]
        logs.append(_run(cmd, verbose))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        logs.append(_run(cmd, verbose))
    # the reference-signature layer, a separate library over the C ABI
    src = os.path.join(HERE, "host", "hr_ref_api.cpp")
    if force or not os.path.exists(REFAPI) or os.path.getmtime(REFAPI) < max(os.path.getmtime(src), hdr_t,
                                                                              os.path.getmtime(LIB)):
        logs.append(_run(["g++"] + CXXFLAGS + ["-shared", src, "-o", REFAPI, "-L", HERE, "-lhighreg_b200",
                          "-Wl,-rpath,$ORIGIN"], verbose))
    # the FFTW-API layer (fftw_plan_r2r_3d / fftw_execute ... over hr_dst1_*)
    src = os.path.join(HERE, "host", "hr_fftw_shim.cpp")
    if force or not os.path.exists(FFTWAPI) or os.path.getmtime(FFTWAPI) < max(os.path.getmtime(src), hdr_t,
                                                                                os.path.getmtime(LIB)):
        logs.append(_run(["g++"] + CXXFLAGS + ["-shared", src, "-o", FFTWAPI, "-L", HERE, "-lhighreg_b200",
                          "-Wl,-rpath,$ORIGIN"], verbose))
    if ptxas_info:
        print("\n".join(l for l in logs if l))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
