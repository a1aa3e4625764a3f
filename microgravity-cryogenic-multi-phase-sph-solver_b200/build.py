"""Builds the native parts of the package in place.

  libcryosph_b200.so   CUDA kernels for sm_100a + the C ABI (include/cryosph_b200.h)
  CryoSPH*.so          pybind11 module with the reference's Python API, on top of
                       the C++ host layer (host/) that calls the C ABI

Run `python build.py` (or import and call build()).  Objects go to _build/
next to this file; a target is rebuilt when any of its inputs is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX_HOST", "/usr/bin/g++")

CU_SOURCES = ["cryo_grid.cu", "cryo_physics.cu", "cryo_phase.cu", "cryo_control.cu", "cryo_setup.cu", "cryo_adjoint.cu",
              "cryo_slab.cu", "cryo_abi.cu", "cryo_io.cu", "cryo_ensemble.cu", "cryo_adj_abi.cu", "cryo_slab_abi.cu"]
# -fmad=false: no FMA contraction, so single-precision results follow the
# reference's IEEE operation sequence (see csrc/cryo_common.cuh).
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "--extended-lambda", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2,-fopenmp", "-I" + INCLUDE,
]
# cryo_physics.cu again for the fast field arithmetic: FMA contraction and
# approximate division / square root (denormals kept).
FAST_FIELD_FLAGS = [f for f in NVCC_FLAGS if f != "-fmad=false"] + [
    "-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-DCRYO_FIELD_NS=fast"]
LIB = os.path.join(HERE, "libcryosph_b200.so")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def _headers(d):
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h", ".hpp"))]


def build_lib(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers(CSRC) + [os.path.join(INCLUDE, "cryosph_b200.h")]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    # the neighbour passes a second time, contracted (namespace cryo::fast)
    s = os.path.join(CSRC, "cryo_physics.cu")
    o = os.path.join(BUILD, "cryo_physics_fast.cu.o")
    objs.append(o)
    if _newer(o, [s] + hdrs):
        jobs.append([NVCC] + FAST_FIELD_FLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for r in ex.map(_run, jobs):
            if verbose and r.stderr:
                print(r.stderr)
    if _newer(LIB, objs):
        _run([NVCC, "-shared", "-o", LIB] + objs + ["-lcudart", "-Xcompiler", "-fopenmp"])
    return LIB


def build_module(verbose=False):
    """pybind11 module `CryoSPH` (host C++ layer over the C ABI)."""
    import pybind11

    if not os.path.isdir(HOST):
        return None
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = os.path.join(HERE, "CryoSPH" + ext)
    srcs = [os.path.join(HOST, f) for f in sorted(os.listdir(HOST)) if f.endswith(".cpp")]
    deps = srcs + _headers(HOST) + [os.path.join(INCLUDE, "cryosph_b200.h"), LIB]
    if _newer(target, deps):
        cmd = [CXX, "-O2", "-std=c++20", "-shared", "-fPIC", "-fopenmp", "-ffp-contract=off",
               "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"], "-I" + INCLUDE, "-I" + HOST,
               "-o", target] + srcs + ["-L" + HERE, "-lcryosph_b200", "-Wl,-rpath,$ORIGIN"]
        _run(cmd)
    return target


def build(verbose=False):
    lib = build_lib(verbose)
    mod = build_module(verbose)
    return lib, mod


if __name__ == "__main__":
    out = build(verbose="-v" in sys.argv)
    print("built:", *[o for o in out if o])
