"""In-tree build of the B200 library and its Python module.

Produces, next to the package sources (so they travel with the tree):
  e8qlib/libe8qcuda.so            CUDA kernels + the C ABI (include/e8qc.h)
  e8qlib/_e8qlib<ext>             pybind11 module over the C ABI

Every .cu file is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a). build_kernels.cu, me8q_kernels.cu and
me8q_fast.cu additionally use --fmad=false (bit-exact encoder, ME8Q fits and
the pruned search's bound arithmetic). Host C++ uses -ffp-contract=off. Objects
are rebuilt when a source or header is newer than its object.

Usage: python e8q-artifact_b200/build.py [-j N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "e8qlib")
OBJ = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(PKG, "libe8qcuda.so")
EXT = os.path.join(PKG, "_e8qlib" + sysconfig.get_config_var("EXT_SUFFIX"))

CU_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC,
            "--expt-relaxed-constexpr", "-diag-suppress", "940"]
PER_FILE = {"build_kernels.cu": ["--fmad=false"], "me8q_kernels.cu": ["--fmad=false"], "me8q_fast.cu": ["--fmad=false"]}
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             "-I" + INC, "-I" + CSRC, "-I" + os.path.join(CUDA, "include")]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "*.h"))


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def _compile(src, force):
    name = os.path.basename(src)
    out = os.path.join(OBJ, name + ".o")
    if not force and not _stale(out, [src] + _headers()):
        return out, False
    if name.endswith(".cu"):
        cmd = [NVCC] + ARCH + CU_FLAGS + PER_FILE.get(name, []) + ["-c", src, "-o", out]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", out]
    _run(cmd)
    return out, True


def build(jobs: int = 8, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(PKG, exist_ok=True)
    lib_srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                      [p for p in glob.glob(os.path.join(CSRC, "*.cpp"))
                       if os.path.basename(p) != "bindings.cpp"])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        res = list(ex.map(lambda s: _compile(s, force), lib_srcs))
    objs = [o for o, _ in res]
    if force or any(c for _, c in res) or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-Xlinker", "-soname=libe8qcuda.so"])
        if verbose:
            print("linked", LIB)
    bsrc = os.path.join(CSRC, "bindings.cpp")
    if force or _stale(EXT, [bsrc, LIB] + _headers()):
        import pybind11

        py_inc = sysconfig.get_paths()["include"]
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden",
              "-I" + pybind11.get_include(), "-I" + py_inc, "-I" + INC, bsrc, "-o", EXT,
              "-L" + PKG, "-le8qcuda", "-Wl,-rpath,$ORIGIN"])
        if verbose:
            print("linked", EXT)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.j, a.force, verbose=True)


if __name__ == "__main__":
    sys.exit(main())
