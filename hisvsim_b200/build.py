"""In-tree build of the native parts of hisvsim_b200.

Outputs (next to this file, git-ignored):
  * ``libhisv.so``  -- the C ABI of include/hisv.h: host planner + sm_100a
    kernels, built with nvcc ``-gencode arch=compute_100a,code=sm_100a``;
  * ``svsimulator_py_wrapper<EXT_SUFFIX>`` -- the pybind11 module with the
    reference's module name and API (py_wrapper.cpp:15-177), linked to
    libhisv.so with an ``$ORIGIN`` rpath.
Run ``python -m hisvsim_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libhisv.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
                  "-I" + CSRC, "--expt-relaxed-constexpr", "-ccbin", "g++"]
PYMOD_NAME = "svsimulator_py_wrapper"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def lib_sources():
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    return [s for s in srcs if not os.path.basename(s).startswith("py_")]


def build_lib(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    hdrs = _headers()
    for src in lib_sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(obj, [src] + hdrs):
            cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC] + NVFLAGS + ["-x", "cu", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"])
    return LIB


BOUNDS_BUILD = os.path.join(HERE, "_build_bounds")
BOUNDS_LIB = os.path.join(HERE, "libhisv_bounds.so")


def build_bounds_lib(verbose=False):
    """The same library with index checks at every kernel memory access
    (-DHS_BOUNDS): libhisv_bounds.so, loaded through HISV_LIB by the
    bounds tests."""
    os.makedirs(BOUNDS_BUILD, exist_ok=True)
    objs = []
    hdrs = _headers()
    for src in lib_sources():
        obj = os.path.join(BOUNDS_BUILD, os.path.basename(src) + ".o")
        if _stale(obj, [src] + hdrs):
            cmd = [NVCC] + NVFLAGS + ["-DHS_BOUNDS"]
            if src.endswith(".cpp"):
                cmd += ["-x", "cu"]
            cmd += ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if _stale(BOUNDS_LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", BOUNDS_LIB] + objs + ["-lcuda"])
    return BOUNDS_LIB


def pymod_path():
    return os.path.join(HERE, PYMOD_NAME + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pymod(verbose=False):
    import pybind11

    src = os.path.join(CSRC, "py_wrapper.cpp")
    out = pymod_path()
    if not os.path.exists(src):
        return None
    if _stale(out, [src, LIB] + _headers()):
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
               "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
               "-I" + INCLUDE, src, "-o", out, "-L" + HERE, "-lhisv",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return out


def build_all(verbose=False):
    build_lib(verbose)
    build_pymod(verbose)
    build_bounds_lib(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print("built", LIB)
