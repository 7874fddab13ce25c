"""Build the native library in-tree: ``python -m dyphur_b200.build``.

Produces ``dyphur_b200/lib/libdyphur_b200.so`` (CUDA kernels for sm_100a plus
the C++ host code behind the C ABI of ``include/dyphur_b200.h``) and the
pybind11 module ``dyphur_b200/lib/dyphur_py*.so`` (the reference's Python
surface over the C++ layer ``include/dyphur_b200.hpp``; it links the library
above through an ``$ORIGIN`` run path). nanobind, which the reference's
bindings use, is not installed; pybind11 is.

Numerics flags: ``--fmad=false -prec-div=true -prec-sqrt=true`` keep every
float operation correctly rounded and uncontracted, which is what makes the
kernels bit-identical to the reference's host arithmetic. The one exception is
the adjoint's reverse kernel (``csrc/reverse.cu``, its own translation unit),
built with approximate division and square root.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
BUILD_DIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NV_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
                   "-ftz=false", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"), "-ccbin", "g++"]
# The adjoint's reverse kernel (csrc/reverse.cu) alone: approximate division
# and square root (it follows recorded branches; its gradients are checked
# against FP64 within 1e-3 relative). Multiply-adds stay uncontracted, so every
# team layout of a scene computes the same gradients bit for bit.
REVERSE_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=false", "-prec-sqrt=false",
                        "-ftz=false", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"), "-ccbin", "g++"]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(ext):
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files if f.endswith(ext)]
    return sorted(out)


def build_native(verbose_ptxas: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    lib = os.path.join(LIB_DIR, "libdyphur_b200.so")
    deps = _sources(".cu") + _sources(".cuh") + _sources(".cpp") + _sources(".h") + \
        [os.path.join(ROOT, "include", "dyphur_b200.h")]
    if not _newer(lib, deps):
        return lib
    cu_obj = os.path.join(BUILD_DIR, "dyphur_b200.o")
    rev_obj = os.path.join(BUILD_DIR, "reverse.o")
    ptxas = ["-Xptxas", "-v"] if verbose_ptxas else []
    _run([NVCC] + NV_FLAGS + ptxas + ["-c", os.path.join(CSRC, "dyphur_b200.cu"), "-o", cu_obj])
    _run([NVCC] + REVERSE_FLAGS + ptxas + ["-c", os.path.join(CSRC, "reverse.cu"), "-o", rev_obj])
    host_objs = []
    for src in ("scenes.cpp",):
        obj = os.path.join(BUILD_DIR, src.replace(".cpp", ".o"))
        _run(["g++"] + CXX_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj])
        host_objs.append(obj)
    _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", "g++", cu_obj, rev_obj] + host_objs +
         ["-o", lib + ".tmp", "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    os.replace(lib + ".tmp", lib)
    return lib


def build_py_module() -> str:
    """The dyphur_py extension module (g++, pybind11) next to the library."""
    import pybind11
    lib = build_native()
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(LIB_DIR, "dyphur_py" + suffix)
    src = os.path.join(CSRC, "dyphur_py.cpp")
    deps = [src, lib, os.path.join(ROOT, "include", "dyphur_b200.hpp"), os.path.join(ROOT, "include", "dyphur_b200.h")]
    if not _newer(out, deps):
        return out
    cuda = os.path.dirname(os.path.dirname(NVCC))
    _run(["g++"] + CXX_FLAGS + ["-shared", "-fvisibility=hidden", "-I" + pybind11.get_include(),
                                "-I" + sysconfig.get_paths()["include"], "-I" + os.path.join(cuda, "include"), src,
                                "-o", out + ".tmp", "-L" + LIB_DIR, "-ldyphur_b200",
                                "-L" + os.path.join(cuda, "lib64"), "-lcudart_static", "-lrt", "-ldl", "-lpthread",
                                "-Wl,-rpath,$ORIGIN"])
    os.replace(out + ".tmp", out)
    return out


def build_all(verbose_ptxas: bool = False) -> None:
    build_native(verbose_ptxas)
    build_py_module()


if __name__ == "__main__":
    build_all(verbose_ptxas="-v" in sys.argv)
