"""Build the in-tree native libraries of fastimaging_b200.

    libstpgpu.so      CUDA kernels + host orchestration + the C ABI
                      (include/stpgpu.h), sm_100a only, static cudart,
                      cuFFT from the CUDA toolkit.
    stp_python*.so    pybind11 module mirroring the reference's stp_python
                      binding, calling the C ABI.
    libstpgpu_peaks.so  FP32/FP64 FMA-throughput probe (the roofline's
                      compute roof, used by bench.py).

Run ``python -m fastimaging_b200.build`` (or ``__graft_entry__.build()``).
Cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(PKG, "libstpgpu.so")


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources():
    out = [os.path.join(ROOT, "include", "stpgpu.h")]
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".h", ".hpp")):
            out.append(os.path.join(CSRC, f))
    return out


def build_lib(verbose=False, force=False):
    srcs = _sources()
    if not force and not _newer(LIB, srcs):
        return LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
           "-cudart", "static", "-o", LIB, os.path.join(CSRC, "api.cu"), "-L" + os.path.join(CUDA_HOME, "lib64"),
           "-lcufft", "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


def build_python(verbose=False, force=False):
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(PKG, "stp_python" + ext)
    srcs = [os.path.join(CSRC, "stp_python.cpp"), os.path.join(ROOT, "include", "stpgpu.h"), LIB]
    if not os.path.exists(srcs[0]):
        return None
    if not force and not _newer(out, srcs):
        return out
    cxx = "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I" + pybind11.get_include(),
           "-I" + sysconfig.get_paths()["include"], "-I" + os.path.join(ROOT, "include"),
           os.path.join(CSRC, "stp_python.cpp"), "-o", out, "-L" + PKG, "-lstpgpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


PEAKS = os.path.join(PKG, "libstpgpu_peaks.so")


def build_peaks(verbose=False, force=False):
    """FMA-throughput probe for the roofline's compute roof (bench.py)."""
    src = os.path.join(CSRC, "peaks.cu")
    if not force and not _newer(PEAKS, [src]):
        return PEAKS
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
           "-cudart", "static", "-o", PEAKS, src]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return PEAKS


def build(verbose=False, force=False):
    build_lib(verbose, force)
    build_python(verbose, force)
    build_peaks(verbose, force)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
