"""Builds libdda_b200.so in-tree with nvcc for sm_100a.

    python -m dda_b200.build          (or dda_b200.build.build())
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdda_b200.so")
SOURCES = ["dda_cuda.cu", "frontend.cpp", "serve.cpp"]
HEADERS = ["fft_engine.cuh", "fft_plan.cuh", "reduce.cuh", "krylov_ops.cuh", "krylov_kernels.cuh",
           "matvec_kernels.cuh", "matvec_planned.cuh", "matvec_dispatch.cuh", "dmatrix_kernels.cuh",
           "farfield_kernels.cuh", "matvec_slot.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx():
    # /usr/bin/g++ ships the full runtime; prefer it as nvcc's host compiler
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else None


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("dda_cuda.h", "dda_frontend.h", "dda_serve.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    cmd = [_nvcc()] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-shared",
                              "-Xcompiler", "-fPIC", "-o", LIB + ".tmp"]
    cxx = _host_cxx()
    if cxx:
        cmd += ["-ccbin", cxx]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
