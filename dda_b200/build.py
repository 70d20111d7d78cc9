"""Builds libdda_b200.so in-tree with nvcc for sm_100a.

    python -m dda_b200.build          (or dda_b200.build.build())
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdda_b200.so")
SOURCES = ["dda_cuda.cu", "frontend.cpp", "serve.cpp"]
# mv_inst.cu is compiled once per (part, double): the kernel-table parts
MV_PARTS = [(part, dbl) for dbl in (0, 1) for part in (0, 1, 2, 3, 4, 5)]
HEADERS = ["fft_engine.cuh", "fft_plan.cuh", "reduce.cuh", "krylov_ops.cuh", "krylov_kernels.cuh",
           "matvec_kernels.cuh", "matvec_planned.cuh", "matvec_dispatch.cuh", "dmatrix_kernels.cuh",
           "farfield_kernels.cuh", "matvec_slot.cuh", "kernel_shapes.cuh", "matvec_pair.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx():
    # /usr/bin/g++ ships the full runtime; prefer it as nvcc's host compiler
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else None


def _deps():
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + ["mv_inst.cu"]]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("dda_cuda.h", "dda_frontend.h", "dda_serve.h")]
    return [d for d in deps if os.path.exists(d)]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _units():
    """(source, object, extra flags) of every translation unit."""
    units = []
    for f in SOURCES:
        units.append((os.path.join(CSRC, f), os.path.join(OBJ, f + ".o"), []))
    for part, dbl in MV_PARTS:
        units.append((os.path.join(CSRC, "mv_inst.cu"), os.path.join(OBJ, "mv_inst_%d_%d.o" % (part, dbl)),
                      ["-DDDA_MV_PART=%d" % part, "-DDDA_MV_DOUBLE=%d" % dbl]))
    return units


def build(force=False, verbose=False, jobs=None):
    """Compiles the translation units in parallel (every unit whose sources
    or headers changed) and links libdda_b200.so."""
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    base = [_nvcc()] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
    cxx = _host_cxx()
    if cxx:
        base += ["-ccbin", cxx]
    cmds = []
    headers = [d for d in deps if not d.endswith((".cu", ".cpp"))]
    for src, obj, extra in _units():
        if force or _stale(obj, headers + [src]):
            cmds.append(base + extra + ["-c", src, "-o", obj + ".tmp"])
    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        os.replace(cmd[-1], cmd[-1][:-4])
        return r.stderr
    n = jobs or max(1, min(len(cmds), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(n) as ex:
        for err in ex.map(run, cmds):
            if verbose and err.strip():
                print(err, file=sys.stderr)
    link = [_nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + [o for _, o, _ in _units()]
    if cxx:
        link[1:1] = ["-ccbin", cxx]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
