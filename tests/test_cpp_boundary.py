"""The C++ half of the drop-in boundary, compiled and linked as a caller
would: include/dda_cuda.hpp (dda::CudaMatVec<T> for MatVec<T>,
DDA/MatVec.hpp:33-55; dda::CudaSolver<T> for IterativeSolverBase<T>::getPolVec,
DDA/IterativeSolverBase.hpp:31-75) through tests/cpp/boundary_demo.cpp, and
the MatVecB200 binding of INTEGRATION.md against stand-ins of the
reference's interfaces (tests/cpp/ref_stub).  On the GPU the demo's matvecs
and solve are compared with the oracle."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dda_b200")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _lib():
    import dda_b200
    dda_b200.lib()  # builds libdda_b200.so when it is missing
    return os.path.join(LIBDIR, "libdda_b200.so")


def build_demo(tmp_path):
    _lib()
    exe = str(tmp_path / "boundary_demo")
    cmd = [CXX, "-std=c++11", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "boundary_demo.cpp"), "-L", LIBDIR, "-ldda_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_header_compiles_and_links(tmp_path):
    exe = build_demo(tmp_path)
    assert os.path.exists(exe)
    if shutil.which("nvidia-smi") is None:
        # no CUDA device here: dda_create fails and CudaMatVec throws dda::Error
        r = subprocess.run([exe, str(tmp_path / "out.bin")], capture_output=True, text=True, timeout=120)
        assert r.returncode == 2, (r.returncode, r.stdout, r.stderr)
        assert "dda::Error" in r.stderr


def test_integration_binding_compiles(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    sketch = next(b for b in blocks if "class MatVecB200" in b)
    src = tmp_path / "matvec_b200.cpp"
    src.write_text(sketch + "\ntemplate class DDA::MatVecB200<double>;\ntemplate class DDA::MatVecB200<float>;\n")
    cmd = [CXX, "-std=c++11", "-Wall", "-Werror", "-Wno-unused-parameter", "-fsyntax-only",
           "-I", os.path.join(ROOT, "tests", "cpp", "ref_stub"), "-I", os.path.join(ROOT, "include"), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_demo_matches_oracle(tmp_path):
    from oracle import oracle as O
    exe = build_demo(tmp_path)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(str(out), dtype=np.float64)
    nvs = int(raw[0])
    n = 3 * nvs
    c = raw[1:1 + 6 * n].view(np.complex128)
    y64, y32, pol = c[:n], c[n:2 * n], c[2 * n:3 * n]
    iters = int(raw[1 + 6 * n])
    pol32 = raw[2 + 6 * n:2 + 8 * n].view(np.complex128)
    og = O.Geometry.sphere("0.5um", "0.1um")
    op = O.Problem(og, [1.5 + 0.1j], "1um")
    assert op.nvs == nvs
    op.build_dmatrix()
    op.set_cc((0, 0, 1), 1, "ldr")
    j = np.arange(n, dtype=np.float64)
    x = np.sin(j) + 1j * np.cos(2 * j)
    for comp in range(3):
        x[comp * nvs + op.nv:(comp + 1) * nvs] = 0
    want = op.matvec(x)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel(y64, want) < 1e-12
    assert rel(y32, want) < 2e-6
    rc, opol, st, _ = op.solve(op.einc((0, 0, 1), 1), "qmr", 1e-8)
    assert rc == 0
    assert abs(iters - st.iterations) <= 1
    assert rel(pol, opol) < 1e-6
    # CudaSolver<float>: complex float vectors through dda_solve_f32, to 1e-5
    assert rel(pol32, opol) < 1e-3
