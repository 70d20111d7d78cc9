"""CPU tests of the oracle (the checker the CUDA path is compared against).

The reference cannot be built here, so these tests pin the restatement with
independent evidence: numpy's FFT, a brute-force direct-sum matvec, the
reference's own geometry fixture (DDA/box_10_8_6.geom) and the dipole counts
of the reference's README workloads.
"""
import os

import numpy as np
import pytest

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "box_10_8_6.geom")


@pytest.mark.parametrize("n", [2, 6, 8, 10, 12, 14, 30, 80, 96, 100, 126, 128, 200, 210, 250, 343, 512])
def test_fft_matches_numpy(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
    scale = np.abs(np.fft.fft(x)).max()
    assert np.abs(oracle.fft(x) - np.fft.fft(x)).max() < 1e-13 * scale
    assert np.abs(oracle.fft(x, inverse=True) - np.fft.ifft(x) * n).max() < 1e-13 * scale


@pytest.mark.parametrize("x,nonpot,expect", [
    (80, True, 80), (80, False, 128), (200, True, 200), (100, True, 100), (200, False, 256),
    (192, True, 192), (128, True, 128), (512, True, 512), (22, True, 24), (26, True, 28),
    (34, True, 36), (38, True, 40), (46, True, 48), (62, True, 64), (1, True, 2), (0, True, 0),
    (13, False, 16), (106, True, 108), (110, True, 112)])
def test_fft_fit(oracle, x, nonpot, expect):
    # DDA/DDAParams.cpp:45-90: even 2,3,5,7-smooth (CPU) or power of two (GPU)
    assert oracle.fft_fit(x, 0, nonpot) == expect


def test_fft_fit_override(oracle):
    assert oracle.fft_fit(80, 96, True) == 96


def test_sphere_cfg1_counts(oracle):
    # README workload: sphere radius 10 um, grid unit 0.5 um
    g = oracle.Geometry.sphere("10um", "0.5um")
    assert g.nv == 33552
    assert g.box_size == (40, 40, 40)
    pos = g.positions()
    assert np.all(np.diff(pos[:, 2].astype(np.int64)) >= 0)  # sorted by z
    key = pos[:, 0] + 40 * (pos[:, 1] + 40 * pos[:, 2].astype(np.int64))
    assert np.all(np.diff(key) > 0)  # z, y, x loop order


def test_box_cfg2_counts_long_double(oracle):
    # 10 um / 0.1 um evaluates below 100 in long double; x < 99.999.. keeps 100
    g = oracle.Geometry.box("10um", "5um", "5um", "0.1um")
    assert g.nv == 250000
    assert g.box_size == (100, 50, 50)


def test_cylinder(oracle):
    g = oracle.Geometry.cylinder("2um", "0.5um", "0.1um")
    assert g.box_size[0] == 20
    pos = g.positions()
    r = 5.0
    yd = pos[:, 1] - r + 0.5
    zd = pos[:, 2] - r + 0.5
    assert np.all(yd * yd + zd * zd <= r * r)


def test_fixture_box_10_8_6(oracle):
    g = oracle.Geometry.load_text(FIXTURE, "0.1um")
    assert g.nv == 480
    assert g.box_size == (10, 8, 6)
    assert g.mat_count == 1
    # DDA_REFERENCE_DIR: a checkout of the reference, to compare with its own
    # fixture file (skipped when unset)
    ref = os.path.join(os.environ.get("DDA_REFERENCE_DIR", ""), "DDA", "box_10_8_6.geom")
    if os.environ.get("DDA_REFERENCE_DIR") and os.path.exists(ref):  # same dipole list as the reference's fixture
        r = oracle.Geometry.load_text(ref, "0.1um")
        assert np.array_equal(r.positions(), g.positions())
        assert np.array_equal(r.materials(), g.materials())


def test_load_rejects_unsorted(oracle, tmp_path):
    f = tmp_path / "bad.geom"
    f.write_text("0 0 1\n0 0 0\n")
    with pytest.raises(ValueError):
        oracle.Geometry.load_text(str(f), "0.1um")


def _small_problem(oracle, lam="1um"):
    pos = [(x, y, z) for z in range(4) for y in range(5) for x in range(6) if (x + y + z) % 5]
    pos = np.array(pos)
    mat = (pos[:, 0] % 2).astype(np.uint8)
    g = oracle.Geometry.from_arrays(pos, mat, "0.1um")
    p = oracle.Problem(g, [1.5 + 0.1j, 1.3 + 0.05j], lam)
    p.set_cc((0.3, 0.4, 0.866), 1, "ldr")
    p.build_dmatrix()
    return p


def _rand_vec(p, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    return x


def test_matvec_equals_direct_sum(oracle):
    p = _small_problem(oracle)
    x = _rand_vec(p, 3)
    y = p.matvec(x)
    yd = p.direct_matvec(x)
    assert np.linalg.norm(y - yd) / np.linalg.norm(yd) < 1e-13


def test_matvec_conj_and_padding(oracle):
    p = _small_problem(oracle)
    x = _rand_vec(p, 4)
    yc = p.matvec(x, conj=True)
    assert np.allclose(yc, np.conj(p.matvec(np.conj(x))), rtol=0, atol=1e-14 * np.abs(yc).max())
    # A is complex symmetric: u.(A v) == v.(A u)
    u = _rand_vec(p, 5)
    assert abs(u @ p.matvec(x) - x @ p.matvec(u)) < 1e-12 * abs(u @ p.matvec(x))


def test_dmatrix_symmetries(oracle):
    # The Green's tensor is even (diagonal) or odd (off-diagonal) per axis, so
    # D-hat has the same parities; the compressed octant layout relies on it.
    p = _small_problem(oracle)
    D = p.dmatrix()  # [kx][kz][ky][6]
    gx, gz, gy, _ = D.shape
    mx = (-np.arange(gx)) % gx
    my = (-np.arange(gy)) % gy
    mz = (-np.arange(gz)) % gz
    sx = np.array([1, -1, -1, 1, 1, 1])
    sy = np.array([1, -1, 1, 1, -1, 1])
    sz = np.array([1, 1, -1, 1, -1, 1])
    scale = np.abs(D).max()
    assert np.abs(D[mx] * sx - D).max() < 1e-12 * scale
    assert np.abs(D[:, :, my] * sy - D).max() < 1e-12 * scale
    assert np.abs(D[:, mz] * sz - D).max() < 1e-12 * scale


@pytest.mark.parametrize("solver", ["qmr", "bicgstab", "bicg", "cgnr"])
def test_solvers_agree(oracle, solver):
    p = _small_problem(oracle)
    e = p.einc((0.3, 0.4, 0.866), 1)
    rc0, pol0, st0, _ = p.solve(e, "qmr", 1e-10)
    rc, pol, st, hist = p.solve(e, solver, 1e-8)
    assert rc0 == 0 and rc == 0
    assert st.relResidual < 1e-8
    assert len(hist) == st.iterations
    assert np.linalg.norm(pol - pol0) / np.linalg.norm(pol0) < 1e-6


def test_couple_constants_cm_ldr(oracle):
    p = _small_problem(oracle)
    p.set_cc((0, 0, 1), 1, "cm")
    cc, ccs, chi = p.cc()
    m2 = (1.5 + 0.1j) ** 2
    vol = p.grid_unit_vol
    cm = 3 * vol / (4 * np.pi) * (m2 - 1) / (m2 + 2)
    assert abs(cc[0] - cm) < 1e-14 * abs(cm)
    assert np.allclose(ccs ** 2, cc, rtol=1e-14)
    p.set_cc((0, 0, 1), 1, "ldr")
    ldr, _, _ = p.cc()
    # LDR with prop=z, pol=y: S = 0 (DDA/PolarizabilityDescription.cpp:96-104)
    kd = p.kd
    t1 = 1j * 2 / 3 * kd ** 3 + (1.8915316 + (-0.1648469) * m2) * kd ** 2
    want = cm / (1 - cm / vol * t1)
    assert abs(ldr[0] - want) < 1e-13 * abs(want)


def test_mie_pins_oracle_cross_sections(oracle):
    # Physics pin: the oracle's DDA (LDR, FFT matvec, QMR-CS, Cext/Cabs of
    # DDA/Beam.cpp:126-133 and DDA/AbsCross.cpp:28-48) converges to the
    # Bohren-Huffman Mie series (EMSim/Mie.cpp) as the grid is refined.
    a = 1e-6
    x = 2 * np.pi * a / 4e-6
    qe, qs, qa = oracle.mie(x, 1.5 + 0.1j)
    errs = []
    for d in ("0.1um", "0.05um"):
        g = oracle.Geometry.sphere("1um", d)
        p = oracle.Problem(g, [1.5 + 0.1j], "4um")
        p.build_dmatrix()
        p.set_cc((0, 0, 1), 1, "ldr")
        e = p.einc((0, 0, 1), 1)
        rc, pol, st, _ = p.solve(e, "qmr", 1e-8)
        assert rc == 0
        cext, cabs = p.cross_sections(pol, (0, 0, 1), 1)
        errs.append((abs(cext / (np.pi * a * a) - qe) / qe, abs(cabs / (np.pi * a * a) - qa) / qa))
    assert errs[1][0] < 1e-3 and errs[1][1] < 3e-3
    assert errs[1][0] < errs[0][0]


def test_mie_known_values(oracle):
    # small-particle limit: Qext ~ Qabs ~ 4x Im((m^2-1)/(m^2+2)) for x -> 0
    x = 1e-3
    m = 1.5 + 0.1j
    qe, qs, qa = oracle.mie(x, m)
    ray = 4 * x * ((m * m - 1) / (m * m + 2)).imag
    assert abs(qa - ray) < 1e-3 * ray
    qe2, qs2, qa2 = oracle.mie(5.0, 1.33)
    assert abs(qa2) < 1e-9 and 2.0 < qe2 < 4.5


@pytest.mark.parametrize("x,m", [(1e-3, 1.5 + 0.1j), (1.57, 1.5 + 0.1j), (5.0, 1.33), (60.0, 1.6 + 0.01j),
                                 (15.0, 2.0 + 0.5j)])
def test_product_mie_matches_oracle(oracle, x, m):
    # the product's Mie series (used by the 512^3 sphere benchmark) against
    # the oracle's long-double restatement
    from dda_b200 import postprocess
    got = postprocess.mie(x, m)
    want = oracle.mie(x, m)
    for g, w in zip(got, want):  # Qabs of a lossless sphere is a difference of equal terms
        assert abs(g - w) <= 1e-9 * max(abs(w), want[0])


def test_float_path_tracks_double(oracle):
    # the reference's --ftype float CPU path (D built in float by
    # DMatrixCpu<float>, matvec, vectors and scalars in float) against its
    # double path on a small target.  Building D in float costs about 1e-4
    # relative accuracy (1/r^3 terms over a wide dynamic range through float
    # FFTs), so the solutions agree to that level, not to float rounding.
    g = oracle.Geometry.sphere("0.6um", "0.1um")
    p = oracle.Problem(g, [1.5 + 0.1j], "1um")
    p.build_dmatrix()
    p.set_cc((0, 0, 1), 1, "ldr")
    e = p.einc((0, 0, 1), 1)
    rc64, p64, st64, _ = p.solve(e, "bicgstab", 1e-5)
    rc32, p32, st32, _ = p.solve(e, "bicgstab", 1e-5, precision="fp32")
    assert rc64 == 0 and rc32 == 0
    assert abs(st64.iterations - st32.iterations) <= 3
    assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) < 1e-3
