"""CPU tests of libdda_b200.so's host side: exported ABI, bit-exact
voxelisation and the couple constants / incident field against the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import dda_b200
from dda_b200 import api, postprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "box_10_8_6.geom")


def _declared_symbols():
    names = set()
    for h in ("dda_cuda.h", "dda_frontend.h", "dda_serve.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(dda_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(api.lib_path)
    syms = _declared_symbols()
    assert len(syms) >= 25
    for s in sorted(syms):
        assert hasattr(L, s), s


@pytest.mark.parametrize("x", [1, 2, 13, 22, 26, 38, 80, 100, 106, 110, 192, 200, 254, 512])
@pytest.mark.parametrize("nonpot", [True, False])
def test_fft_fit_matches_oracle(oracle, x, nonpot):
    assert dda_b200.fft_fit(x, 0, nonpot) == oracle.fft_fit(x, 0, nonpot)


@pytest.mark.parametrize("shape", [
    ("sphere", ("10um", "0.5um")), ("sphere", ("1.3um", "0.1um")), ("sphere", ("12.8um", "0.8um")),
    ("box", ("10um", "5um", "5um", "0.1um")), ("box", ("1um", "0.7um", "0.3um", "0.1um")),
    ("cylinder", ("2um", "0.5um", "0.1um")), ("cylinder", ("1.05um", "0.33um", "0.07um"))])
def test_voxelisation_bit_exact(oracle, shape):
    kind, args = shape
    if kind == "sphere":
        g, o = dda_b200.Geometry.sphere(*args), oracle.Geometry.sphere(*args)
    elif kind == "box":
        g, o = dda_b200.Geometry.box_shape(*args), oracle.Geometry.box(*args)
    else:
        g, o = dda_b200.Geometry.cylinder(*args), oracle.Geometry.cylinder(*args)
    assert g.nv == o.nv and g.box == o.box_size
    assert np.array_equal(g.positions, o.positions())
    assert np.array_equal(g.materials, o.materials())


def test_load_fixture(oracle):
    g = dda_b200.Geometry.load(FIXTURE, "0.1um")
    o = oracle.Geometry.load_text(FIXTURE, "0.1um")
    assert g.nv == 480 and g.box == (10, 8, 6)
    assert np.array_equal(g.positions, o.positions())


def test_load_rejects_bad(tmp_path):
    f = tmp_path / "bad.geom"
    f.write_text("0 0 1\n0 0 0\n")
    with pytest.raises(dda_b200.DDAError):
        dda_b200.Geometry.load(str(f), "0.1um")
    f.write_text("0 0 0 0\n")  # material 0 is invalid (1-based)
    with pytest.raises(dda_b200.DDAError):
        dda_b200.Geometry.load(str(f), "0.1um")


def test_params_cfg2_grid():
    g = dda_b200.Geometry.box_shape("10um", "5um", "5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    assert p.nv == 250000 and p.grid == (200, 100, 100)
    p2 = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um", support_nonpot=False)
    assert p2.grid == (256, 128, 128)


@pytest.mark.parametrize("kind", ["cm", "ldr", "ldr-avgpol"])
@pytest.mark.parametrize("prop,pol", [((0, 0, 1), 1), ((0, 0, 1), 2), ((0, 1, 0), 1), ((0.3, 0.4, 0.866), 2)])
def test_couple_constants_match_oracle(oracle, kind, prop, pol):
    mats = [1.5 + 0.1j, (1.33 + 0.01j, 1.4 + 0.02j, 1.6 + 0.0j)]
    pos = np.array([[0, 0, 0], [1, 0, 0]], dtype=np.uint32)
    mat = np.array([0, 1], dtype=np.uint8)
    g = dda_b200.Geometry.from_arrays(pos, mat, "0.1um")
    p = dda_b200.DDAParams(g, mats, "0.6um")
    cc = dda_b200.CoupleConstants(p, prop, pol, kind)
    og = oracle.Geometry.from_arrays(pos, mat, "0.1um")
    op = oracle.Problem(og, mats, "0.6um")
    op.set_cc(prop, pol, kind)
    occ, ocs, oci = op.cc()
    assert np.allclose(cc.cc, occ, rtol=1e-13, atol=0)
    assert np.allclose(cc.cc_sqrt, ocs, rtol=1e-13, atol=0)
    assert np.allclose(cc.chi_inv, oci, rtol=1e-13, atol=0)


def test_einc_matches_oracle(oracle):
    g = dda_b200.Geometry.sphere("1um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "0.6um")
    og = oracle.Geometry.sphere("1um", "0.1um")
    op = oracle.Problem(og, [1.5 + 0.1j], "0.6um")
    for prop, pol in [((0, 0, 1), 1), ((0.3, -0.4, 0.866), 2)]:
        e = p.einc(prop, pol)
        oe = op.einc(prop, pol)
        assert np.abs(e - oe).max() < 1e-12


def test_beam_pol_convention():
    # DDA/Beam.cpp:41-50: prop = z gives pol1 = y, pol2 = x
    p1, _ = dda_b200.beam_pol((0, 0, 1), 1)
    p2, _ = dda_b200.beam_pol((0, 0, 1), 2)
    assert np.allclose(p1, (0, 1, 0)) and np.allclose(p2, (1, 0, 0))
    q1, pn = dda_b200.beam_pol((0, 1, 0), 1)
    assert abs(np.dot(q1, pn)) < 1e-15


def test_grid_angles_follow_angle_list():
    t, p = postprocess.grid_angles("0..180/3", "0..360/4")
    assert len(t) == 12
    assert np.allclose(np.degrees(t[::4]), [0, 90, 180])
    assert np.allclose(np.degrees(p[:4]), [0, 120, 240, 360])
    t1, p1 = postprocess.grid_angles("30", "45")
    assert np.allclose(np.degrees([t1[0], p1[0]]), [30, 45])


def test_geometry_without_dipoles_is_rejected():
    # an empty dipole list or a shape too small to hold a dipole centre is an
    # error of the front end, not an empty problem
    import dda_b200
    for make in (lambda: dda_b200.Geometry.from_arrays(np.zeros((0, 3), np.uint32), np.zeros(0, np.uint8), "0.1um"),
                 lambda: dda_b200.Geometry.sphere("0.01um", "0.1um")):
        with pytest.raises(dda_b200.api.DDAError, match="no dipoles"):
            make()
