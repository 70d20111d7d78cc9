"""Gaussian incident beams (Beams::Gaussian::createEInc, DDA/Beam.cpp:196-263)
and the extinction of an arbitrary beam (Beam::extCross, DDA/Beam.cpp:58-67):
the front end against the oracle's numpy restatement, and the properties the
published beam formulas have (plane-wave limit, Gaussian profile in the focal
plane, the three kinds equal on the axis)."""
import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess
from oracle import oracle as O


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def pair(lam="1um"):
    g = dda_b200.Geometry.sphere("0.6um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], lam)
    og = O.Geometry.sphere("0.6um", "0.1um")
    op = O.Problem(og, [1.5 + 0.1j], lam)
    assert p.nv == op.nv and p.nvs == op.nvs
    return p, op


@pytest.mark.parametrize("kind", ["lminus", "davis3", "barton5"])
@pytest.mark.parametrize("pol", [1, 2])
def test_gaussian_einc_matches_oracle(kind, pol):
    p, op = pair()
    prop = (0.3, -0.2, 0.9)
    beam = dda_b200.Beam("gaussian:%s,0.7um,(0.1um,-0.2um,0.3um)" % kind)
    assert beam.kind == kind and beam.waist == pytest.approx(0.7e-6)
    got = p.einc(prop, pol, beam=beam)
    ref = op.einc_gaussian(prop, pol, kind, 0.7e-6, (0.1e-6, -0.2e-6, 0.3e-6))
    assert rel(got, ref) < 1e-13
    assert np.all(got.reshape(3, p.nvs)[:, p.nv:] == 0)


@pytest.mark.parametrize("kind", ["lminus", "davis3", "barton5"])
def test_wide_gaussian_is_the_plane_wave(kind):
    # waist >> target and wavelength: zeta, rho^2 and s = 1/(k w0) all vanish,
    # and every kind tends to the plane wave of the same polarisation
    p, _ = pair()
    prop = (0.0, 0.6, 0.8)
    for pol in (1, 2):
        plane = p.einc(prop, pol)
        g = p.einc(prop, pol, beam="gaussian:%s,1m" % kind)
        assert rel(g, plane) < 1e-6


def test_lminus_focal_plane_profile():
    # z = 0 layer of an odd box through the focus: psi0 = exp(-rho^2), real
    g = dda_b200.Geometry.box_shape("0.9um", "0.9um", "0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5], "1um")
    assert p.box[2] % 2 == 1
    w0 = 0.4e-6
    e = p.einc((0, 0, 1), 2, beam="gaussian:lminus,0.4um").reshape(3, p.nvs)[:, :p.nv]
    pos = g.positions.astype(np.float64)
    c = (pos - (np.array(p.box) - 1) / 2.0) * p.grid_unit
    mid = np.abs(c[:, 2]) < 1e-15
    assert mid.sum() == p.box[0] * p.box[1]
    inc, _ = dda_b200.beam_pol((0, 0, 1), 2)
    rho2 = (c[mid, 0] ** 2 + c[mid, 1] ** 2) / w0 ** 2
    for a in range(3):
        assert np.allclose(e[a, mid], inc[a] * np.exp(-rho2), rtol=1e-13, atol=1e-15)


def test_kinds_agree_on_the_axis():
    # on the beam axis (xi = eta = 0) the third- and fifth-order corrections
    # vanish: davis3 and barton5 equal lminus there
    g = dda_b200.Geometry.box_shape("0.1um", "0.1um", "1.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5], "1um")
    assert p.box[:2] == (1, 1)
    ref = p.einc((0, 0, 1), 1, beam="gaussian:lminus,0.5um")
    for kind in ("davis3", "barton5"):
        assert rel(p.einc((0, 0, 1), 1, beam="gaussian:%s,0.5um" % kind), ref) < 1e-15


def test_beam_strings():
    assert dda_b200.Beam("plane").plane
    b = dda_b200.Beam("gaussian:barton5,2um,(1um,0um,-0.5um)")
    assert b.kind == "barton5" and np.allclose(b.center, (1e-6, 0, -0.5e-6))
    for bad in ("plane:1", "gaussian:foo,1um", "gaussian:lminus,0um", "gaussian:davis3,1um,(1um,2um)", "cone"):
        with pytest.raises((ValueError, dda_b200.api.DDAError)):
            dda_b200.Beam(bad)


def test_general_extinction_equals_optical_theorem_for_a_plane_wave():
    # 4 pi k sum Im(P . conj(Einc)) is the optical theorem's Cext when Einc
    # is a plane wave: oracle FP64 solve of a small sphere
    p, op = pair("2um")
    prop = (0, 0, 1)
    for pol in (1, 2):
        op.set_cc(prop, pol, "ldr")
        op.build_dmatrix()
        einc = op.einc(prop, pol)
        rc, P, _, _ = op.solve(einc, "qmr", 1e-10)
        assert rc == 0
        cext_ot, _ = op.cross_sections(P, prop, pol)
        assert postprocess.ext_cross_general(p, P, einc) == pytest.approx(cext_ot, rel=1e-9)
