"""Particle orientation (--orient, ZYZ Euler angles in degrees): the beam's
vectors in the particle frame (DipoleGeometry::orientationInverse,
DDA/DipoleGeometry.cpp:149-152, applied as in DDA/Beam.hpp:69-81,
DDA/PolarizabilityDescription.cpp:96-98 and DDA/FarFieldCalc.cpp:165-170)
against the oracle's rotation-matrix restatement, and the incident fields
and couple constants built from them."""
import numpy as np
import pytest

import dda_b200
from oracle import oracle as O

CASES = [((0, 0, 1), (90, 0, 0)), ((0.3, 0.4, 0.5), (30, 40, 50)), ((1, 0, 0), (-20, 135, 75)),
         ((0, -1, 0.2), (0, 90, 0))]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prop,orient", CASES)
def test_beam_frame_matches_rotation_matrices(prop, orient):
    center = (1e-6, -2e-6, 0.5e-6)
    got = dda_b200.beam_frame(prop, orient, center)
    want = O.beam_frame(prop, orient, center)
    for g, w in zip(got, want):
        assert np.allclose(g, w, rtol=0, atol=1e-15 * max(1.0, np.abs(w).max()))
    # an orthonormal right-handed frame: pol2 x pol1 = prop
    assert np.allclose(np.cross(got[2], got[1]), got[0], atol=1e-15)


def test_quarter_turn_about_z():
    pn, p1, p2, _ = dda_b200.beam_frame((0, 0, 1), (90, 0, 0))
    assert np.allclose(pn, (0, 0, 1), atol=1e-16)
    assert np.allclose(p1, (1, 0, 0), atol=1e-16) and np.allclose(p2, (0, -1, 0), atol=1e-16)


def pair():
    g = dda_b200.Geometry.box_shape("0.7um", "0.5um", "0.4um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    op = O.Problem(O.Geometry.box("0.7um", "0.5um", "0.4um", "0.1um"), [1.5 + 0.1j], "1um")
    assert op.nv == p.nv
    return p, op


def test_no_orientation_changes_nothing():
    p, _ = pair()
    for pol in (1, 2):
        e = p.einc((0.3, 0.4, 0.5), pol)
        assert np.array_equal(p.einc((0.3, 0.4, 0.5), pol, orient=(0, 0, 0)), e)
        c0 = dda_b200.CoupleConstants(p, (0.3, 0.4, 0.5), pol, "ldr")
        c1 = dda_b200.CoupleConstants(p, (0.3, 0.4, 0.5), pol, "ldr", orient=(0, 0, 0))
        assert np.array_equal(c0.cc, c1.cc)


@pytest.mark.parametrize("prop,orient", CASES)
def test_oriented_plane_wave_and_couple_constants(prop, orient):
    p, op = pair()
    pn, p1, p2, _ = O.beam_frame(prop, orient)
    for pol, pv in ((1, p1), (2, p2)):
        assert rel(p.einc(prop, pol, orient=orient), op.einc_frame(pn, pv)) < 1e-13
        cc = dda_b200.CoupleConstants(p, prop, pol, "ldr", orient=orient)
        op.set_cc_frame(pn, pv, "ldr")
        assert rel(cc.cc, op.cc()[0]) < 1e-13


@pytest.mark.parametrize("kind", ["lminus", "barton5"])
def test_oriented_gaussian_beam(kind):
    p, op = pair()
    prop, orient = (0.3, 0.4, 0.5), (30, 40, 50)
    beam = dda_b200.Beam("gaussian:%s,0.6um,(0.1um,0.2um,-0.1um)" % kind)
    for pol in (1, 2):
        got = p.einc(prop, pol, beam=beam, orient=orient)
        want = op.einc_gaussian(prop, pol, kind, 0.6e-6, (0.1e-6, 0.2e-6, -0.1e-6), orient=orient)
        assert rel(got, want) < 1e-13
