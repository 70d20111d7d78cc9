"""Far field, Jones matrices and cross sections on the GPU against the oracle
(FarFieldCalc::calcEField, JonesCalculus::getJonesMatrix, PlaneWave::extCross,
AbsCross::absCross) and against the Mie series."""
import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess as PP
from pairs import Pair, aniso_arrays, rel, scrambled_arrays

pytestmark = pytest.mark.gpu

PROP = (0.0, 0.6, 0.8)


def _dirs(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@pytest.mark.parametrize("case", ["aniso", "scrambled"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_far_field_matches_oracle(case, precision, tol):
    arrs = aniso_arrays() if case == "aniso" else scrambled_arrays()
    pr = Pair("arrays", arrs, [1.5 + 0.1j, 1.3 + 0.05j], "1um", precision=precision, max_rhs=2)
    x = np.stack([pr.rand_vec(1), pr.rand_vec(2)])
    dirs = _dirs(11, 3)
    e = pr.mv.far_field(dirs, nrhs=2, pol=x)
    for b in range(2):
        want = np.array([pr.op.calc_field(x[b], n) for n in dirs])
        assert rel(e[:, b, :], want) < tol


def test_jones_and_cross_sections_match_oracle():
    pr = Pair("sphere", ("0.5um", "0.1um"), [1.5 + 0.1j], "1um", max_rhs=2)
    ccs = [pr.set_cc(PROP, 1, rhs=0), pr.set_cc(PROP, 2, rhs=1)]
    einc = np.stack([pr.p.einc(PROP, 1), pr.p.einc(PROP, 2)])
    pol = dda_b200.CudaSolver(pr.mv, "qmr").get_pol_vec(einc, 1e-8)
    theta, phi = PP.grid_angles("0..180/7", "0..360/5")
    # far fields of the polarisations left on the device by the solve
    j = PP.jones_far_field(pr.mv, PROP, theta, phi)
    want = pr.op.jones(pol[0], pol[1], PROP, theta, phi)
    assert rel(j, want) < 1e-10
    for r, p in enumerate((1, 2)):
        pr.op.set_cc(PROP, p, "ldr")
        cext_o, cabs_o = pr.op.cross_sections(pol[r], PROP, p)
        _, prop_n = dda_b200.beam_pol(PROP, p)
        ef = pr.mv.far_field(prop_n[None, :], nrhs=1, pol=pol[r])[0, 0]
        cext, cabs, _, _ = PP.cross_sections(pr.p, ccs[r], pol[r], ef, PROP, p)
        assert abs(cext - cext_o) < 1e-10 * abs(cext_o)
        assert abs(cabs - cabs_o) < 1e-10 * abs(cabs_o)


def test_jones_end_to_end_against_oracle_solve():
    # each side solves for itself; the Jones matrices then agree to the
    # solver tolerance
    pr = Pair("sphere", ("0.5um", "0.1um"), [1.5 + 0.1j], "1um", max_rhs=2)
    pr.set_cc(PROP, 1, rhs=0)
    pr.set_cc(PROP, 2, rhs=1)
    einc = np.stack([pr.p.einc(PROP, 1), pr.p.einc(PROP, 2)])
    dda_b200.CudaSolver(pr.mv, "bicgstab").get_pol_vec(einc, 1e-9)
    pols = []
    for p in (1, 2):
        pr.op.set_cc(PROP, p, "ldr")
        rc, pv, _, _ = pr.op.solve(pr.op.einc(PROP, p), "bicgstab", 1e-9)
        assert rc == 0
        pols.append(pv)
    theta, phi = PP.grid_angles("0..180/13", "0..360/9")
    j = PP.jones_far_field(pr.mv, PROP, theta, phi)
    assert rel(j, pr.op.jones(pols[0], pols[1], PROP, theta, phi)) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cross_sections_approach_mie(precision):
    # sphere radius 1 um, d 0.05 um, lambda 4 um, m 1.5+0.1i (the oracle's
    # own Mie pin at the same resolution)
    g = dda_b200.Geometry.sphere("1um", "0.05um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "4um")
    mv = dda_b200.CudaMatVec(p, precision)
    cc = dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr")
    mv.set_couple_constants(cc)
    pol = dda_b200.CudaSolver(mv, "qmr").get_pol_vec(p.einc((0, 0, 1), 1), 1e-8)
    _, prop_n = dda_b200.beam_pol((0, 0, 1), 1)
    ef = mv.far_field(prop_n[None, :])[0, 0]
    cext, cabs, _, _ = PP.cross_sections(p, cc, pol, ef, (0, 0, 1), 1)
    from oracle import oracle as O
    qe, _, qa = O.mie(2 * np.pi * 1e-6 / 4e-6, 1.5 + 0.1j)
    area = np.pi * 1e-12
    # the oracle lands within 1e-3 (Qext) and 3e-3 (Qabs) of Mie here
    assert abs(cext / area - qe) / qe < 1e-3
    assert abs(cabs / area - qa) / qa < 3e-3

