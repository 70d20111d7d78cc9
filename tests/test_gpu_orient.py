"""Oriented particles on the GPU (--orient): a quarter turn about the beam
axis leaves a cubic-symmetric voxel sphere's Jones matrices and cross
sections unchanged, and an oriented solve matches the oracle's FP64 solve of
the same beam in the particle frame."""
import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess
from oracle import oracle as O


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def solve(p, prop, orient, prec="fp64"):
    mv = dda_b200.CudaMatVec(p, prec, max_rhs=2)
    ccs = []
    for r, pol in enumerate((1, 2)):
        ccs.append(dda_b200.CoupleConstants(p, prop, pol, "ldr", orient=orient))
        mv.set_couple_constants(ccs[-1], rhs=r)
    einc = np.stack([p.einc(prop, pol, orient=orient) for pol in (1, 2)])
    pol = dda_b200.CudaSolver(mv, "qmr").get_pol_vec(einc, 1e-10)
    return mv, ccs, einc, pol


@pytest.mark.gpu
def test_quarter_turn_of_a_symmetric_sphere():
    g = dda_b200.Geometry.sphere("0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    prop = (0.0, 0.0, 1.0)
    theta, phi = postprocess.grid_angles("0..180/19", "0..360/13")
    out = []
    for orient in ((0, 0, 0), (90, 0, 0)):
        mv, ccs, einc, pol = solve(p, prop, orient)
        jones = postprocess.jones_far_field(mv, prop, theta, phi, pol=pol, orient=orient)
        pn = dda_b200.beam_frame(prop, orient)[0]
        ef = mv.far_field(pn[None, :], nrhs=2, pol=pol)[0]
        cs = [postprocess.cross_sections(p, ccs[r], pol[r], ef[r], prop, r + 1, orient=orient)[:2] for r in range(2)]
        out.append((jones, np.array(cs)))
        mv.close()
    assert rel(out[1][0], out[0][0]) < 1e-9
    assert np.allclose(out[1][1], out[0][1], rtol=1e-9, atol=0)


@pytest.mark.gpu
def test_oriented_solve_matches_oracle():
    g = dda_b200.Geometry.box_shape("0.7um", "0.5um", "0.4um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    op = O.Problem(O.Geometry.box("0.7um", "0.5um", "0.4um", "0.1um"), [1.5 + 0.1j], "1um")
    op.build_dmatrix()
    prop, orient = (0.0, 0.0, 1.0), (30, 40, 50)
    mv, ccs, einc, pol = solve(p, prop, orient)
    pn, p1, p2, _ = O.beam_frame(prop, orient)
    for r, pv in enumerate((p1, p2)):
        op.set_cc_frame(pn, pv, "ldr")
        rc, want, _, _ = op.solve(op.einc_frame(pn, pv), "qmr", 1e-10)
        assert rc == 0
        assert rel(pol[r], want) < 1e-8
    mv.close()


@pytest.mark.gpu
def test_cli_orient(tmp_path, capsys):
    from dda_b200 import cli
    vals = []
    for orient, sub in (("(0,0,0)", "a"), ("(90,0,0)", "b")):
        rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                       "--orient", orient, "--epsilon", "10", "--output-dir", str(tmp_path / sub)])
        assert rc == 0
        vals.append(dict(l.split(" = ") for l in open(tmp_path / sub / "CrossSec-Pol1.txt").read().splitlines()))
    capsys.readouterr()
    for key in ("Cext", "Cabs"):
        assert float(vals[1][key]) == pytest.approx(float(vals[0][key]), rel=1e-8)
