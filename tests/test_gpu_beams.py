"""Solves driven by Gaussian beams on the GPU against the oracle's FP64
solves of the same incident field (Beams::Gaussian::createEInc,
DDA/Beam.cpp:196-263; Beam::extCross, DDA/Beam.cpp:58-67), and the command
line's --beam option."""
import os

import numpy as np
import pytest

import dda_b200
from dda_b200 import cli, postprocess
from oracle import oracle as O


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["lminus", "barton5"])
def test_gaussian_beam_solve_matches_oracle(kind):
    g = dda_b200.Geometry.sphere("0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "2um")
    op = O.Problem(O.Geometry.sphere("0.5um", "0.1um"), [1.5 + 0.1j], "2um")
    op.build_dmatrix()
    prop = (0.0, 0.6, 0.8)
    beam = dda_b200.Beam("gaussian:%s,0.8um,(0.2um,0um,0um)" % kind)
    mv = dda_b200.CudaMatVec(p, "fp64", max_rhs=2)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
    einc = np.stack([beam.einc(p, prop, pol) for pol in (1, 2)])
    P = dda_b200.CudaSolver(mv, "qmr").get_pol_vec(einc, 1e-10)
    for r, pol in enumerate((1, 2)):
        op.set_cc(prop, pol, "ldr")
        e_ref = op.einc_gaussian(prop, pol, kind, 0.8e-6, (0.2e-6, 0.0, 0.0))
        assert rel(einc[r], e_ref) < 1e-13
        rc, P_ref, _, _ = op.solve(e_ref, "qmr", 1e-10)
        assert rc == 0
        assert rel(P[r], P_ref) < 1e-8
        c = postprocess.ext_cross_general(p, P[r], einc[r])
        assert c == pytest.approx(postprocess.ext_cross_general(p, P_ref, e_ref), rel=1e-8)
        assert c > 0
    mv.close()


@pytest.mark.gpu
def test_cli_gaussian_beam(tmp_path, capsys):
    rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                   "--beam", "gaussian:davis3,0.6um", "--epsilon", "8", "--store-incbeam",
                   "--output-dir", str(tmp_path)])
    assert rc == 0
    out = capsys.readouterr().out
    assert "Cext Pol1" in out and "Mie solution" not in out  # Mie only for plane waves
    vals = dict(l.split(" = ") for l in open(tmp_path / "CrossSec-Pol1.txt").read().splitlines())
    assert float(vals["Cext"]) > float(vals["Cabs"]) > 0
    assert os.path.exists(tmp_path / "IncBeam-Pol2.hdf5")
    g = dda_b200.Geometry.sphere("0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    from dda_b200 import datafiles
    stored = datafiles.load_dip_pol(str(tmp_path / "IncBeam-Pol2"), p)
    assert rel(stored, p.einc((0, 0, 1), 2, beam="gaussian:davis3,0.6um")) < 1e-12
