"""The command line: option parsing and the default grid unit on the CPU, one
small run on the GPU."""
import math
import os

import numpy as np
import pytest

import dda_b200
from dda_b200 import cli


def test_default_grid_unit_rule():
    # DDA/DDAMain.cpp:134-150: lambda / (10 max|m|), at most a 16th of each dimension
    assert abs(cli.default_grid_unit(6e-6, [20e-6], [1.5 + 0.1j]) - 6e-6 / (10 * abs(1.5 + 0.1j))) < 1e-18
    assert cli.default_grid_unit(6e-6, [1e-6], [1.5]) == pytest.approx(1e-6 / 16)


def test_geometry_strings_match_the_shapes():
    g, refr, mie = cli.build_geometry("sphere:1um,1.5+0.1i", "0.1um", [], 1e-6)
    ref = dda_b200.Geometry.sphere("1um", "0.1um")
    assert np.array_equal(g.positions, ref.positions) and refr == [1.5 + 0.1j] and mie[0] == "sphere"
    g, refr, _ = cli.build_geometry("box:(1um,0.5um,0.3um),1.33", "0.1um", [], 1e-6)
    assert g.box == (10, 5, 3) and refr == [1.33 + 0j]
    g, _, _ = cli.build_geometry("cylinder:1um,0.3um,2+0.5i", "0.1um", [], 1e-6)
    assert g.nv > 0


@pytest.mark.gpu
def test_cli_run_writes_cross_sections(tmp_path, capsys):
    rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                   "--epsilon", "8", "--efield-grid", "--output-dir", str(tmp_path)])
    assert rc == 0
    out = capsys.readouterr().out
    assert "Cext Pol1" in out and "Mie solution" in out
    for f in ("CrossSec-Pol1.txt", "CrossSec-Pol2.txt", "MieCrossSec.txt", "EFieldGrid.txt"):
        assert os.path.exists(tmp_path / f)
    assert sum(1 for _ in open(tmp_path / "EFieldGrid.txt")) == 1 + 91 * 61
    vals = dict(l.split(" = ") for l in open(tmp_path / "CrossSec-Pol1.txt").read().splitlines())
    # the same problem through the API
    g = dda_b200.Geometry.sphere("0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    mv = dda_b200.CudaMatVec(p, "fp64")
    cc = dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr")
    mv.set_couple_constants(cc)
    pol = dda_b200.CudaSolver(mv, "qmr").get_pol_vec(p.einc((0, 0, 1), 1), 1e-8)
    _, pn = dda_b200.beam_pol((0, 0, 1), 1)
    ef = mv.far_field(pn[None, :])[0, 0]
    from dda_b200 import postprocess
    cext, cabs, _, _ = postprocess.cross_sections(p, cc, pol, ef, (0, 0, 1), 1)
    assert abs(float(vals["Cext"]) - cext) <= 1e-12 * abs(cext)
    assert abs(float(vals["Cabs"]) - cabs) <= 1e-12 * abs(cabs)
