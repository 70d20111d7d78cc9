"""The FieldDiff tool (DDA/FieldDiff.cpp): text files by column groups,
HDF5 result files by their data."""
import math

import numpy as np
import pytest

import dda_b200
from dda_b200 import datafiles as F, fielddiff as D


def _write(path, rows, header="#theta phi a b c d"):
    with open(path, "w") as f:
        f.write(header + "\n")
        for r in rows:
            f.write(" ".join("%.17g" % x for x in r) + "\n")
        f.write("\n")  # blank lines are skipped


def test_text_groups_and_exit_codes(tmp_path, capsys):
    rng = np.random.default_rng(4)
    a = rng.normal(size=(7, 6))
    b = a.copy()
    b[:, 2:] = 2 * a[:, 2:] * (1 + 1e-6 * rng.normal(size=(7, 4)))
    _write(tmp_path / "a.txt", a)
    _write(tmp_path / "b.txt", b)
    res, n = D.compare_text(str(tmp_path / "a.txt"), str(tmp_path / "b.txt"), [(2, 1.0), (4, 2.0)])
    assert n == 7 and res[0][4] == 0.0
    x, y = 2 * a[:, 2:], b[:, 2:]
    want = math.sqrt(np.sum((y - x) ** 2) / ((np.sum(x * x) + np.sum(y * y)) / 2))
    assert res[1][0] == 28 and res[1][4] == pytest.approx(want, rel=1e-12)
    args = [str(tmp_path / "a.txt"), str(tmp_path / "b.txt"), "2", "4:2"]
    assert D.main(args) == 0 and "normalized error is" in capsys.readouterr().out
    assert D.main(["--max-error", "1e-7"] + args) == 1  # the second group is about 1e-6 apart
    assert "group 1 too large" in capsys.readouterr().err
    assert D.main(["--print-only"] + args) == 0
    assert [float(v) for v in capsys.readouterr().out.split()] == pytest.approx([0.0, want], rel=1e-9)
    _write(tmp_path / "short.txt", a[:5])
    assert D.main([str(tmp_path / "a.txt"), str(tmp_path / "short.txt"), "6"]) == 1
    assert "is longer than" in capsys.readouterr().err
    assert D.main([str(tmp_path / "a.txt"), str(tmp_path / "b.txt"), "5"]) == 1
    assert "extra fields" in capsys.readouterr().err


def test_hdf5_result_files(tmp_path, capsys):
    g = dda_b200.Geometry.sphere("0.3um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    rng = np.random.default_rng(5)
    v = np.zeros(p.vec_size, dtype=complex)
    for c in range(3):
        v[c * p.nvs:c * p.nvs + p.nv] = rng.normal(size=p.nv) + 1j * rng.normal(size=p.nv)
    w = v * (1 + 1e-5j)
    for name, vec in (("a", v), ("b", w)):
        F.write(str(tmp_path / name), F.field_file(p, F.parameters(p), F.dipole_list_geometry(p),
                                                   "DipolePolarization", 1, vec))
    assert D.main(["--print-only", str(tmp_path / "a.hdf5"), str(tmp_path / "b.hdf5")]) == 0
    got = float(capsys.readouterr().out)
    assert got == pytest.approx(D.normalised_rms(v, w), rel=1e-12) and got == pytest.approx(1e-5, rel=1e-3)
    assert D.main([str(tmp_path / "a.hdf5"), str(tmp_path / "b.hdf5")]) == 0
    assert D.main(["--max-error", "1e-6", str(tmp_path / "a.hdf5"), str(tmp_path / "b.hdf5")]) == 1
    F.write(str(tmp_path / "cs"), F.cross_section_file(1, 2e-12, 1e-12, 1.0, 0.5))
    assert D.main([str(tmp_path / "a.hdf5"), str(tmp_path / "cs.hdf5")]) == 1  # different shapes
