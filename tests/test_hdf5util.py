"""Hdf5Util (EMSim/Hdf5Util.cpp): the .hdf5 result files converted to the
text layouts give the same text as the command line writes directly."""
import numpy as np

import dda_b200
from dda_b200 import datafiles as F, hdf5util as H, matfile as M, postprocess as P


def _params():
    g = dda_b200.Geometry.from_arrays(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 1], [2, 2, 1], [1, 1, 2]]),
                                      np.array([0, 1, 0, 1, 1]), "0.1um")
    return dda_b200.DDAParams(g, [1.5 + 0.1j, 1.3], "1um")


def test_text_of_every_file_type(tmp_path, capsys):
    p = _params()
    rng = np.random.default_rng(6)
    v = np.zeros(p.vec_size, dtype=complex)
    for c in range(3):
        v[c * p.nvs:c * p.nvs + p.nv] = rng.normal(size=p.nv) + 1j * rng.normal(size=p.nv)
    pars, geo = F.parameters(p), F.dipole_list_geometry(p)
    theta, phi = P.grid_angles("0..360/9", "0..90/2")
    j = rng.normal(size=(len(theta), 2, 2)) + 1j * rng.normal(size=(len(theta), 2, 2))
    m = P.mueller(j)
    files = {
        "IntField-Pol2": (F.field_file(p, pars, geo, "InternalField", 2, v),
                          lambda out: F.field_txt(out, p, "InternalField", 2, v)),
        "Geometry": (F.geometry_file(p), lambda out: F.geometry_txt(out, p)),
        "CrossSec-Pol1": (F.cross_section_file(1, 2e-12, 0.5e-12, 1.25, 0.3125),
                          lambda out: F.cross_section_txt(out, 2e-12, 0.5e-12, 1.25, 0.3125)),
        "FarX": (F.jones_file(pars, geo, theta, phi, 3e14, j), lambda out: P.store_jones_txt(out, theta, phi, j)),
        "FarX.mueller": (F.mueller_file(pars, geo, theta, phi, 3e14, m),
                         lambda out: P.store_mueller_txt(out, theta, phi, m)),
    }
    for name, (members, writer) in files.items():
        base = str(tmp_path / name)
        F.write(base, members, writer)
        assert H.main(["hdf5-to-text", base + ".hdf5", "-o", base + ".conv.txt"]) == 0
        assert open(base + ".conv.txt").read() == open(base + ".txt").read(), name
    assert H.main(["cat", str(tmp_path / "CrossSec-Pol1.hdf5")]) == 0
    assert capsys.readouterr().out == open(tmp_path / "CrossSec-Pol1.txt").read()
    # far fields cut to theta <= 180 degrees (removeThetaLarger180), with and without phi
    assert H.main(["hdf5-to-text", "--theta-max-180", "--no-phi", str(tmp_path / "FarX.hdf5")]) == 0
    lines = open(tmp_path / "FarX.txt").read().splitlines()
    assert lines[0].startswith("#theta s1.r") and len(lines) == 1 + 5 * 2
    assert H.main(["resave-hdf5", "--theta-max-180", str(tmp_path / "FarX.mueller.hdf5")]) == 0
    cut = M.load(str(tmp_path / "FarX.mueller.new.hdf5"))["MuellerFarField"]
    assert cut["Data"].shape == (1, 10, 4, 4) and np.array_equal(cut["Data"][0], m[:10].transpose(0, 2, 1))
    assert H.main(["resave-hdf5", str(tmp_path / "IntField-Pol2.hdf5"), "-o", str(tmp_path / "again.hdf5")]) == 0
    assert np.array_equal(M.load(str(tmp_path / "again.hdf5"))["Field"]["Data"],
                          M.load(str(tmp_path / "IntField-Pol2.hdf5"))["Field"]["Data"])
    assert H.main(["cat", str(tmp_path / "IntField-Pol2.hdf5"), "--type", "Nonsense"]) == 1
    assert H.main(["hdf5-to-text", "a.hdf5", "b.hdf5", "-o", "x.txt"]) == 1


def test_jones_to_mueller(tmp_path):
    p = _params()
    rng = np.random.default_rng(7)
    theta, phi = P.grid_angles("0..180/5", "0..90/2")
    j = rng.normal(size=(len(theta), 2, 2)) + 1j * rng.normal(size=(len(theta), 2, 2))
    F.write(str(tmp_path / "FarX"), F.jones_file(F.parameters(p), F.dipole_list_geometry(p, full=False), theta, phi,
                                                 3e14, j))
    assert H.main(["jones-to-mueller", str(tmp_path / "FarX.hdf5")]) == 0
    m = M.load(str(tmp_path / "FarX.mueller.hdf5"))
    assert m["Type"] == "MuellerFarField" and m["Geometry"]["Type"] == "DDADipoleList" and m["Parameters"]["Method"] == "DDA"
    assert np.allclose(m["MuellerFarField"]["Data"][0], P.mueller(j).transpose(0, 2, 1), rtol=1e-15, atol=0)
    assert m["MuellerFarField"]["Frequency"].tolist() == [3e14]
