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
    g, refr, mie, _ = cli.build_geometry("sphere:1um,1.5+0.1i", "0.1um", [], 1e-6)
    ref = dda_b200.Geometry.sphere("1um", "0.1um")
    assert np.array_equal(g.positions, ref.positions) and refr == [1.5 + 0.1j] and mie[0] == "sphere"
    g, refr, _, _ = cli.build_geometry("box:(1um,0.5um,0.3um),1.33", "0.1um", [], 1e-6)
    assert g.box == (10, 5, 3) and refr == [1.33 + 0j]
    g, _, _, _ = cli.build_geometry("cylinder:1um,0.3um,2+0.5i", "0.1um", [], 1e-6)
    assert g.nv > 0


def test_far_field_option_parsing():
    from dda_b200 import postprocess as P
    assert P.parse_far_field("Plane=0..359/360,90,no-phi") == ("Plane", "0..359/360", "90", True, False, True)
    assert P.parse_far_field("X=10,20,both") == ("X", "10", "20", True, True, False)
    assert P.parse_far_field("Y=0..180/7,0,mueller")[3:5] == (False, True)
    for bad in ("Z=10", "Z=1,2,jones,mueller", "Z=1,2,foo", "a/b=1,2"):
        with pytest.raises(ValueError):
            P.parse_far_field(bad)


def test_mueller_of_simple_jones_matrices():
    from dda_b200 import postprocess as P
    eye = np.array([[[1, 0], [0, 1]]], dtype=complex)
    assert np.allclose(P.mueller(eye)[0], np.eye(4))
    # a linear polariser along the first axis: S11 = 1, the rest 0
    pol = np.array([[[1, 0], [0, 0]]], dtype=complex)
    m = P.mueller(pol)[0]
    assert np.allclose(m, 0.5 * np.array([[1, 1, 0, 0], [1, 1, 0, 0], [0, 0, 0, 0], [0, 0, 0, 0]]))


def test_field_files_round_trip(tmp_path):
    from dda_b200 import datafiles as F
    g = dda_b200.Geometry.sphere("0.3um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    rng = np.random.default_rng(2)
    v = np.zeros(p.vec_size, dtype=complex)
    for c in range(3):
        v[c * p.nvs:c * p.nvs + p.nv] = rng.normal(size=p.nv) + 1j * rng.normal(size=p.nv)
    base = str(tmp_path / "DipPol-Pol1")
    F.write(base, F.field_file(p, F.parameters(p), F.dipole_list_geometry(p), "DipolePolarization", 1, v),
            lambda path: F.field_txt(path, p, "DipolePolarization", 1, v))
    assert np.array_equal(F.load_dip_pol(base, p), v)  # the .hdf5 file, bit for bit
    assert np.max(np.abs(F.read_field_txt(base + ".txt", p) - v)) <= 1e-9 * np.max(np.abs(v))  # 10 digits
    head = open(base + ".txt").readline().split()
    assert head[:5] == ["#x", "y", "z", "|DipolePolarization-Pol1|^2", "DipolePolarization-Pol1.x.r"]
    os.remove(base + ".hdf5")
    assert np.max(np.abs(F.load_dip_pol(base, p) - v)) <= 1e-9 * np.max(np.abs(v))  # only the .txt left


@pytest.mark.gpu
def test_cli_run_writes_cross_sections(tmp_path, capsys):
    rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                   "--epsilon", "8", "--efield-grid", "--efield", "--ntheta", "36", "--mueller-matrix-grid",
                   "--far-field", "Side=90,0..360/5,both", "--store-dippol", "--store-intfield",
                   "--store-incbeam", "--write-txt", "--output-dir", str(tmp_path)])
    assert rc == 0
    out = capsys.readouterr().out
    assert "Cext Pol1" in out and "Mie solution" in out
    for f in ("CrossSec-Pol1", "CrossSec-Pol2", "MieCrossSec", "FarGrid", "FarGrid.mueller", "FarPlane", "FarSide",
              "FarSide.mueller", "DipPol-Pol1", "IntField-Pol2", "IncBeam-Pol1", "Geometry"):
        for ext in (".txt", ".hdf5"):
            assert os.path.exists(tmp_path / (f + ext)), f + ext
    from dda_b200 import matfile
    jf = matfile.load(str(tmp_path / "FarGrid.hdf5"))
    assert jf["Type"] == "JonesFarField" and jf["JonesFarField"]["Data"].shape == (1, 91 * 61, 2, 2)
    assert "DipolePositions" not in jf["Geometry"] and jf["Geometry"]["Type"] == "DDADipoleList"
    txt = np.loadtxt(tmp_path / "FarGrid.txt")
    d = jf["JonesFarField"]["Data"][0]  # [n][j][i] = J[i][j]; s1..s4 = S22, S11, S12, S21
    assert np.allclose(txt[:, 2], d[:, 1, 1].real, rtol=1e-9, atol=1e-9 * np.abs(d).max())
    assert np.allclose(txt[:, 6], d[:, 1, 0].real, rtol=1e-9, atol=1e-9 * np.abs(d).max())
    mf = matfile.load(str(tmp_path / "FarGrid.mueller.hdf5"))
    assert mf["MuellerFarField"]["Data"].shape == (1, 91 * 61, 4, 4)
    # the Mie series' far field beside it (MieFar*, DDAMain.cpp:476-489): the DDA sphere's
    # Jones matrices within the discretisation error of |m| k d = 0.95
    mie = matfile.load(str(tmp_path / "MieFarGrid.hdf5"))
    assert mie["Geometry"]["Type"] == "Mie" and mie["Geometry"]["Radius"][0] == pytest.approx(0.5e-6)
    assert np.allclose(mie["Geometry"]["RefractiveIndex"], 1.5 + 0.1j)
    assert mie["Parameters"]["Method"] == "Mie" and mie["Parameters"]["Polarizations"].shape == (2, 3)
    dm = mie["JonesFarField"]["Data"][0]
    err = np.linalg.norm(d - dm) / np.linalg.norm(dm)
    with capsys.disabled():
        print("DDA vs Mie Jones, relative 2-norm difference: %.4f" % err)
    assert err < 0.1
    for f in ("MieFarGrid.txt", "MieFarGrid.mueller.hdf5", "MieFarPlane.hdf5", "MieFarSide.mueller.txt"):
        assert os.path.exists(tmp_path / f), f
    assert sum(1 for _ in open(tmp_path / "FarGrid.txt")) == 1 + 91 * 61
    assert sum(1 for _ in open(tmp_path / "FarPlane.txt")) == 1 + 36
    assert len(open(tmp_path / "FarPlane.txt").readline().split()) == 1 + 8  # no-phi
    assert len(open(tmp_path / "FarGrid.mueller.txt").readlines()[1].split()) == 2 + 16
    # the far fields of the loaded polarisations are the same
    out2 = tmp_path / "again"
    rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                   "--load-dip-pol", str(tmp_path), "--efield-grid", "--output-dir", str(out2)])
    assert rc == 0 and "Loaded dipole polarisations" in capsys.readouterr().out
    a = matfile.load(str(tmp_path / "FarGrid.hdf5"))["JonesFarField"]["Data"]
    b = matfile.load(str(out2 / "FarGrid.hdf5"))["JonesFarField"]["Data"]
    assert np.allclose(a, b, rtol=1e-12, atol=0)
    assert not os.path.exists(out2 / "FarGrid.txt")  # text only with --write-txt
    # a solve started from the stored polarisations ends at once
    rc = cli.main(["--geometry", "sphere:0.5um,1.5+0.1i", "--lambda", "1um", "--grid-unit", "0.1um",
                   "--epsilon", "8", "--load-start-dip-pol", str(tmp_path), "--output-dir", str(out2)])
    assert rc == 0
    its = [int(l.split(":")[1].split()[0]) for l in capsys.readouterr().out.splitlines() if l.startswith("Pol")]
    assert its and max(its) <= 2
    cs = matfile.load(str(tmp_path / "CrossSec-Pol1.hdf5"))
    assert cs["Type"] == "CrossSection" and cs["BeamPolarization"].tolist() == [1]
    vals = {k: v[0] for k, v in cs["CrossSection"].items()}
    txt = dict(l.split(" = ") for l in open(tmp_path / "CrossSec-Pol1.txt").read().splitlines())
    assert list(txt) == ["Cext", "Qext", "Cabs", "Qabs", "Csca", "Qsca"]
    assert float(txt["Cext"]) == pytest.approx(vals["Cext"], rel=1e-9)
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
    mv.close()
    # the stored Geometry.hdf5 as the target: grid unit and refractive index from the file
    out3 = tmp_path / "loaded"
    rc = cli.main(["--geometry", "load:file=" + str(tmp_path), "--lambda", "1um", "--epsilon", "8",
                   "--output-dir", str(out3)])
    assert rc == 0 and "Mie solution" not in capsys.readouterr().out
    cs3 = matfile.load(str(out3 / "CrossSec-Pol1.hdf5"))["CrossSection"]
    # both solves stop at the relative residual 1e-8
    assert abs(cs3["Cext"][0] - vals["Cext"]) <= 1e-8 * abs(vals["Cext"])
    assert abs(cs3["Cabs"][0] - vals["Cabs"]) <= 1e-8 * abs(vals["Cabs"])


def test_adda_options_translate():
    # DDA/AddaOptions.cpp:57-238 on the option sets of DDA/test-adda.sh
    T = cli.translate_adda
    a = cli.parser().parse_args(T("-dpl 15".split()))
    assert api_len(a.grid_unit) == pytest.approx(2 * math.pi / 15 * 1e-6)
    assert api_len(a.geometry.split(":")[1].split(",")[0]) == pytest.approx(8 * 2 * math.pi / 15 * 1e-6)
    assert a.geometry.endswith(",1.5") and a.efield and a.mueller_matrix and a.write_txt and not a.efield_grid
    a = cli.parser().parse_args(T(("-lambda 30 -shape read box.geom -dpl 30 -store_scat_grid -scat_matr both "
                                   "-prop 10 -2 3 -orient -5 -30 10 -iter bicgstab -beam barton5 1 1 6 3").split()))
    assert a.geometry == "load:file=box.geom" and a.m == ["1.5"] and api_len(a.grid_unit) == pytest.approx(1e-6)
    assert a.efield_grid and a.mueller_matrix_grid and not a.efield and not a.mueller_matrix
    assert cli.parse_vector(a.prop) == [10, -2, 3] and cli.parse_vector(a.orient) == [-5, -30, 10]
    assert a.iter == "bicgstab"
    b = dda_b200.Beam(a.beam)
    assert b.kind == "barton5" and b.waist == pytest.approx(1e-6) and np.allclose(b.center, (1e-6, 6e-6, 3e-6))
    a = cli.parser().parse_args(T(("-dpl 15 -scat_matr muel -pol ldr avgpol -m 1.4 -0.2 -ntheta 3 -eps 1 "
                                   "-iter cgnr -maxiter 50 -store_beam -store_dip_pol -dir out").split()))
    assert a.pol == "ldr-avgpol" and a.ntheta == 6 and a.geometry.endswith(",1.4-0.2i")
    assert a.mueller_matrix and not a.efield and a.epsilon == 1 and a.iter == "cgnr" and a.maxiter == 50
    assert a.store_incbeam and a.store_dippol and a.output_dir == "out"
    assert cli.parser().parse_args(T("-dpl 15 -beam plane -scat_matr none".split())).beam == "plane"
    for bad in ("-lambda 6", "-dpl 15 -dpl 15", "-dpl 15 -size 10", "-dpl 15 -dda-cpu", "-dpl 15 -m 1.5",
                "-dpl 15 -shape box", "dpl 15"):
        with pytest.raises(SystemExit):
            T(bad.split())


def api_len(s):
    return dda_b200.api.parse_length(s)


@pytest.mark.gpu
def test_cli_adda_options_run(tmp_path, capsys):
    rc = cli.main(["--adda-options", "-dpl", "15", "-scat_matr", "both", "-prop", "1", "2", "3", "-orient", "40", "70",
                   "100", "-beam", "barton5", "10", "-pol", "ldr", "-ntheta", "4", "-dir", str(tmp_path)])
    assert rc == 0
    out = capsys.readouterr().out
    assert "Cext Pol1" in out and "Mie solution" not in out
    for f in ("CrossSec-Pol1.txt", "CrossSec-Pol2.txt", "FarPlane.txt", "FarPlane.mueller.txt", "DipPol-Pol1.txt",
              "DipPol-Pol1.hdf5", "FarPlane.hdf5"):
        assert os.path.exists(tmp_path / f), f
    assert sum(1 for _ in open(tmp_path / "FarPlane.txt")) == 1 + 8


def test_output_directories_and_tags(tmp_path):
    # EMSim/OutputDirectory.cpp: output_<n> numbered by the counter file, tags as links beside it
    parent = str(tmp_path / "out")
    a = cli.output_directory(parent)
    b = cli.output_directory(parent)
    assert os.path.basename(a) == "output_0" and os.path.basename(b) == "output_1"
    assert open(os.path.join(parent, "counter")).read().split() == ["2"]
    cli.create_tag(a, "running")
    cli.create_tag(b, "running")  # moves to the newer directory
    assert os.readlink(os.path.join(parent, "running")) == "output_1"
    for bad in ("", "a/b", ".hidden", "output_7"):
        with pytest.raises(SystemExit):
            cli.create_tag(a, bad)


def test_option_errors_before_any_gpu_work(tmp_path):
    base = ["--geometry", "sphere:0.5um,1.5", "--output-dir", str(tmp_path)]
    for extra, msg in ((["--periodicity-1", "(1um,0,0)"], "periodic"), (["--cpu", "--opencl"], "exclude"),
                       (["--tag", "x"], "both --output-dir and --tag"), (["--device", "list"], "device index")):
        with pytest.raises(SystemExit, match=msg):
            cli.main(base + extra)
    a = cli.parser().parse_args(["--cpu", "--sync", "--dmatrix-host", "--opencl-fft", "apple", "--device", "0",
                                 "--gamma", "0.01", "--verbose", "--mem-info", "--periodicity-2", "(0,0,0)"])
    assert a.cpu and a.gamma == 0.01 and a.device == "0" and a.output_dir is None


@pytest.mark.gpu
def test_cli_output_parent_dir_tags_and_log(tmp_path, capsys):
    rc = cli.main(["--geometry", "sphere:0.3um,1.5", "--lambda", "1um", "--grid-unit", "0.1um", "--ftype", "float",
                   "--efield", "--output-parent-dir", str(tmp_path), "--tag", "mine", "--verbose", "--mem-info"])
    assert rc == 0
    cap = capsys.readouterr()
    assert "couple constants" in cap.out and "Particle grid" in cap.out and "Alloc 'context'" in cap.err
    d = tmp_path / "output_0"
    log = open(d / "log").read()
    assert log.startswith("Output directory: ") and "Command: " in log and "Cext Pol1" in log
    assert "Overall time" in log
    prof = open(d / "prof").read()
    for phase in ("ddaParams cr", "Dmatrix", "res12", "output dippol", "output", "farfield", "====", "overall"):
        assert phase in prof, phase
    for tag in ("running", "mine", "latest"):
        assert os.readlink(tmp_path / tag) == "output_0"
    assert os.path.exists(d / "DipPol-Pol1.hdf5") and os.path.exists(d / "CrossSec-Pol2.txt")
    assert open(d / "meminfo").read().startswith("Alloc 'context'")
    assert "RE_00001 = " in log
    # --ftype float: fields and far fields in single precision, the Mie series in double
    from dda_b200 import matfile
    assert matfile.load(str(d / "DipPol-Pol1.hdf5"))["Field"]["Data"].dtype == np.complex64
    assert matfile.reader(str(d / "FarPlane.hdf5")).attrs_of("JonesFarField/Data") == {"MATLAB_class": "single"}
    assert matfile.load(str(d / "MieFarPlane.hdf5"))["JonesFarField"]["Data"].dtype == np.complex128


def test_help_topics(capsys):
    # "--beam help" and the like (Beam.cpp:78, GeometryParser.cpp:87, PolarizabilityDescription.cpp:36,
    # FarFieldCalc.cpp:52) print the accepted values instead of running
    for args, word in ((["--beam", "help"], "barton5"), (["--geometry=help"], "load:file="),
                       (["--pol", "help"], "ldr-avgpol"), (["--far-field", "help"], "no-phi"),
                       (["--beam", "gaussian:help"], "davis3")):
        assert cli.main(args) == 0
        assert word in capsys.readouterr().out


def test_prof_file_layout():
    # ProfilingData::toString (Core/Profiling.cpp): phases, "====", per-name totals, overall
    p = cli._Prof()
    for name in ("a", "bb", "a"):
        p.begin(name)
    p.end()
    lines = p.text().splitlines()
    assert [l.split()[0] for l in lines] == ["a", "bb", "a", "====", "=a", "=bb", "=a", "overall"]
    assert lines[-1].split()[4] == "100.0%"


def test_residual_lines():
    # RE_%05d = %12.6e with the trend mark of DDA/IterativeSolverBase.cpp:77-83
    assert cli.residual_lines([0.5, 0.25, 0.3, 0.28, 0.1]).splitlines() == [
        "RE_00001 = 5.000000e-01  + ", "RE_00002 = 2.500000e-01  + ", "RE_00003 = 3.000000e-01  - ",
        "RE_00004 = 2.800000e-01  -+", "RE_00005 = 1.000000e-01  + "]
