"""Command line in the shape of the reference's `dda` (DDA/Options.cpp:41-97,
DDA/DDAMain.cpp:611-771): one target, both polarisations, cross sections and
the far-field outputs asked for.

    python -m dda_b200.cli --geometry 'sphere:10um,1.5+0.1i' --lambda 6um --grid-unit 0.5um \\
        --iter qmr --epsilon 5 --efield-grid --output-dir out

Options (the reference's names): --lambda, --prop, --beam (plane |
gaussian:<lminus|davis3|barton5>,<waist>[,(x,y,z)]; extinction of a Gaussian beam
from the dipoles' work on the incident field), --orient (alpha,beta,gamma): the
particle orientation as ZYZ Euler angles in degrees, --pol (ldr, cm, ldr-avgpol),
--geometry (sphere:R,m | cylinder:L,R,m | box:(X,Y,Z),m | load:file=<text dipole
list> with -m), --grid-unit (default: the reference's rule, lambda / (10 max|m|)
and at most a 16th of every particle dimension, DDAMain.cpp:134-150), -m,
--fft-grid, --epsilon (stop at 10^-epsilon), --maxiter, --iter, --ftype (float,
double; plus mixed), --no-symmetry (both polarisations are always solved),
--far-field Name=theta,phi[,jones|mueller|both|none][,no-phi], --efield and
--mueller-matrix (the YZ plane, --ntheta angles, DDAMain.cpp:323-344),
--efield-grid and --mueller-matrix-grid (theta 0..180/91, phi 0..360/61),
--load-dip-pol DIR (skip the solve), --load-start-dip-pol DIR (start values),
--store-dippol, --store-intfield, --store-incbeam, --write-txt, --profiling-run
(per-stage matvec times instead of a solve), --output-dir.

--adda-options, followed by options in ADDA's syntax (-dpl, -lambda, -m, -shape
read, -prop, -orient, -beam, -pol, -eps, -iter, -maxiter, -ntheta, -scat_matr,
-store_scat_grid, -store_beam, -store_int_field, -store_dip_pol, -dir,
-dda-ftype), translated as DDA/AddaOptions.cpp:57-238 does.

Output files are text (the reference's MATLAB-style HDF5 files are not
written: no HDF5 library on these machines): CrossSec-Pol<n>.txt,
MieCrossSec.txt (spheres), Far<Name>.txt (Jones matrices, the column layout
of JonesCalculus::storeTxt) and Far<Name>.mueller.txt (Mueller matrices,
MuellerCalculus::storeTxt), and with --store-dippol / --write-txt,
--store-intfield, --store-incbeam: DipPol-Pol<n>.txt, IntField-Pol<n>.txt,
IncBeam-Pol<n>.txt (one dipole per line: grid x y z, then re, im of the x, y,
z components).  --load-dip-pol and --load-start-dip-pol read DipPol-Pol<n>.txt
files of that layout.
"""
import argparse
import math
import os
import sys

import numpy as np

from . import api, postprocess


def parse_complex(s):
    """'1.5+0.1i' (EMSim::parse) -> complex."""
    return complex(s.strip().replace(" ", "").replace("i", "j"))


def parse_vector(s, conv=float):
    v = [conv(x) for x in s.strip().strip("()").split(",")]
    if len(v) != 3:
        raise ValueError("expected three components: " + s)
    return v


def default_grid_unit(lambda_m, dims_m, refr):
    """DDA/DDAMain.cpp:134-150."""
    mmax = max(abs(c) for m in refr for c in (m if isinstance(m, (list, tuple)) else (m,)))
    gu = lambda_m / (10 * mmax)
    for d in dims_m:
        gu = min(gu, d / 16.0)
    return gu


def build_geometry(spec, grid_unit, m_opts, lambda_m):
    name, _, rest = spec.partition(":")
    name = name.strip()
    if name == "sphere":
        r, m = rest.split(",", 1)
        refr = [parse_complex(m)]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, [2 * api.parse_length(r)], refr)
        return api.Geometry.sphere(r, gu), refr, ("sphere", api.parse_length(r))
    if name == "cylinder":
        length, r, m = rest.split(",", 2)
        refr = [parse_complex(m)]
        dims = [api.parse_length(length), 2 * api.parse_length(r)]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, dims, refr)
        return api.Geometry.cylinder(length, r, gu), refr, None
    if name == "box":
        i = rest.index(")")
        xyz = rest[:i + 1].strip("()").split(",")
        refr = [parse_complex(rest[i + 1:].lstrip(","))]
        dims = [api.parse_length(x) for x in xyz]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, dims, refr)
        return api.Geometry.box_shape(*xyz, gu), refr, None
    if name == "load":
        path = rest.split("=", 1)[1] if rest.startswith("file=") else rest
        if not grid_unit:
            raise SystemExit("No --grid-unit option given but needed for loading text geometry file")
        if not m_opts:
            raise SystemExit("No -m option given for the loaded geometry")
        return api.Geometry.load(path, grid_unit), [parse_complex(m) for m in m_opts], None
    raise SystemExit("Unknown geometry option `%s'" % name)


def _is_adda_option(s):
    return len(s) >= 2 and s[0] == "-" and s[1].isalpha()


def translate_adda(args):
    """The options of an ADDA command line (what follows --adda-options) as
    options of this command line, the way parseAddaOptions does
    (DDA/AddaOptions.cpp:57-238): lengths in micrometres, -dpl dipoles per
    wavelength giving the grid unit, the default target a sphere of diameter
    16 grid units, text output, and the far fields of -scat_matr (default
    both, as in the reference) on the YZ plane or, with -store_scat_grid, on
    the angle grid."""
    opts, had = [], set()
    dpl, lam, m_values, shape = None, 2 * math.pi, [], None
    muel, ampl, grid = True, True, False
    i = 0
    while i < len(args):
        if not _is_adda_option(args[i]):
            raise SystemExit("adda options: expected an option, got `%s'" % args[i])
        name = args[i][1:]
        pars = []
        while i + 1 < len(args) and not _is_adda_option(args[i + 1]):
            i += 1
            pars.append(args[i])
        i += 1
        if name in had:
            raise SystemExit("Got adda option `%s' more than once" % name)
        had.add(name)

        def want(*counts):
            if len(pars) not in counts:
                raise SystemExit("adda option -%s: %s parameters" % (name, len(pars)))

        if name == "dpl":
            want(1)
            dpl = float(pars[0])
        elif name == "lambda":
            want(1)
            lam = float(pars[0])
        elif name == "pol":
            want(1, 2)
            opts += ["--pol", "-".join(pars)]
        elif name == "beam":
            if not pars:
                want(1)
            if pars[0] == "plane":
                want(1)
                opts += ["--beam", "plane"]
            else:
                want(2, 5)
                c = pars[2:] if len(pars) == 5 else ["0", "0", "0"]
                opts += ["--beam", "gaussian:%s,%sum,(%s)" % (pars[0], pars[1], ",".join(x + "um" for x in c))]
        elif name in ("prop", "orient"):
            want(3)
            opts += ["--" + name, "(%s)" % ",".join(pars)]
        elif name == "m":
            if not pars or len(pars) % 2:
                raise SystemExit("adda option -m: pairs of real and imaginary parts")
            m_values += ["%s%+gi" % (pars[k], float(pars[k + 1])) for k in range(0, len(pars), 2)]
        elif name == "shape":
            if not pars or pars[0] != "read":
                raise SystemExit("Unknown shape type `%s', only 'read' is known" % (pars[0] if pars else ""))
            want(2)
            shape = pars[1]
        elif name == "store_scat_grid":
            want(0)
            grid = True
        elif name == "store_beam":
            want(0)
            opts.append("--store-incbeam")
        elif name == "store_int_field":
            want(0)
            opts.append("--store-intfield")
        elif name == "store_dip_pol":
            want(0)
            opts.append("--store-dippol")
        elif name == "scat_matr":
            want(1)
            modes = {"muel": (True, False), "ampl": (False, True), "both": (True, True), "none": (False, False)}
            if pars[0] not in modes:
                raise SystemExit("Invalid value for -scat_matr `%s'" % pars[0])
            muel, ampl = modes[pars[0]]
        elif name == "eps":
            want(1)
            opts += ["--epsilon", pars[0]]
        elif name == "iter":
            want(1)
            opts += ["--iter", pars[0]]
        elif name == "maxiter":
            want(1)
            opts += ["--maxiter", pars[0]]
        elif name == "ntheta":
            want(1)
            opts += ["--ntheta", str(2 * int(pars[0]))]
        elif name == "dir":
            want(1)
            opts += ["--output-dir", pars[0]]
        elif name == "dda-ftype":
            want(1)
            opts += ["--ftype", pars[0]]
        else:  # -dda-cpu and -dda-device select the reference's OpenCL device: no counterpart
            raise SystemExit("Unknown adda option `%s'" % name)
    if dpl is None:
        raise SystemExit("No dpl option given")
    gu = lam / dpl
    opts += ["--lambda", "%.17gum" % lam, "--grid-unit", "%.17gum" % gu, "--write-txt"]
    if not m_values:
        m_values = ["1.5"]
    if shape is None:
        if len(m_values) != 1:
            raise SystemExit("adda options: one -m value for the default sphere")
        opts += ["--geometry", "sphere:%.17gum,%s" % (gu * 16 / 2, m_values[0])]
    else:
        opts += ["--geometry", "load:file=" + shape]
        for m in m_values:
            opts += ["-m", m]
    if grid:
        opts += ["--mueller-matrix-grid"] * muel + ["--efield-grid"] * ampl
    else:
        opts += ["--mueller-matrix"] * muel + ["--efield"] * ampl
    return opts


def cc_vector(params, per_material):
    """Per-material, per-axis values (nmat*3) spread over the vector layout."""
    mat = params.geometry.materials.astype(np.int64)
    v = np.zeros(params.vec_size, dtype=np.complex128)
    for c in range(3):
        v[c * params.nvs:c * params.nvs + params.nv] = np.asarray(per_material)[mat * 3 + c]
    return v


def write_field(path, params, vec):
    """One dipole per line: grid x y z, then re, im of the x, y, z components."""
    nv, nvs = params.nv, params.nvs
    cols = [params.geometry.positions.astype(np.float64)]
    for c in range(3):
        cols += [vec[c * nvs:c * nvs + nv].real[:, None], vec[c * nvs:c * nvs + nv].imag[:, None]]
    np.savetxt(path, np.hstack(cols), fmt=["%d"] * 3 + ["%.17g"] * 6,
               header="x y z  Ex.r Ex.i Ey.r Ey.i Ez.r Ez.i")


def read_field(path, params):
    """Inverse of write_field; the dipoles must be those of the target."""
    d = np.loadtxt(path, ndmin=2)
    if d.shape != (params.nv, 9) or not np.array_equal(d[:, :3].astype(np.uint32), params.geometry.positions):
        raise SystemExit("`%s' does not hold this target's dipoles" % path)
    v = np.zeros(params.vec_size, dtype=np.complex128)
    for c in range(3):
        v[c * params.nvs:c * params.nvs + params.nv] = d[:, 3 + 2 * c] + 1j * d[:, 4 + 2 * c]
    return v


def parser():
    """The command line's options (the reference's names, DDA/Options.cpp:41-97)."""
    ap = argparse.ArgumentParser(prog="dda_b200.cli", description=__doc__.split("\n\n")[0])
    ap.add_argument("--lambda", dest="lam", default="%.17gum" % (2 * math.pi))
    ap.add_argument("--prop", default="(0,0,1)")
    ap.add_argument("--beam", default="plane")
    ap.add_argument("--orient", default="(0,0,0)")
    ap.add_argument("--pol", default="ldr", choices=["ldr", "cm", "ldr-avgpol"])
    ap.add_argument("--geometry", default="sphere:3.35103um,1.5")
    ap.add_argument("--grid-unit")
    ap.add_argument("-m", action="append", default=[])
    ap.add_argument("--no-symmetry", action="store_true")
    ap.add_argument("--fft-grid", default="(0,0,0)")
    ap.add_argument("--epsilon", type=float, default=5)
    ap.add_argument("--maxiter", type=int, default=0)
    ap.add_argument("--iter", default="qmr", choices=sorted(api.SOLVERS))
    ap.add_argument("--ftype", default="double", choices=["float", "double", "mixed"])
    ap.add_argument("--far-field", action="append", default=[])
    ap.add_argument("--efield", action="store_true")
    ap.add_argument("--mueller-matrix", action="store_true")
    ap.add_argument("--ntheta", type=int, default=0)
    ap.add_argument("--efield-grid", action="store_true")
    ap.add_argument("--mueller-matrix-grid", action="store_true")
    ap.add_argument("--load-dip-pol")
    ap.add_argument("--load-start-dip-pol")
    ap.add_argument("--store-dippol", action="store_true")
    ap.add_argument("--store-intfield", action="store_true")
    ap.add_argument("--store-incbeam", action="store_true")
    ap.add_argument("--write-txt", action="store_true")
    ap.add_argument("--profiling-run", action="store_true")
    ap.add_argument("--output-dir", default=".")
    return ap


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if "--adda-options" in argv:  # DDA/Options.cpp:122-133
        k = argv.index("--adda-options")
        argv = argv[:k] + translate_adda(argv[k + 1:])
    a = parser().parse_args(argv)

    lambda_m = api.parse_length(a.lam)
    prop = tuple(parse_vector(a.prop))
    orient = tuple(parse_vector(a.orient))
    geom, refr, mie_geom = build_geometry(a.geometry, a.grid_unit, a.m, lambda_m)
    grid = tuple(int(x) for x in parse_vector(a.fft_grid, float))
    params = api.DDAParams(geom, refr, lambda_m, grid=grid if any(grid) else None)
    prec = {"float": "fp32", "double": "fp64", "mixed": "mixed"}[a.ftype]
    os.makedirs(a.output_dir, exist_ok=True)
    out = sys.stdout
    out.write("nv = %d, grid unit = %.6g um, box = %s, FFT grid = %s\n"
              % (params.nv, params.grid_unit * 1e6, params.box, params.grid))

    mv = api.CudaMatVec(params, prec, max_rhs=2)
    ccs = []
    for r, pol in enumerate((1, 2)):
        ccs.append(api.CoupleConstants(params, prop, pol, a.pol, orient=orient))
        mv.set_couple_constants(ccs[-1], rhs=r)
    if a.profiling_run:  # IterativeSolverBase::profilingRun, DDA/IterativeSolverBase.cpp:105-136
        ms = mv.profile(nrhs=2, reps=5)
        out.write("matvec (2 rhs): %.3f ms  [x forward %.3f, y/z %.3f, x inverse %.3f]\n"
                  % (ms[3], ms[0], ms[1], ms[2]))
        mv.close()
        return 0
    beam = api.Beam(a.beam)
    einc = np.stack([beam.einc(params, prop, 1, orient=orient), beam.einc(params, prop, 2, orient=orient)])
    if a.store_incbeam:
        for r in range(2):
            write_field(os.path.join(a.output_dir, "IncBeam-Pol%d.txt" % (r + 1)), params, einc[r])
    if a.load_dip_pol:  # DDA/DDAMain.cpp:374-378
        pol = np.stack([read_field(os.path.join(a.load_dip_pol, "DipPol-Pol%d.txt" % (r + 1)), params)
                        for r in range(2)])
        out.write("Loaded dipole polarisations from %s\n" % a.load_dip_pol)
    else:
        start = None
        if a.load_start_dip_pol:  # DDA/DDAMain.cpp:391-394
            start = np.stack([read_field(os.path.join(a.load_start_dip_pol, "DipPol-Pol%d.txt" % (r + 1)),
                                         params) for r in range(2)])
        solver = api.CudaSolver(mv, a.iter, max_iter=a.maxiter)
        pol = solver.get_pol_vec(einc, 10.0 ** -a.epsilon, start=start)
        for r, (st, hist) in enumerate(zip(solver.last_stats, solver.last_history)):
            out.write("Pol%d: %d iterations, relative residual %.3e\n" % (r + 1, st.iterations, st.rel_residual))
            for i, h in enumerate(hist):
                out.write("RE_%d = %.10g\n" % (i + 1, h))
    for r in range(2):
        if a.store_dippol or a.write_txt:
            write_field(os.path.join(a.output_dir, "DipPol-Pol%d.txt" % (r + 1)), params, pol[r])
        if a.store_intfield:  # internal field chi^-1 P, DDA/DDAMain.cpp:411-417
            write_field(os.path.join(a.output_dir, "IntField-Pol%d.txt" % (r + 1)), params,
                        cc_vector(params, ccs[r].chi_inv) * pol[r])

    pn = api.beam_frame(prop, orient)[0]  # forward direction in the particle frame
    ef = mv.far_field(pn[None, :], nrhs=2, pol=pol)[0]
    for r in range(2):
        cext, cabs, qext, qabs = postprocess.cross_sections(params, ccs[r], pol[r], ef[r], prop, r + 1,
                                                            einc=None if beam.plane else einc[r], orient=orient)
        csca, qsca = cext - cabs, qext - qabs
        label = "Pol%d" % (r + 1)
        out.write("Cext %s = %-25s Qext %s = %.10g\n" % (label, "%.10g um^2" % (cext * 1e12), label, qext))
        out.write("Cabs %s = %-25s Qabs %s = %.10g\n" % (label, "%.10g um^2" % (cabs * 1e12), label, qabs))
        out.write("Csca %s = %-25s Qsca %s = %.10g\n" % (label, "%.10g um^2" % (csca * 1e12), label, qsca))
        with open(os.path.join(a.output_dir, "CrossSec-%s.txt" % label), "w") as f:
            f.write("BeamPolarization = %d\nCext = %.17g\nQext = %.17g\nCabs = %.17g\nQabs = %.17g\n"
                    "Csca = %.17g\nQsca = %.17g\n" % (r + 1, cext, qext, cabs, qabs, csca, qsca))
    if mie_geom is not None and beam.plane:  # DDA/DDAMain.cpp:431
        radius = mie_geom[1]
        x = 2 * math.pi * radius / lambda_m
        qe, qs, qa = postprocess.mie(x, refr[0])
        out.write("Mie solution:\nQext = %.10g Qabs = %.10g Qsca = %.10g\n" % (qe, qa, qs))
        with open(os.path.join(a.output_dir, "MieCrossSec.txt"), "w") as f:
            f.write("Qext = %.17g\nQabs = %.17g\nQsca = %.17g\n" % (qe, qa, qs))
    # far fields (DDA/DDAMain.cpp:318-353): the angle lists of all options,
    # each list computed once for both polarisations
    far = [postprocess.parse_far_field(x) for x in a.far_field]
    if a.efield or a.mueller_matrix:
        nt = a.ntheta or (180 if params.nv < 1000 else 360 if params.nv < 10000 else 720 if params.nv < 100000
                          else 1440)
        th = "0..%.20f/%d" % (360.0 - 360.0 / nt, nt)
        if a.efield:
            far.append(("Plane", th, "90", True, False, True))
        if a.mueller_matrix:
            far.append(("Plane", th, "90", False, True, True))
    if a.efield_grid:
        far.append(("Grid", "0..180/91", "0..360/61", True, False, False))
    if a.mueller_matrix_grid:
        far.append(("Grid", "0..180/91", "0..360/61", False, True, False))
    cache = {}
    for name, ts, ps, want_j, want_m, no_phi in far:
        if (ts, ps) not in cache:
            theta, phi = postprocess.grid_angles(ts, ps)
            cache[(ts, ps)] = (theta, phi, postprocess.jones_far_field(mv, prop, theta, phi, pol=pol,
                                                                       orient=orient))
        theta, phi, jones = cache[(ts, ps)]
        if want_j:
            postprocess.store_jones_txt(os.path.join(a.output_dir, "Far%s.txt" % name), theta, phi, jones,
                                        store_phi=not no_phi)
        if want_m:
            postprocess.store_mueller_txt(os.path.join(a.output_dir, "Far%s.mueller.txt" % name), theta, phi,
                                          postprocess.mueller(jones), no_phi=no_phi)
    mv.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
