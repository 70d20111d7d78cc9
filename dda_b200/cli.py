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
list, with -m and --grid-unit> | load:file=<HDF5 geometry file, or a directory
holding Geometry.hdf5>: grid unit, refractive indices and orientation from the
file unless --grid-unit, -m or --orient are given, DDAMain.cpp:156-235),
--grid-unit (default: the reference's rule, lambda / (10 max|m|)
and at most a 16th of every particle dimension, DDAMain.cpp:134-150), -m,
--fft-grid, --epsilon (stop at 10^-epsilon), --maxiter, --iter, --ftype (float,
double; plus mixed), --no-symmetry (both polarisations are always solved),
--far-field Name=theta,phi[,jones|mueller|both|none][,no-phi], --efield and
--mueller-matrix (the YZ plane, --ntheta angles, DDAMain.cpp:323-344),
--efield-grid and --mueller-matrix-grid (theta 0..180/91, phi 0..360/61),
--load-dip-pol DIR (skip the solve), --load-start-dip-pol DIR (start values),
--store-dippol, --store-intfield, --store-incbeam, --write-txt, --profiling-run
(per-stage matvec times instead of a solve), --verbose (the couple constants and the
beam), --mem-info (the context's device memory on stderr; always in the meminfo file), --gamma (stored in the output
files' parameters), --periodicity-1/-2 (only (0,0,0): periodic targets are not
supported), --device (the CUDA device index; auto = 0), --cpu, --opencl, --sync,
--dmatrix-host, --opencl-fft (accepted; the solve runs on the GPU with CUDA).
Output directory (DDAMain.cpp:683-706, EMSim/OutputDirectory.cpp): --output-dir,
or else a new output_<n> under --output-parent-dir (default ./output) numbered by
its counter file, tagged "running" while the run lasts and with --tag names and
"latest" at its end (symbolic links beside it); stdout is copied to its log file.

--adda-options, followed by options in ADDA's syntax (-dpl, -lambda, -m, -shape
read, -prop, -orient, -beam, -pol, -eps, -iter, -maxiter, -ntheta, -scat_matr,
-store_scat_grid, -store_beam, -store_int_field, -store_dip_pol, -dir,
-dda-ftype), translated as DDA/AddaOptions.cpp:57-238 does.

Output files, as the reference writes them (DDAMain.cpp:265, 380-480): the
MATLAB-style HDF5 files (dda_b200.matfile; dda_b200.datafiles for their
structures) Geometry.hdf5, DipPol-Pol<n>.hdf5, CrossSec-Pol<n>.hdf5,
MieCrossSec.hdf5 (spheres, plane wave), Far<Name>.hdf5 (Jones matrices) and
Far<Name>.mueller.hdf5 (Mueller matrices), for spheres under a plane wave also
the Mie series' MieFar<Name>.hdf5 and MieFar<Name>.mueller.hdf5, with --store-intfield
IntField-Pol<n>.hdf5 and with --store-incbeam IncBeam-Pol<n>.hdf5; the cross
sections also as CrossSec-Pol<n>.txt and MieCrossSec.txt; with --write-txt
every file also in the reference's text layout (.txt: fields one dipole per
line with coordinates in metres and |E|^2, JonesCalculus::storeTxt,
MuellerCalculus::storeTxt, the geometry's dipole list).  --load-dip-pol and
--load-start-dip-pol read DipPol-Pol<n>.hdf5, or DipPol-Pol<n>.txt where only
that exists (DDA/Load.cpp:110-135).
"""
import argparse
import math
import os
import sys
import time

import numpy as np

from . import api, datafiles, matfile, postprocess


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


def load_hdf5_geometry(path, grid_unit, m_opts):
    """--geometry load:file=<HDF5 file> (DDAMain.cpp:163-235): (geometry,
    refractive indices, orientation from the file or None)."""
    try:
        f = datafiles.load_geometry(path)
    except (ValueError, matfile.MatFileError) as e:
        raise SystemExit("`%s': %s" % (path, e))
    if grid_unit:
        gu = api.parse_length(grid_unit)
    elif "grid_unit" in f:
        gu = f["grid_unit"]
    else:
        raise SystemExit("No --grid-unit option and no GridSpacing object in Geometry object in geometry file")
    if m_opts:
        refr = [parse_complex(m) for m in m_opts]
    elif "refractive_indices" in f:
        refr = [r[0] if r[0] == r[1] == r[2] else r for r in f["refractive_indices"]]
    else:
        raise SystemExit("No -m option given and no RefractiveIndices object in Geometry object in geometry file")
    geom = api.Geometry.from_arrays(f["positions"], f["materials"], "%.17gm" % gu)
    if "origin" in f:
        # this library places the dipole box's centre at the origin
        # (DipoleGeometry::moveToCenter); other grid origins are not supported
        centred = -(np.asarray(geom.box, dtype=np.float64) - 1) / 2 * gu
        if np.max(np.abs(f["origin"] + f["shift"] * gu - centred)) > 1e-6 * gu:
            raise SystemExit("`%s': a GridOrigin other than the centre of the dipole box is not supported" % path)
    return geom, refr, f.get("orientation")


def build_geometry(spec, grid_unit, m_opts, lambda_m):
    """(geometry, refractive indices, ("sphere", radius) for Mie or None,
    orientation stored in a loaded HDF5 geometry or None)."""
    name, _, rest = spec.partition(":")
    name = name.strip()
    if name == "sphere":
        r, m = rest.split(",", 1)
        refr = [parse_complex(m)]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, [2 * api.parse_length(r)], refr)
        return api.Geometry.sphere(r, gu), refr, ("sphere", api.parse_length(r)), None
    if name == "cylinder":
        length, r, m = rest.split(",", 2)
        refr = [parse_complex(m)]
        dims = [api.parse_length(length), 2 * api.parse_length(r)]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, dims, refr)
        return api.Geometry.cylinder(length, r, gu), refr, None, None
    if name == "box":
        i = rest.index(")")
        xyz = rest[:i + 1].strip("()").split(",")
        refr = [parse_complex(rest[i + 1:].lstrip(","))]
        dims = [api.parse_length(x) for x in xyz]
        gu = grid_unit or "%.17gm" % default_grid_unit(lambda_m, dims, refr)
        return api.Geometry.box_shape(*xyz, gu), refr, None, None
    if name == "load":
        path = rest.split("=", 1)[1] if rest.startswith("file=") else rest
        if os.path.isdir(path):
            path = os.path.join(path, "Geometry.hdf5")
        if matfile.is_hdf5(path):
            geom, refr, orient = load_hdf5_geometry(path, grid_unit, m_opts)
            return geom, refr, None, orient
        if not grid_unit:
            raise SystemExit("No --grid-unit option given but needed for loading text geometry file")
        if not m_opts:
            raise SystemExit("No -m option given for the loaded geometry")
        return api.Geometry.load(path, grid_unit), [parse_complex(m) for m in m_opts], None, None
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


def residual_lines(hist):
    """The RE lines of IterativeSolverBase::getPolVec (DDA/IterativeSolverBase.cpp:
    64-95): the iteration as five digits, the relative residual in scientific
    notation, and "+ " for a new minimum, "-+" for a drop below the previous
    step's residual, "- " otherwise (the progress and time-left columns, which
    need per-iteration wall times, are left out)."""
    lines, best, prev = [], None, None
    for i, h in enumerate(hist):
        if best is None or h <= best:
            mark, best = "+ ", h
        elif h < prev:
            mark = "-+"
        else:
            mark = "- "
        lines.append("RE_%05d = %12.6e  %s\n" % (i + 1, h, mark))
        prev = h
    return "".join(lines)


def cc_vector(params, per_material):
    """Per-material, per-axis values (nmat*3) spread over the vector layout."""
    mat = params.geometry.materials.astype(np.int64)
    v = np.zeros(params.vec_size, dtype=np.complex128)
    for c in range(3):
        v[c * params.nvs:c * params.nvs + params.nv] = np.asarray(per_material)[mat * 3 + c]
    return v


def parser():
    """The command line's options (the reference's names, DDA/Options.cpp:41-97)."""
    ap = argparse.ArgumentParser(prog="dda_b200.cli", description=__doc__.split("\n\n")[0])
    ap.add_argument("--lambda", dest="lam", default="%.17gum" % (2 * math.pi))
    ap.add_argument("--prop", default="(0,0,1)")
    ap.add_argument("--beam", default="plane")
    ap.add_argument("--orient")
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
    ap.add_argument("--output-dir")
    ap.add_argument("--output-parent-dir", action="append", default=[])
    ap.add_argument("--tag", action="append", default=[])
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--mem-info", action="store_true")
    ap.add_argument("--gamma", type=float, default=0.001)
    ap.add_argument("--periodicity-1", dest="periodicity1", default="(0,0,0)")
    ap.add_argument("--periodicity-2", dest="periodicity2", default="(0,0,0)")
    ap.add_argument("--device", default="auto")
    for flag in ("--cpu", "--opencl", "--sync", "--dmatrix-host"):
        ap.add_argument(flag, action="store_true")
    ap.add_argument("--opencl-fft")
    return ap


def output_directory(parent):
    """A new directory output_<n> under `parent` (EMSim::OutputDirectory,
    EMSim/OutputDirectory.cpp:46-116): n is read from parent/counter and the
    counter advanced under a lock on parent/counter.lck."""
    import fcntl
    os.makedirs(parent, exist_ok=True)
    counter = os.path.join(parent, "counter")
    with open(counter + ".lck", "a") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        try:
            with open(counter) as f:
                n = int(f.read().split()[0])
        except (OSError, ValueError, IndexError):
            n = 0
        with open(counter + ".new", "w") as f:
            f.write("%d\n" % (n + 1))
        os.replace(counter + ".new", counter)
    path = os.path.join(parent, "output_%d" % n)
    os.mkdir(path)
    return path


def create_tag(path, tag):
    """A symbolic link `tag` beside the output directory `path`
    (OutputDirectory::createTag, EMSim/OutputDirectory.cpp:118-128)."""
    if not tag or "/" in tag or tag[0] == "." or tag.startswith("output_"):
        raise SystemExit("Invalid tag `%s'" % tag)
    link = os.path.join(os.path.dirname(path), tag)
    if os.path.lexists(link):
        os.unlink(link)
    os.symlink(os.path.basename(path), link)


class _Prof:
    """Consecutive named phases with their wall-clock and CPU time, written as
    the reference's prof file (ProfilingData::toString, Core/Profiling.cpp:
    47-150: per phase the milliseconds and the share of the total, then the
    totals per name and overall)."""

    def __init__(self):
        self.phases, self.cur = [], None

    def begin(self, name):
        self.end()
        self.cur = (name, time.perf_counter(), time.process_time())

    def end(self):
        if self.cur:
            name, t, c = self.cur
            self.phases.append((name, (time.perf_counter() - t) * 1e3, (time.process_time() - c) * 1e3))
            self.cur = None

    def overall(self):
        self.end()
        return sum(p[1] for p in self.phases), sum(p[2] for p in self.phases)

    def text(self):
        real, cpu = self.overall()
        width = max([len("overall")] + [len(p[0]) for p in self.phases]) + 1
        pct = lambda v, o: 100.0 * v / o if o > 0 else float("nan")
        row = lambda n, r, c: "%-*s %10.3f ms = %5.1f%% %10.3f ms = %5.1f%% \n" % (width, n, r, pct(r, real), c,
                                                                                    pct(c, cpu))
        totals = {}
        for n, r, c in self.phases:
            tr, tc = totals.get(n, (0.0, 0.0))
            totals[n] = (tr + r, tc + c)
        return ("".join(row(n, r, c) for n, r, c in self.phases) + "====\n"
                + "".join(row("=" + n, *totals[n]) for n, _, _ in self.phases) + row("overall", real, cpu))


class _Tee:
    """stdout copied to the output directory's log file (DDAMain.cpp:711-712)."""

    def __init__(self, *streams):
        self.streams = streams

    def write(self, text):
        for st in self.streams:
            st.write(text)

    def flush(self):
        for st in self.streams:
            st.flush()


HELP_TOPICS = {
    "--geometry": ("Geometry options:\n"
                   "  sphere:<radius>,<m>\n"
                   "  cylinder:<length>,<radius>,<m>\n"
                   "  box:(<x>,<y>,<z>),<m>\n"
                   "  load:file=<filename>   a text dipole list (with -m and --grid-unit), an HDF5\n"
                   "                         geometry file, or a directory holding Geometry.hdf5\n"),
    "--beam": ("Beams:\n"
               "  plane\n"
               "  gaussian:lminus,<waist size>[,(x,y,z)]\n"
               "  gaussian:davis3,<waist size>[,(x,y,z)]\n"
               "  gaussian:barton5,<waist size>[,(x,y,z)]\n"),
    "--pol": ("Polarizability descriptions:\n"
              "  cm          Clausius-Mossotti\n"
              "  ldr         lattice dispersion relation (Draine and Goodman)\n"
              "  ldr-avgpol  lattice dispersion relation, polarisation-averaged\n"),
    "--far-field": ("--far-field FileName=theta,phi[,jones|mueller|both|none][,no-phi]\n"
                    "  theta and phi: an angle in degrees, or start..end/count (degrees)\n"
                    "  jones (default), mueller or both: the matrices written\n"
                    "  no-phi: no phi column in the text files\n"
                    "  files: Far<FileName>.hdf5, Far<FileName>.mueller.hdf5 (and .txt with --write-txt)\n"),
}


def help_topic(argv):
    """The text for `--geometry help`, `--beam help` (or `gaussian:help`),
    `--pol help` and `--far-field help` (the help values of GeometryParser,
    Beam, PolarizabilityDescription and FarFieldOption), or None."""
    for i, arg in enumerate(argv):
        opt, eq, val = arg.partition("=")
        if not eq:
            val = argv[i + 1] if i + 1 < len(argv) else ""
        if opt in HELP_TOPICS and val in ("help", "gaussian:help"):
            return HELP_TOPICS[opt]
    return None


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    topic = help_topic(argv)
    if topic is not None:
        sys.stdout.write(topic)
        return 0
    if "--adda-options" in argv:  # DDA/Options.cpp:122-133
        k = argv.index("--adda-options")
        argv = argv[:k] + translate_adda(argv[k + 1:])
    a = parser().parse_args(argv)
    if a.cpu and a.opencl:  # DDAMain.cpp:709
        raise SystemExit("--cpu and --opencl exclude each other")
    if a.output_dir and a.tag:
        raise SystemExit("Error: Got both --output-dir and --tag")
    for per in (a.periodicity1, a.periodicity2):
        if any(api.parse_length(x.strip()) != 0 for x in per.strip().strip("()").split(",")):
            raise SystemExit("periodic targets (--periodicity-1, --periodicity-2) are not supported")
    if a.device != "auto" and not a.device.isdigit():
        raise SystemExit("--device takes a CUDA device index or `auto' (the OpenCL device names do not apply)")
    device = 0 if a.device == "auto" else int(a.device)
    if a.output_dir:
        out_dir, tagged = a.output_dir, None
        os.makedirs(out_dir, exist_ok=True)
    else:
        tagged = out_dir = output_directory(a.output_parent_dir[-1] if a.output_parent_dir else "output")
        create_tag(tagged, "running")
    a.output_dir = out_dir
    log = open(os.path.join(out_dir, "log"), "w")
    prof = _Prof()
    try:
        out = _Tee(sys.stdout, log)
        rc = _run(a, argv, out, device, prof)
        with open(os.path.join(out_dir, "prof"), "w") as f:  # DDAMain.cpp:744-755
            f.write(prof.text() + "\n")
        out.write("Overall time %10.3f ms, %10.3f ms\n" % prof.overall())
        out.write("Output directory: %s\n" % os.path.abspath(out_dir))
    finally:
        log.close()
    if tagged:
        for t in a.tag:
            create_tag(tagged, t)
        create_tag(tagged, "latest")
    return rc


def _run(a, argv, out, device, prof):
    out.write("Output directory: %s\n" % os.path.abspath(a.output_dir))
    out.write("Command: %s\n" % " ".join(argv))
    prof.begin("ddaParams cr")  # the phase names of DDAMain.cpp's ProfileHandles
    lambda_m = api.parse_length(a.lam)
    prop = tuple(parse_vector(a.prop))
    geom, refr, mie_geom, file_orient = build_geometry(a.geometry, a.grid_unit, a.m, lambda_m)
    # the orientation stored in a loaded geometry, unless --orient is given (DDAMain.cpp:221-225)
    orient = tuple(parse_vector(a.orient)) if a.orient else (file_orient or (0.0, 0.0, 0.0))
    grid = tuple(int(x) for x in parse_vector(a.fft_grid, float))
    params = api.DDAParams(geom, refr, lambda_m, grid=grid if any(grid) else None)
    prec = {"float": "fp32", "double": "fp64", "mixed": "mixed"}[a.ftype]
    ftype = "float" if a.ftype == "float" else "double"
    out.write("Particle grid: (%d, %d, %d), FFT grid: (%d, %d, %d)\n" % (tuple(params.box) + tuple(params.grid)))
    out.write("Total dipoles: %d, Non-void dipoles: %d\n" % (int(np.prod(params.box)), params.nv))
    out.write("nv = %d, grid unit = %.6g um, box = %s, FFT grid = %s\n"
              % (params.nv, params.grid_unit * 1e6, params.box, params.grid))
    odir = lambda name: os.path.join(a.output_dir, name)
    txt = a.write_txt
    pars = datafiles.parameters(params, a.geometry, a.gamma)
    full_geometry = datafiles.dipole_list_geometry(params, orient, full=True)
    datafiles.write(odir("Geometry"), {"Type": "Geometry", "Geometry": full_geometry},
                    (lambda p: datafiles.geometry_txt(p, params)) if txt else None)  # DDAMain.cpp:265

    def store_field(base, name, r, vec):  # createDDAFieldFile(...)->write, DDAMain.cpp:380-425
        datafiles.write(odir(base), datafiles.field_file(params, pars, full_geometry, name, r + 1, vec, ftype),
                        (lambda p: datafiles.field_txt(p, params, name, r + 1, vec, ftype)) if txt else None)

    def load_pol(d):  # Load<ftype>::loadDipPol, DDA/Load.cpp:110-135
        try:
            return np.stack([datafiles.load_dip_pol(os.path.join(d, "DipPol-Pol%d" % (r + 1)), params)
                             for r in range(2)])
        except (OSError, ValueError, KeyError, matfile.MatFileError) as e:
            raise SystemExit("cannot load dipole polarisations from %s: %s" % (d, e))

    prof.begin("Dmatrix")  # context: D matrix on the GPU, FFT plans, autotuning
    mv = api.CudaMatVec(params, prec, max_rhs=2, device=device)
    ccs = []
    for r, pol in enumerate((1, 2)):
        ccs.append(api.CoupleConstants(params, prop, pol, a.pol, orient=orient))
        mv.set_couple_constants(ccs[-1], rhs=r)
    if a.verbose:  # DDAParams::dump (DDAMain.cpp:272-273)
        out.write("wavelength = %.10g m, k d = %.10g, beam = %s, prop = %s, orient = %s\n"
                  % (lambda_m, params.kd, a.beam, prop, orient))
        for r in range(2):
            out.write("Pol%d couple constants sqrt(cc) = %s\n" % (r + 1, np.asarray(ccs[r].cc_sqrt).tolist()))
    # <out>/meminfo, and with --mem-info also stderr (DDAMain.cpp:577-601); this
    # library allocates per context, so the context's device bytes are listed
    lay = mv.layout
    mem = ("Alloc 'context' (D matrix, plane buffers, Krylov vectors; y/z path %s) = %d kB, sum = %d kB\n"
           % (lay["yz_path"], (lay["device_bytes"] + 1023) // 1024, (lay["device_bytes"] + 1023) // 1024))
    with open(os.path.join(a.output_dir, "meminfo"), "w") as f:
        f.write(mem)
    if a.mem_info:
        sys.stderr.write(mem)
    if a.profiling_run:  # IterativeSolverBase::profilingRun, DDA/IterativeSolverBase.cpp:105-136
        ms = mv.profile(nrhs=2, reps=5)
        out.write("matvec (2 rhs): %.3f ms  [x forward %.3f, y/z %.3f, x inverse %.3f]\n"
                  % (ms[3], ms[0], ms[1], ms[2]))
        mv.close()
        return 0
    prof.begin("res12")  # incident fields and the solve of both polarisations
    beam = api.Beam(a.beam)
    einc = np.stack([beam.einc(params, prop, 1, orient=orient), beam.einc(params, prop, 2, orient=orient)])
    if a.store_incbeam:
        for r in range(2):
            store_field("IncBeam-Pol%d" % (r + 1), "IncidentBeam", r, einc[r])
    if a.load_dip_pol:  # DDA/DDAMain.cpp:374-378
        pol = load_pol(a.load_dip_pol)
        out.write("Loaded dipole polarisations from %s\n" % a.load_dip_pol)
    else:
        start = None
        if a.load_start_dip_pol:  # DDA/DDAMain.cpp:391-394
            start = load_pol(a.load_start_dip_pol)
        solver = api.CudaSolver(mv, a.iter, max_iter=a.maxiter)
        pol = solver.get_pol_vec(einc, 10.0 ** -a.epsilon, start=start)
        for r, (st, hist) in enumerate(zip(solver.last_stats, solver.last_history)):
            out.write("Pol%d: %d iterations, relative residual %.3e\n" % (r + 1, st.iterations, st.rel_residual))
            out.write(residual_lines(hist))
    prof.begin("output dippol")
    for r in range(2):
        store_field("DipPol-Pol%d" % (r + 1), "DipolePolarization", r, pol[r])  # always, DDAMain.cpp:412
    if a.store_intfield:  # internal field chi^-1 P, DDA/DDAMain.cpp:420-425
        prof.begin("output intfield")
        for r in range(2):
            store_field("IntField-Pol%d" % (r + 1), "InternalField", r, cc_vector(params, ccs[r].chi_inv) * pol[r])
    prof.begin("output")

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
        # createCrossSectionFile(...)->write (output, ".txt"), DDAMain.cpp:302
        datafiles.write(odir("CrossSec-" + label), datafiles.cross_section_file(r + 1, cext, cabs, qext, qabs),
                        lambda p: datafiles.cross_section_txt(p, cext, cabs, qext, qabs))
    if mie_geom is not None and beam.plane:  # DDA/DDAMain.cpp:431
        radius = mie_geom[1]
        x = 2 * math.pi * radius / lambda_m
        qe, qs, qa = postprocess.mie(x, refr[0])
        out.write("Mie solution:\nQext = %.10g Qabs = %.10g Qsca = %.10g\n" % (qe, qa, qs))
        area = math.pi * radius ** 2  # CrossSection::setCFromQ, DDAMain.cpp:454-456
        datafiles.write(odir("MieCrossSec"), datafiles.cross_section_file(0, qe * area, qa * area, qe, qa),
                        lambda p: datafiles.cross_section_txt(p, qe * area, qa * area, qe, qa))
    # far fields (DDA/DDAMain.cpp:318-353): the angle lists of all options,
    # each list computed once for both polarisations
    prof.begin("farfield")
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
    far_geometry = datafiles.dipole_list_geometry(params, orient, full=False)  # FarFieldCalc.cpp:173
    freq = datafiles.SPEED_OF_LIGHT / lambda_m
    mie_far = mie_geom is not None and beam.plane  # the Mie far field beside it, DDAMain.cpp:476-489
    if mie_far:
        mie_pars = datafiles.mie_parameters(lambda_m, a.geometry, prop, a.beam,
                                            [api.beam_pol(prop, 1)[0], api.beam_pol(prop, 2)[0]], " ".join(argv))
        mie_g = datafiles.mie_geometry(mie_geom[1], refr[0])
        mie_x = 2 * math.pi * mie_geom[1] / lambda_m
    for name, ts, ps, want_j, want_m, no_phi in far:
        if (ts, ps) not in cache:
            theta, phi = postprocess.grid_angles(ts, ps)
            cache[(ts, ps)] = (theta, phi, postprocess.jones_far_field(mv, prop, theta, phi, pol=pol,
                                                                       orient=orient))
        theta, phi, jones = cache[(ts, ps)]
        # FarFieldCalc<ftype>::store, DDA/FarFieldCalc.hpp:82-97
        if want_j:
            datafiles.write(odir("Far" + name), datafiles.jones_file(pars, far_geometry, theta, phi, freq, jones, ftype),
                            (lambda p: postprocess.store_jones_txt(p, theta, phi, jones, store_phi=not no_phi))
                            if txt else None)
        if want_m:
            m = postprocess.mueller(jones)
            datafiles.write(odir("Far%s.mueller" % name),
                            datafiles.mueller_file(pars, far_geometry, theta, phi, freq, m, ftype),
                            (lambda p: postprocess.store_mueller_txt(p, theta, phi, m, no_phi=no_phi))
                            if txt else None)
        if mie_far:  # FarFieldCalc<ldouble>::store (outputDir / "MieFar", ...): double precision files
            mj = postprocess.mie_jones(mie_x, refr[0], theta, params.wave_num)
            if want_j:
                datafiles.write(odir("MieFar" + name), datafiles.jones_file(mie_pars, mie_g, theta, phi, freq, mj),
                                (lambda p: postprocess.store_jones_txt(p, theta, phi, mj, store_phi=not no_phi))
                                if txt else None)
            if want_m:
                mm = postprocess.mueller(mj)
                datafiles.write(odir("MieFar%s.mueller" % name),
                                datafiles.mueller_file(mie_pars, mie_g, theta, phi, freq, mm),
                                (lambda p: postprocess.store_mueller_txt(p, theta, phi, mm, no_phi=no_phi))
                                if txt else None)
    mv.close()
    prof.end()
    return 0


if __name__ == "__main__":
    sys.exit(main())
