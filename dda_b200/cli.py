"""Command line in the shape of the reference's `dda` (DDA/Options.cpp:41-97,
DDA/DDAMain.cpp:611-771): one target, both polarisations, cross sections and,
on request, the far-field grid.

    python -m dda_b200.cli --geometry 'sphere:10um,1.5+0.1i' --lambda 6um --grid-unit 0.5um \\
        --iter qmr --epsilon 5 --efield-grid --output-dir out

Supported options: --lambda, --prop, --pol (ldr, cm, ldr-avgpol), --geometry
(sphere:R,m | cylinder:L,R,m | box:(X,Y,Z),m | load:file=<text dipole list> with -m),
--grid-unit (default: the reference's rule, lambda / (10 max|m|) and at most a
16th of every particle dimension, DDAMain.cpp:134-150), -m, --fft-grid, --epsilon
(stop at 10^-epsilon), --maxiter, --iter, --ftype (float, double; plus mixed),
--efield-grid, --no-symmetry (both polarisations are always solved), --output-dir.
Output files are text: CrossSec-Pol1.txt, CrossSec-Pol2.txt, MieCrossSec.txt
(spheres), EFieldGrid.txt (--efield-grid: theta, phi and the Jones matrix
S11, S12, S21, S22 per direction), DipPol-Pol<n>.txt (--store-dippol).  The
reference's MATLAB-style HDF5 files are not written (no HDF5 library here).
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


def main(argv=None):
    ap = argparse.ArgumentParser(prog="dda_b200.cli", description=__doc__.split("\n\n")[0])
    ap.add_argument("--lambda", dest="lam", default="%.17gum" % (2 * math.pi))
    ap.add_argument("--prop", default="(0,0,1)")
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
    ap.add_argument("--efield-grid", action="store_true")
    ap.add_argument("--store-dippol", action="store_true")
    ap.add_argument("--output-dir", default=".")
    a = ap.parse_args(argv)

    lambda_m = api.parse_length(a.lam)
    prop = tuple(parse_vector(a.prop))
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
        ccs.append(api.CoupleConstants(params, prop, pol, a.pol))
        mv.set_couple_constants(ccs[-1], rhs=r)
    einc = np.stack([params.einc(prop, 1), params.einc(prop, 2)])
    solver = api.CudaSolver(mv, a.iter, max_iter=a.maxiter)
    pol = solver.get_pol_vec(einc, 10.0 ** -a.epsilon)
    for r, (st, hist) in enumerate(zip(solver.last_stats, solver.last_history)):
        out.write("Pol%d: %d iterations, relative residual %.3e\n" % (r + 1, st.iterations, st.rel_residual))
        for i, h in enumerate(hist):
            out.write("RE_%d = %.10g\n" % (i + 1, h))

    _, pn = api.beam_pol(prop, 1)
    ef = mv.far_field(pn[None, :], nrhs=2)[0]
    for r in range(2):
        cext, cabs, qext, qabs = postprocess.cross_sections(params, ccs[r], pol[r], ef[r], prop, r + 1)
        csca, qsca = cext - cabs, qext - qabs
        label = "Pol%d" % (r + 1)
        out.write("Cext %s = %-25s Qext %s = %.10g\n" % (label, "%.10g um^2" % (cext * 1e12), label, qext))
        out.write("Cabs %s = %-25s Qabs %s = %.10g\n" % (label, "%.10g um^2" % (cabs * 1e12), label, qabs))
        out.write("Csca %s = %-25s Qsca %s = %.10g\n" % (label, "%.10g um^2" % (csca * 1e12), label, qsca))
        with open(os.path.join(a.output_dir, "CrossSec-%s.txt" % label), "w") as f:
            f.write("BeamPolarization = %d\nCext = %.17g\nQext = %.17g\nCabs = %.17g\nQabs = %.17g\n"
                    "Csca = %.17g\nQsca = %.17g\n" % (r + 1, cext, qext, cabs, qabs, csca, qsca))
        if a.store_dippol:
            np.savetxt(os.path.join(a.output_dir, "DipPol-%s.txt" % label),
                       np.column_stack([pol[r].real, pol[r].imag]), header="re im, [x: nvs][y: nvs][z: nvs]")
    if mie_geom is not None:
        radius = mie_geom[1]
        x = 2 * math.pi * radius / lambda_m
        qe, qs, qa = postprocess.mie(x, refr[0])
        out.write("Mie solution:\nQext = %.10g Qabs = %.10g Qsca = %.10g\n" % (qe, qa, qs))
        with open(os.path.join(a.output_dir, "MieCrossSec.txt"), "w") as f:
            f.write("Qext = %.17g\nQabs = %.17g\nQsca = %.17g\n" % (qe, qa, qs))
    if a.efield_grid:
        theta, phi = postprocess.grid_angles("0..180/91", "0..360/61")  # DDA/DDAMain.cpp:346-347
        jones = postprocess.jones_far_field(mv, prop, theta, phi)
        with open(os.path.join(a.output_dir, "EFieldGrid.txt"), "w") as f:
            f.write("# theta_deg phi_deg  re/im of S11 S12 S21 S22\n")
            for t, p_, j in zip(theta, phi, jones):
                vals = " ".join("%.10e %.10e" % (z.real, z.imag) for z in j.reshape(-1))
                f.write("%.6f %.6f %s\n" % (math.degrees(t), math.degrees(p_), vals))
    mv.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
