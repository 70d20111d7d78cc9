"""The reference's Hdf5Util (EMSim/Hdf5Util.cpp, EMSim/Hdf5ToText.cpp,
EMSim/ResaveHdf5.cpp) on this project's HDF5 reader and writer:

    python -m dda_b200.hdf5util [options] <command> <input-file.hdf5> [...]

commands:
  hdf5-to-text   write each input's text layout to <input>.txt (or --output)
  cat            print each input's text layout
  resave-hdf5    write each input again, to <input>.new.hdf5 (or --output)
  jones-to-mueller
                 the Mueller matrices of each Jones far-field input, to
                 <input>.mueller.hdf5 (or --output)

options: --output/-o FILE (one input only), --theta-max-180 (keep far-field
entries with theta <= 180 degrees), --no-phi (far-field text without the phi
column), --type TYPE (instead of the file's Type), --verbose.

The text layouts by Type (EMSim/Hdf5ToText.cpp:61-93): JonesFarField
(JonesCalculus::storeTxt), MuellerFarField (MuellerCalculus::storeTxt),
DDAField (DDAFieldFile::writeTxt), Geometry (DDADipoleListGeometryFile::writeTxt),
CrossSection (CrossSectionFile::writeTxt).
"""
import argparse
import math
import os
import sys

import numpy as np

from . import datafiles, matfile, postprocess


def _far_field(f, key, theta_max_180):
    """(theta, phi, matrices [n][i][j]) of a far-field file; the stored
    Data is the Fortran [d][d][n][1] array with its dimensions reversed."""
    ff = f[key]
    theta = np.asarray(ff["Theta"], dtype=np.float64).reshape(-1)
    phi = np.asarray(ff["Phi"], dtype=np.float64).reshape(-1)
    data = np.asarray(ff["Data"])
    mats = data.reshape(-1, len(theta), data.shape[-2], data.shape[-1])[0].transpose(0, 2, 1)
    if theta_max_180:  # removeThetaLarger180 (EMSim/ResaveHdf5.cpp:30-92)
        keep = theta * 180 / math.pi <= 180.0001
        theta, phi, mats = theta[keep], phi[keep], mats[keep]
    return theta, phi, mats


def to_text(path, out, type_override=None, theta_max_180=False, no_phi=False):
    """hdf5ToText (EMSim/Hdf5ToText.cpp:61-93); `out` is a path or a text stream."""
    f = matfile.load(path)
    kind = type_override or f.get("Type")
    if kind == "JonesFarField":
        theta, phi, j = _far_field(f, "JonesFarField", theta_max_180)
        postprocess.store_jones_txt(out, theta, phi, j, store_phi=not no_phi)
    elif kind == "MuellerFarField":
        theta, phi, m = _far_field(f, "MuellerFarField", theta_max_180)
        postprocess.store_mueller_txt(out, theta, phi, m, no_phi=no_phi)
    elif kind == "DDAField":
        g, fld = f["Geometry"], f["Field"]
        if g.get("DipolePositions") is None:
            raise ValueError("`%s': no DipolePositions in the Geometry object" % path)
        pos = np.asarray(g["DipolePositions"], dtype=np.float64).reshape(-1, 3)
        coords = (np.asarray(g["GridOrigin"], dtype=np.float64).reshape(-1)
                  + np.asarray(g["GridSpacing"], dtype=np.float64).reshape(-1) * pos)
        rows = np.asarray(fld["Data"]).reshape(-1, 3)
        datafiles.field_txt_rows(out, coords, rows, fld["FieldName"], int(np.asarray(fld["BeamPolarization"])[0]))
    elif kind == "Geometry":
        g = f["Geometry"]
        datafiles.geometry_txt_rows(out, np.asarray(g["Size"]).reshape(-1),
                                    np.asarray(g["DipolePositions"]).reshape(-1, 3),
                                    np.asarray(g["DipoleMaterialIndices"]).reshape(-1))
    elif kind == "CrossSection":
        cs = {k: float(np.asarray(v).reshape(-1)[0]) for k, v in f["CrossSection"].items()}
        datafiles.cross_section_txt(out, cs["Cext"], cs["Cabs"], cs["Qext"], cs["Qabs"], cs["Csca"], cs["Qsca"])
    else:
        raise ValueError("Unknown file type '%s'" % kind)


def resave(path, out, type_override=None, theta_max_180=False):
    """resaveHdf5 (EMSim/ResaveHdf5.cpp): the file read and written again,
    far fields optionally cut to theta <= 180 degrees."""
    f = matfile.load(path)
    kind = type_override or f.get("Type")
    if theta_max_180 and kind in ("JonesFarField", "MuellerFarField"):
        theta, phi, mats = _far_field(f, kind, True)
        ff = dict(f[kind])
        ff["Theta"], ff["Phi"] = theta, phi
        ff["Data"] = np.ascontiguousarray(mats.transpose(0, 2, 1)[None].astype(np.asarray(f[kind]["Data"]).dtype))
        f[kind] = ff
    matfile.save(out, f)


def jones_to_mueller(path, out, theta_max_180=False):
    """jonesToMueller (EMSim/JonesToMueller.cpp:32-48): a MuellerFarField file
    from a JonesFarField file, its Parameters and Geometry carried over."""
    f = matfile.load(path)
    theta, phi, j = _far_field(f, "JonesFarField", theta_max_180)
    freq = np.asarray(f["JonesFarField"]["Frequency"], dtype=np.float64).reshape(-1)
    m = postprocess.mueller(j)
    members = {"Type": "MuellerFarField", "Parameters": f.get("Parameters"), "Geometry": f.get("Geometry"),
               "MuellerFarField": {"Theta": theta, "Phi": phi, "Frequency": freq,
                                   "Data": np.ascontiguousarray(m.transpose(0, 2, 1)[None])}}
    matfile.save(out, members)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="dda_b200.hdf5util", description=__doc__.split("\n\n")[0])
    ap.add_argument("command", choices=["hdf5-to-text", "cat", "resave-hdf5", "jones-to-mueller"])
    ap.add_argument("inputs", nargs="+")
    ap.add_argument("-o", "--output")
    ap.add_argument("--theta-max-180", action="store_true")
    ap.add_argument("--no-phi", action="store_true")
    ap.add_argument("--type")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    if len(a.inputs) > 1 and a.output:
        sys.stderr.write("Error: Got multiple input files and a --output option\n")
        return 1
    try:
        for inp in a.inputs:
            if a.command == "cat":
                if a.verbose:
                    sys.stderr.write("Showing '%s':\n" % inp)
                to_text(inp, sys.stdout, a.type, a.theta_max_180, a.no_phi)
                continue
            ext = {"hdf5-to-text": ".txt", "resave-hdf5": ".new.hdf5", "jones-to-mueller": ".mueller.hdf5"}[a.command]
            out = a.output or os.path.splitext(inp)[0] + ext
            if a.verbose:
                sys.stderr.write("Converting '%s' to '%s' ..." % (inp, out))
            if a.command == "hdf5-to-text":
                to_text(inp, out, a.type, a.theta_max_180, a.no_phi)
            elif a.command == "jones-to-mueller":
                jones_to_mueller(inp, out, a.theta_max_180)
            else:
                resave(inp, out, a.type, a.theta_max_180)
            if a.verbose:
                sys.stderr.write(" done\n")
    except (OSError, ValueError, KeyError, matfile.MatFileError) as e:
        sys.stderr.write("Error: %s\n" % e)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
