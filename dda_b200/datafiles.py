"""The reference's data files: what its command line stores and loads.

Structures (EMSim/DataFiles.hpp:68-220, EMSim/DataFilesDDA.hpp:48-187) and
how they are filled (DDA/DataFilesDDAUtil.cpp:31-120):

* Parameters: Method "DDA", MethodParameters {PolarizabilityType, Gamma,
  Frequency}, GeometryString, CmdLine, RefractiveIndexMedium,
  PropagationVector, BeamString, Polarizations;
* DDADipoleListGeometry: Type "DDADipoleList", GridSpacing, Size, GridOrigin,
  Orientation (quaternion a, b, c, d), RefractiveIndices, DipolePositions and
  DipoleMaterialIndices (left out of the far-field files), Periodicity;
* DDAFieldFile: Type "DDAField", Parameters, Geometry, Field {FieldName,
  BeamPolarization, Data [nv][3] complex} -- DipPol-Pol<n>, IntField-Pol<n>,
  IncBeam-Pol<n>;
* DDADipoleListGeometryFile: Type "Geometry", Geometry -- Geometry.hdf5;
* CrossSectionFile: Type "CrossSection", BeamPolarization, CrossSection {Cext,
  Cabs, Csca, Qext, Qabs, Qsca} -- CrossSec-Pol<n>, MieCrossSec;
* JonesFarFieldFile / MuellerFarFieldFile: Type, Parameters, Geometry,
  JonesFarField / MuellerFarField {Theta, Phi, Frequency, Data} -- the
  matrices of Fortran-ordered [2][2][n][1] / [4][4][n][1] arrays, stored with
  the dimensions reversed.

Each is written as a MATLAB-style HDF5 file (`matfile`) and, where the
reference has one, in its text layout.  Vectors on the Python side are this
library's [3 nvs] complex layout (component c of dipole i at c nvs + i).
"""
import math
import os

import numpy as np

from . import matfile

SPEED_OF_LIGHT = 299792458.0


# --------------------------------------------------------------------------
# orientation

def orientation_quaternion(orient):
    """(a, b, c, d) of the rotation Rz(alpha) Ry(beta) Rz(gamma), the ZYZ Euler
    angles in degrees (EMSim::Rotation::fromZYZDeg, EMSim/Rotation.hpp:85-102);
    the identity for None."""
    if orient is None:
        return np.array([1.0, 0.0, 0.0, 0.0])
    al, be, ga = (math.radians(float(x)) for x in orient)

    def mul(p, q):
        a1, b1, c1, d1 = p
        a2, b2, c2, d2 = q
        return (a1 * a2 - b1 * b2 - c1 * c2 - d1 * d2, a1 * b2 + b1 * a2 + c1 * d2 - d1 * c2,
                a1 * c2 - b1 * d2 + c1 * a2 + d1 * b2, a1 * d2 + b1 * c2 - c1 * b2 + d1 * a2)

    qz = lambda t: (math.cos(t / 2), 0.0, 0.0, math.sin(t / 2))
    qy = (math.cos(be / 2), 0.0, math.sin(be / 2), 0.0)
    return np.array(mul(mul(qz(al), qy), qz(ga)))


def zyz_from_quaternion(q):
    """ZYZ Euler angles in degrees of the rotation of the unit quaternion
    (a, b, c, d), from its rotation matrix R = Rz(alpha) Ry(beta) Rz(gamma):
    R22 = cos beta, (R02, R12) = sin beta (cos alpha, sin alpha), (R20, R21) =
    sin beta (-cos gamma, sin gamma); with sin beta = 0 only alpha +- gamma is
    defined and gamma is taken as 0."""
    a, b, c, d = (float(x) for x in q)
    n = math.sqrt(a * a + b * b + c * c + d * d)
    a, b, c, d = a / n, b / n, c / n, d / n
    r00, r01 = 1 - 2 * (c * c + d * d), 2 * (b * c - a * d)
    r02, r10 = 2 * (b * d + a * c), 2 * (b * c + a * d)
    r11, r12 = 1 - 2 * (b * b + d * d), 2 * (c * d - a * b)
    r20, r21, r22 = 2 * (b * d - a * c), 2 * (c * d + a * b), 1 - 2 * (b * b + c * c)
    sb = math.hypot(r02, r12)
    if sb > 1e-9:
        al, be, ga = math.atan2(r12, r02), math.atan2(sb, r22), math.atan2(r21, -r20)
    elif r22 > 0:
        al, be, ga = math.atan2(r10, r00), 0.0, 0.0
    else:
        al, be, ga = math.atan2(-r01, r11), math.pi, 0.0
    return tuple(math.degrees(x) for x in (al, be, ga))


# --------------------------------------------------------------------------
# structures

def _vec_rows(params, vec):
    """[nv][3] rows of a [3 nvs] vector."""
    v = np.asarray(vec).reshape(3, params.nvs)[:, :params.nv]
    return np.ascontiguousarray(v.T)


def _cdtype(ftype):
    return np.complex64 if ftype == "float" else np.complex128


def grid_origin(params):
    """The position of grid cell (0, 0, 0): the dipole box centred on the
    origin (DipoleGeometry::moveToCenter, DDA/DipoleGeometry.cpp:75-80)."""
    return -(np.asarray(params.box, dtype=np.float64) - 1.0) / 2 * params.grid_unit


def dipole_coords(params):
    """Dipole coordinates [nv][3] in metres (origin + spacing * position)."""
    return grid_origin(params) + params.grid_unit * params.geometry.positions.astype(np.float64)


def parameters(params, geometry_string="", gamma=0.001):
    """Parameters<DDAParameters> (DDA/DataFilesDDAUtil.cpp:31-50)."""
    return {"Method": "DDA",
            "MethodParameters": {"PolarizabilityType": "", "Gamma": np.array([gamma]),
                                 "Frequency": np.array([SPEED_OF_LIGHT / params.wavelength])},
            "GeometryString": geometry_string, "CmdLine": "",
            "RefractiveIndexMedium": np.ones(3), "PropagationVector": np.zeros(3), "BeamString": "",
            "Polarizations": np.zeros((0, 3))}


def dipole_list_geometry(params, orient=None, full=True):
    """DDADipoleListGeometry (DDA/DataFilesDDAUtil.cpp:53-86); `full` adds the
    dipole positions and material indices."""
    refr = np.array([m if isinstance(m, (list, tuple)) else (m, m, m) for m in params.materials],
                    dtype=np.complex128).reshape(-1, 3)
    g = {"Type": "DDADipoleList", "GridSpacing": np.full(3, params.grid_unit),
         "Size": np.asarray(params.box, dtype=np.uint32), "GridOrigin": grid_origin(params),
         "Orientation": orientation_quaternion(orient), "RefractiveIndices": refr,
         "DipolePositions": None, "DipoleMaterialIndices": None, "Periodicity": np.zeros((0, 3))}
    if full:
        g["DipolePositions"] = np.ascontiguousarray(params.geometry.positions, dtype=np.uint32)
        g["DipoleMaterialIndices"] = np.ascontiguousarray(params.geometry.materials, dtype=np.uint8)
    return g


def field_file(params, pars, geometry, field_name, pol, vec, ftype="double"):
    """DDAFieldFile (DDA/DataFilesDDAUtil.cpp:96-120)."""
    return {"Type": "DDAField", "Parameters": pars, "Geometry": geometry,
            "Field": {"FieldName": field_name, "BeamPolarization": np.array([pol], dtype=np.uint32),
                      "Data": _vec_rows(params, vec).astype(_cdtype(ftype))}}


def cross_section_file(pol, cext, cabs, qext, qabs):
    """CrossSectionFile (EMSim/DataFiles.hpp:196-220); Csca = Cext - Cabs."""
    cs = {"Cext": cext, "Cabs": cabs, "Csca": cext - cabs, "Qext": qext, "Qabs": qabs, "Qsca": qext - qabs}
    return {"Type": "CrossSection", "BeamPolarization": np.array([pol], dtype=np.uint32),
            "CrossSection": {k: np.array([float(v)]) for k, v in cs.items()}}


def jones_file(pars, geometry, theta, phi, frequency, jones, ftype="double"):
    """JonesFarFieldFile (EMSim/JonesCalculus.hpp:84-92, JonesCalculus.cpp:50-72):
    jones [n][2][2] (element [i][j] of the reference's JonesMatrix) stored as
    the Fortran [2][2][n][1] array, i.e. HDF5 dims [1][n][2][2] with [0][p][j][i]."""
    data = np.asarray(jones).transpose(0, 2, 1)[None].astype(_cdtype(ftype))
    return {"Type": "JonesFarField", "Parameters": pars, "Geometry": geometry,
            "JonesFarField": {"Theta": np.asarray(theta, dtype=np.float64), "Phi": np.asarray(phi, dtype=np.float64),
                              "Frequency": np.array([frequency]), "Data": np.ascontiguousarray(data)}}


def mueller_file(pars, geometry, theta, phi, frequency, mueller, ftype="double"):
    """MuellerFarFieldFile (EMSim/MuellerCalculus.hpp:83-92, MuellerCalculus.cpp:63-85)."""
    data = np.asarray(mueller).transpose(0, 2, 1)[None].astype(np.float32 if ftype == "float" else np.float64)
    return {"Type": "MuellerFarField", "Parameters": pars, "Geometry": geometry,
            "MuellerFarField": {"Theta": np.asarray(theta, dtype=np.float64),
                                "Phi": np.asarray(phi, dtype=np.float64), "Frequency": np.array([frequency]),
                                "Data": np.ascontiguousarray(data)}}


def mie_parameters(wavelength, geometry_string, prop, beam_string, pols, cmd_line=""):
    """Parameters<MieParameters> of the Mie far-field files
    (createParametersMie, EMSim/DataFilesUtil.cpp:29-47; DDAMain.cpp:438-443)."""
    return {"Method": "Mie", "MethodParameters": {"Frequency": np.array([SPEED_OF_LIGHT / wavelength])},
            "GeometryString": geometry_string, "CmdLine": cmd_line, "RefractiveIndexMedium": np.ones(3),
            "PropagationVector": np.asarray(prop, dtype=np.float64), "BeamString": beam_string,
            "Polarizations": np.asarray(pols, dtype=np.float64).reshape(-1, 3)}


def mie_geometry(radius, m):
    """MieGeometry (EMSim/DataFiles.hpp:144-157)."""
    return {"Type": "Mie", "Radius": np.array([float(radius)]), "RefractiveIndex": np.full(3, complex(m))}


def geometry_file(params, orient=None):
    """DDADipoleListGeometryFile (DDA/DataFilesDDAUtil.cpp:88-93)."""
    return {"Type": "Geometry", "Geometry": dipole_list_geometry(params, orient, True)}


# --------------------------------------------------------------------------
# text layouts

def _g10(x):
    """A number as an ostream of precision 10 prints it."""
    return "%.10g" % x


def field_txt(path, params, field_name, pol, vec, ftype="double"):
    """DDAFieldFile::writeTxt (EMSim/DataFilesDDA.cpp:34-54) of a [3 nvs]
    vector of this target."""
    field_txt_rows(path, dipole_coords(params), _vec_rows(params, vec).astype(_cdtype(ftype)), field_name, pol)


def field_txt_rows(out, coords, rows, field_name, pol):
    """The text layout of a field: coordinates in metres, |E|^2, then re, im of
    the x, y, z components, one dipole ([nv][3] rows) per line; `out` is a
    path or a text stream."""
    name = field_name + ("-Pol%d" % pol if pol else "")
    norm = (np.abs(rows) ** 2).sum(axis=1, dtype=rows.real.dtype)
    with open_out(out) as f:
        f.write("#x y z |%s|^2 " % name + " ".join("%s.%s.%s" % (name, c, p) for c in "xyz" for p in "ri") + "\n")
        for xyz, n2, r in zip(coords, norm, rows):
            f.write(" ".join(_g10(x) for x in xyz) + " " + _g10(n2) + " "
                    + " ".join(_g10(z) for v in r for z in (v.real, v.imag)) + "\n")


class open_out:
    """A path opened for writing, or a text stream used as it is."""

    def __init__(self, out):
        self.out, self.f = out, None

    def __enter__(self):
        if isinstance(self.out, str):
            self.f = open(self.out, "w")
            return self.f
        return self.out

    def __exit__(self, *exc):
        if self.f is not None:
            self.f.close()


def read_field_txt(path, params):
    """Load::loadFields (DDA/Load.cpp:71-104): one line per dipole, the
    coordinates checked against this target's (to a thousandth of the grid
    unit), |E|^2 against the components (1e-5, as there)."""
    d = np.loadtxt(path, ndmin=2, comments="#")
    if d.shape != (params.nv, 10):
        raise ValueError("`%s' does not hold %d dipoles of 10 columns" % (path, params.nv))
    if np.max(np.abs(d[:, :3] - dipole_coords(params))) > 1e-3 * params.grid_unit:
        raise ValueError("`%s' does not hold this target's dipoles" % path)
    rows = d[:, 4:10:2] + 1j * d[:, 5:10:2]
    if np.max(np.abs(d[:, 3] - (np.abs(rows) ** 2).sum(axis=1))) >= 1e-5:
        raise ValueError("`%s': |E|^2 column does not match the components" % path)
    return _from_rows(params, rows)


def _from_rows(params, rows):
    v = np.zeros(params.vec_size, dtype=np.complex128)
    for c in range(3):
        v[c * params.nvs:c * params.nvs + params.nv] = rows[:, c]
    return v


def cross_section_txt(out, cext, cabs, qext, qabs, csca=None, qsca=None):
    """CrossSectionFile::writeTxt (EMSim/DataFiles.cpp:32-42); Csca and Qsca
    default to the differences (CrossSection::setSca)."""
    csca = cext - cabs if csca is None else csca
    qsca = qext - qabs if qsca is None else qsca
    with open_out(out) as f:
        for k, v in (("Cext", cext), ("Qext", qext), ("Cabs", cabs), ("Qabs", qabs), ("Csca", csca), ("Qsca", qsca)):
            f.write("%s = %s\n" % (k, _g10(v)))


def geometry_txt(path, params):
    """DDADipoleListGeometryFile::writeTxt of this target."""
    geometry_txt_rows(path, params.box, params.geometry.positions, params.geometry.materials)


def geometry_txt_rows(out, box, pos, mat):
    """DDADipoleListGeometryFile::writeTxt (EMSim/DataFilesDDA.cpp:58-82): the
    box size, Nmat when there is more than one material, one dipole per line
    (with its 1-based material index when there are several)."""
    mat = np.asarray(mat).astype(np.int64)
    nmat = int(mat.max()) + 1 if len(mat) else 0
    with open_out(out) as f:
        f.write("#box size: %dx%dx%d\n" % tuple(int(b) for b in box))
        if nmat != 1:
            f.write("Nmat=%d\n" % nmat)
        for p, m in zip(pos, mat):
            f.write("%d %d %d" % tuple(p) + (" %d" % (m + 1) if nmat != 1 else "") + "\n")


# --------------------------------------------------------------------------
# loading

def load_dip_pol(basename, params):
    """Load<ftype>::loadDipPol (DDA/Load.cpp:110-135): <basename>.hdf5, or
    <basename>.txt when only that exists; the stored dipole positions must be
    this target's."""
    h5, txt = basename + ".hdf5", basename + ".txt"
    if not os.path.exists(h5) and os.path.exists(txt):
        return read_field_txt(txt, params)
    f = matfile.load(h5)
    rows = np.asarray(f["Field"]["Data"]).reshape(-1, 3)
    if rows.shape[0] != params.nv:
        raise ValueError("`%s' holds %d dipoles, the target %d" % (h5, rows.shape[0], params.nv))
    pos = f.get("Geometry", {}).get("DipolePositions")
    if pos is not None and not np.array_equal(np.asarray(pos).reshape(-1, 3), params.geometry.positions):
        raise ValueError("`%s' does not hold this target's dipoles" % h5)
    return _from_rows(params, rows.astype(np.complex128))


def load_geometry(path):
    """A dipole-list geometry file (DDAMain.cpp:163-235): a dict with
    positions [n][3] uint32 (normalised so that each coordinate's minimum is
    0, DipoleGeometry::normalize, DDA/DipoleGeometry.cpp:109-132; `shift` is
    what was subtracted), materials [n] uint8 and, where the file holds them,
    grid_unit, origin (GridOrigin as stored, before the shift), orientation
    (ZYZ degrees) and refractive_indices (a list of 3-tuples).  A directory
    stands for its Geometry.hdf5."""
    if os.path.isdir(path):
        path = os.path.join(path, "Geometry.hdf5")
    g = matfile.load(path).get("Geometry")
    if g is None:
        raise ValueError("No Geometry object in geometry file")
    if g.get("DipolePositions") is None:
        raise ValueError("No DipolePositions object in Geometry object in geometry file")
    if g.get("DipoleMaterialIndices") is None:
        raise ValueError("No DipoleMaterialIndices object in Geometry object in geometry file")
    pos = np.asarray(g["DipolePositions"]).reshape(-1, 3).astype(np.uint32)
    mat = np.asarray(g["DipoleMaterialIndices"]).reshape(-1).astype(np.uint8)
    if len(mat) != len(pos):
        raise ValueError("DipolePositions and DipoleMaterialIndices differ in length")
    per = g.get("Periodicity")
    if per is not None and np.asarray(per).size:
        raise ValueError("periodic targets are not supported")
    if len(pos) and np.any(np.diff(pos[:, 2].astype(np.int64)) < 0):
        raise ValueError("the dipoles must be ordered by z")
    lo = pos.min(axis=0) if len(pos) else np.zeros(3, dtype=np.uint32)
    out = {"positions": pos - lo, "materials": mat, "shift": lo.astype(np.float64)}
    if g.get("GridSpacing") is not None:
        s = np.asarray(g["GridSpacing"], dtype=np.float64).reshape(-1)
        if not (s[0] == s[1] == s[2]) or not s[0] > 0:
            raise ValueError("GridSpacing must be one positive value for all axes")
        out["grid_unit"] = float(s[0])
    if g.get("GridOrigin") is not None:
        out["origin"] = np.asarray(g["GridOrigin"], dtype=np.float64).reshape(-1)
    if g.get("Orientation") is not None:
        out["orientation"] = zyz_from_quaternion(np.asarray(g["Orientation"]).reshape(-1))
    if g.get("RefractiveIndices") is not None:
        r = np.asarray(g["RefractiveIndices"]).astype(np.complex128).reshape(-1, 3)
        out["refractive_indices"] = [tuple(complex(z) for z in row) for row in r]
    return out


def write(basename, members, txt_writer=None):
    """<basename>.hdf5 and, given a text writer, <basename>.txt
    (the write() of the file structures, e.g. EMSim/DataFilesDDA.cpp:57-63)."""
    matfile.save(basename + ".hdf5", members)
    if txt_writer is not None:
        txt_writer(basename + ".txt")
