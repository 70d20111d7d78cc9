"""ctypes front end of the CPU oracle (oracle/dda_oracle.cpp).

TEST INFRASTRUCTURE ONLY: this module is the checker for the CUDA path.  Only
tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline / reference
arm import it.  Parity against outputs of the reference itself is UNPINNED
(the reference cannot be built here); see the header of dda_oracle.cpp for
the independent checks that pin the restatement instead.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libdda_oracle.so")
_lib = None

SOLVERS = {"qmr": 0, "bicgstab": 1, "bicg": 2, "cgnr": 3}
POLARIZABILITIES = {"cm": 0, "ldr": 1, "ldr-avgpol": 2}


class OrcStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("matvecs", ctypes.c_int64),
                ("residScale", ctypes.c_double), ("inprodR", ctypes.c_double),
                ("relResidual", ctypes.c_double), ("status", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


def build():
    """Compiles the oracle library with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, u32p, u8p, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), \
            ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_double)
        ld = ctypes.c_longdouble
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_parse_number.argtypes = [ctypes.c_char_p, ctypes.POINTER(ld)]
        L.orc_parse_length.argtypes = [ctypes.c_char_p, ctypes.POINTER(ld)]
        L.orc_fft.argtypes = [dp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        L.orc_fft_fit.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
        L.orc_fft_fit.restype = ctypes.c_uint32
        for name, args in [("orc_geom_sphere", [ld, ld]),
                           ("orc_geom_cylinder", [ld, ld, ld]),
                           ("orc_geom_box", [ld, ld, ld, ld]),
                           ("orc_geom_load_text", [ctypes.c_char_p, ld]),
                           ("orc_geom_from_arrays", [u32p, u8p, ctypes.c_uint32, ld])]:
            getattr(L, name).argtypes = args
            getattr(L, name).restype = vp
        L.orc_geom_nv.argtypes = [vp]
        L.orc_geom_nv.restype = ctypes.c_uint32
        L.orc_geom_matcount.argtypes = [vp]
        L.orc_geom_matcount.restype = ctypes.c_uint32
        L.orc_geom_box_size.argtypes = [vp, u32p]
        L.orc_geom_positions.argtypes = [vp, u32p]
        L.orc_geom_materials.argtypes = [vp, u8p]
        L.orc_geom_free.argtypes = [vp]
        L.orc_problem_create.argtypes = [vp, ctypes.POINTER(ld), ctypes.c_uint32, ld,
                                         u32p, ctypes.c_int]
        L.orc_problem_create.restype = vp
        L.orc_problem_free.argtypes = [vp]
        L.orc_problem_info.argtypes = [vp, u32p, dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_beam_pol.argtypes = [dp, ctypes.c_int, dp, dp]
        L.orc_set_cc.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int]
        L.orc_get_cc.argtypes = [vp, dp, dp, dp]
        L.orc_set_cc_sqrt.argtypes = [vp, dp]
        L.orc_build_dmatrix.argtypes = [vp]
        L.orc_get_dmatrix.argtypes = [vp, dp]
        L.orc_set_dmatrix.argtypes = [vp, dp]
        L.orc_matvec.argtypes = [vp, dp, dp, ctypes.c_int]
        L.orc_direct_matvec.argtypes = [vp, dp, dp]
        L.orc_einc.argtypes = [vp, dp, ctypes.c_int, dp]
        L.orc_coords.argtypes = [vp, dp]
        L.orc_set_cc_frame.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc_solve.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_int64,
                                dp, dp, ctypes.POINTER(OrcStats), ctypes.c_int64, dp,
                                ctypes.c_int64]
        L.orc_solve.restype = ctypes.c_int
        L.orc_solve_f32.argtypes = L.orc_solve.argtypes
        L.orc_solve_f32.restype = ctypes.c_int
        L.orc_calc_field.argtypes = [vp, dp, dp, dp]
        L.orc_cross_sections.argtypes = [vp, dp, dp, ctypes.c_int, dp, dp]
        L.orc_jones.argtypes = [vp, dp, dp, dp, dp, dp, ctypes.c_int64, dp]
        L.orc_mie.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def parse_length(s):
    """EMSim::Length parse: returns the long-double value as a ctypes object."""
    v = ctypes.c_longdouble()
    if lib().orc_parse_length(s.encode(), ctypes.byref(v)) != 0:
        raise ValueError("bad length %r" % s)
    return v


def parse_number(s):
    v = ctypes.c_longdouble()
    if lib().orc_parse_number(str(s).encode(), ctypes.byref(v)) != 0:
        raise ValueError("bad number %r" % s)
    return v


def fft_fit(x, override=0, support_nonpot=True):
    return int(lib().orc_fft_fit(x, override, 1 if support_nonpot else 0))


def fft(x, inverse=False):
    """Unnormalised DFT along the last axis (FFTW sign convention)."""
    a = np.array(x, dtype=np.complex128, order="C", copy=True)
    n = a.shape[-1]
    lib().orc_fft(_dp(a), n, a.size // n, 1 if inverse else 0)
    return a


def rotation_inverse(orient):
    """The inverse of the particle orientation R = Rz(alpha) Ry(beta) Rz(gamma)
    (ZYZ Euler angles in degrees; EMSim::Rotation::fromZYZDeg,
    EMSim/Rotation.hpp:94-102) as a 3x3 matrix: Rz(-gamma) Ry(-beta) Rz(-alpha),
    built from rotation matrices rather than the quaternions the reference
    uses."""
    a, b, g = (np.radians(float(x)) for x in orient)

    def rz(t):
        return np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])

    def ry(t):
        return np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])

    return rz(-g) @ ry(-b) @ rz(-a)


def beam_frame(prop, orient, center=(0.0, 0.0, 0.0)):
    """(prop, pol1, pol2, center) of the beam in the particle frame
    (DDA/Beam.hpp:69-81 with DipoleGeometry::orientationInverse)."""
    m = rotation_inverse(orient)
    p1, pn = beam_pol(prop, 1)
    p2, _ = beam_pol(prop, 2)
    return m @ pn, m @ p1, m @ p2, m @ np.asarray(center, dtype=np.float64)


def beam_pol(prop, pol):
    out = np.zeros(3)
    pr = np.zeros(3)
    lib().orc_beam_pol(_dp(np.asarray(prop, dtype=np.float64)), pol, _dp(out), _dp(pr))
    return out, pr


class Geometry:
    """Dipole list (positions z-sorted, 0-based material indices)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("oracle geometry: " + lib().orc_last_error().decode())
        self.h = handle

    @classmethod
    def sphere(cls, radius, grid_unit):
        return cls(lib().orc_geom_sphere(parse_length(radius), parse_length(grid_unit)))

    @classmethod
    def cylinder(cls, length, radius, grid_unit):
        return cls(lib().orc_geom_cylinder(parse_length(length), parse_length(radius),
                                           parse_length(grid_unit)))

    @classmethod
    def box(cls, sx, sy, sz, grid_unit):
        return cls(lib().orc_geom_box(parse_length(sx), parse_length(sy), parse_length(sz),
                                      parse_length(grid_unit)))

    @classmethod
    def load_text(cls, path, grid_unit):
        return cls(lib().orc_geom_load_text(path.encode(), parse_length(grid_unit)))

    @classmethod
    def from_arrays(cls, positions, materials, grid_unit):
        pos = np.ascontiguousarray(positions, dtype=np.uint32).reshape(-1, 3)
        mat = np.ascontiguousarray(materials, dtype=np.uint8)
        return cls(lib().orc_geom_from_arrays(
            pos.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            mat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(mat),
            parse_length(grid_unit)))

    @property
    def nv(self):
        return int(lib().orc_geom_nv(self.h))

    @property
    def box_size(self):
        b = (ctypes.c_uint32 * 3)()
        lib().orc_geom_box_size(self.h, b)
        return tuple(b)

    @property
    def mat_count(self):
        return int(lib().orc_geom_matcount(self.h))

    def positions(self):
        out = np.zeros((self.nv, 3), dtype=np.uint32)
        lib().orc_geom_positions(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return out

    def materials(self):
        out = np.zeros(self.nv, dtype=np.uint8)
        lib().orc_geom_materials(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_geom_free(self.h)
            self.h = None


class Problem:
    """DDAParams + couple constants + D matrix + matvec + solvers (FP64)."""

    def __init__(self, geom, materials, lam, grid=None, support_nonpot=True):
        nmat = len(materials)
        arr = (ctypes.c_longdouble * (nmat * 6))()
        for i, m in enumerate(materials):
            comps = m if isinstance(m, (list, tuple)) else (m, m, m)
            for j in range(3):
                c = complex(comps[j])
                # decimal text parsed in long double, like EMSim::parse
                for k, part in enumerate((c.real, c.imag)):
                    v = parse_number(repr(part))
                    ctypes.memmove(ctypes.addressof(arr) + (i * 6 + 2 * j + k) * ctypes.sizeof(v),
                                   ctypes.addressof(v), ctypes.sizeof(v))
        lam_ld = parse_length(lam) if isinstance(lam, str) else ctypes.c_longdouble(lam)
        g = (ctypes.c_uint32 * 3)(*(grid or (0, 0, 0)))
        self.h = lib().orc_problem_create(geom.h, arr, nmat, lam_ld, g,
                                          1 if support_nonpot else 0)
        if not self.h:
            raise ValueError("oracle problem: " + lib().orc_last_error().decode())
        info = (ctypes.c_uint32 * 9)()
        dinfo = (ctypes.c_double * 4)()
        lib().orc_problem_info(self.h, info, dinfo)
        self.nv, self.nvs = info[0], info[1]
        self.box = tuple(info[2:5])
        self.grid = tuple(info[5:8])
        self.nmat = info[8]
        self.grid_unit, self.wave_num, self.kd, self.grid_unit_vol = tuple(dinfo)
        self.geom = geom

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_problem_free(self.h)
            self.h = None

    @property
    def vec_size(self):
        return 3 * self.nvs

    def set_cc(self, prop=(0, 0, 1), pol=1, kind="ldr"):
        lib().orc_set_cc(self.h, POLARIZABILITIES[kind], _dp(np.asarray(prop, dtype=np.float64)), pol)

    def set_cc_frame(self, prop_p, pol_p, kind="ldr"):
        """Couple constants for a beam given in the particle frame."""
        lib().orc_set_cc_frame(self.h, POLARIZABILITIES[kind], _dp(np.asarray(prop_p, dtype=np.float64)),
                               _dp(np.asarray(pol_p, dtype=np.float64)))

    def einc_frame(self, prop_p, pol_p):
        """Plane-wave incident field [3 nvs] for a propagation direction and a
        polarisation vector in the particle frame (DDA/Beam.cpp:113-117):
        exp(i k r . prop_p) pol_p, in numpy."""
        ph = self.coords() @ np.asarray(prop_p, dtype=np.float64) * self.wave_num
        out = np.zeros((3, self.nvs), dtype=np.complex128)
        out[:, :self.nv] = np.asarray(pol_p, dtype=np.float64)[:, None] * np.exp(1j * ph)[None, :]
        return out.reshape(-1)

    def set_cc_sqrt(self, cc_sqrt):
        a = np.ascontiguousarray(cc_sqrt, dtype=np.complex128)
        lib().orc_set_cc_sqrt(self.h, _dp(a.view(np.float64)))

    def cc(self):
        n = self.nmat * 3
        a, b, c = (np.zeros(n, dtype=np.complex128) for _ in range(3))
        lib().orc_get_cc(self.h, _dp(a), _dp(b), _dp(c))
        return a, b, c

    def build_dmatrix(self):
        lib().orc_build_dmatrix(self.h)

    def dmatrix(self):
        gx, gy, gz = self.grid
        out = np.zeros((gx, gz, gy, 6), dtype=np.complex128)
        lib().orc_get_dmatrix(self.h, _dp(out))
        return out

    def set_dmatrix(self, d):
        a = np.ascontiguousarray(d, dtype=np.complex128)
        lib().orc_set_dmatrix(self.h, _dp(a))

    def matvec(self, arg, conj=False):
        a = np.ascontiguousarray(arg, dtype=np.complex128)
        out = np.zeros(self.vec_size, dtype=np.complex128)
        lib().orc_matvec(self.h, _dp(a), _dp(out), 1 if conj else 0)
        return out

    def direct_matvec(self, arg):
        a = np.ascontiguousarray(arg, dtype=np.complex128)
        out = np.zeros(self.vec_size, dtype=np.complex128)
        lib().orc_direct_matvec(self.h, _dp(a), _dp(out))
        return out

    def einc(self, prop=(0, 0, 1), pol=1):
        out = np.zeros(self.vec_size, dtype=np.complex128)
        lib().orc_einc(self.h, _dp(np.asarray(prop, dtype=np.float64)), pol, _dp(out))
        return out

    def coords(self):
        """Dipole coordinates [nv][3] in metres (origin at the box centre)."""
        out = np.zeros((self.nv, 3))
        lib().orc_coords(self.h, _dp(out))
        return out

    def einc_gaussian(self, prop, pol, kind, waist, center=(0.0, 0.0, 0.0), orient=(0, 0, 0)):
        """Gaussian-beam incident field [3 nvs] (Beams::Gaussian::createEInc,
        DDA/Beam.cpp:196-263), restated in numpy over all dipoles at once, in
        the reference's order of operations: beam frame ex = polarisation
        vector, ey = -pol-2 vector (pol 1) or the pol-1 vector (pol 2), z along
        prop; Q = 1/(2 zeta - i), psi0 = -i Q exp(i rho^2 Q), phase exp(i k z);
        kind "lminus" (DDA/Beam.cpp:217-218), "davis3" (225-238), "barton5"
        (239-256)."""
        k = self.wave_num
        pn, p1, p2, cp = beam_frame(prop, orient, center)
        ex = p1 if pol == 1 else p2
        ey = -p2 if pol == 1 else p1
        w0 = waist
        b = k * w0 * w0
        coord = self.coords() - cp[None, :]
        x, y, z = coord @ ex, coord @ ey, coord @ pn
        xi, eta, zeta = x / w0, y / w0, z / b
        rho2 = xi * xi + eta * eta
        Q = 1.0 / (2 * zeta - 1j)
        psi0 = -1j * Q * np.exp(1j * rho2 * Q)
        phase = np.exp(1j * k * z)
        zero = np.zeros_like(Q)
        if kind == "lminus":
            xf, yf, zf = np.ones_like(Q), zero, zero
        else:
            s = 1 / (k * w0)
            s2 = s * s
            rho4 = rho2 * rho2
            Q2 = Q * Q
            Q3 = Q2 * Q
            Q4 = Q2 * Q2
            xi2 = xi * xi
            if kind == "davis3":
                s3 = s2 * s
                xf = 1 + s2 * (-4 * Q2 * xi2 - 1j * Q3 * rho4)
                yf = zero
                zf = -s * 2 * Q * xi + s3 * (8 * Q3 * rho2 * xi + 2j * Q4 * rho4 * xi - 4j * Q2 * xi)
            elif kind == "barton5":
                Q5 = Q4 * Q
                xf = (1 + s2 * (-rho2 * Q2 - 1j * rho4 * Q3 - 2 * Q2 * xi2)
                      + s ** 4 * (2 * rho4 * Q4 + 3j * rho4 * rho2 * Q5 - 0.5 * rho4 * rho4 * Q4 * Q2
                                  + (8 * rho2 * Q4 + 2j * rho4 * Q5) * xi2))
                yf = s2 * (-2 * Q2 * xi * eta) + s2 * s2 * ((8 * rho2 * Q4 + 2j * rho4 * Q5) * xi * eta)
                zf = (s * (-2 * Q * xi) + s2 * s * ((6 * rho2 * Q3 + 2j * rho4 * Q4) * xi)
                      + s2 * s2 * s * ((-20 * rho4 * Q5 - 10j * rho4 * rho2 * Q4 * Q2 + rho4 * rho4 * Q4 * Q3) * xi))
            else:
                raise ValueError("unknown gaussian beam type " + kind)
        out = np.zeros((3, self.nvs), dtype=np.complex128)
        for a in range(3):
            out[a, :self.nv] = (ex[a] * (xf * psi0 * phase) + ey[a] * (yf * psi0 * phase)
                                + pn[a] * (zf * psi0 * phase))
        return out.reshape(-1)

    def calc_field(self, pvec, n):
        p = np.ascontiguousarray(pvec, dtype=np.complex128)
        out = np.zeros(3, dtype=np.complex128)
        lib().orc_calc_field(self.h, _dp(p), _dp(np.asarray(n, dtype=np.float64)), _dp(out))
        return out

    def cross_sections(self, pvec, prop, pol):
        """(Cext, Cabs) for the couple constants currently set."""
        p = np.ascontiguousarray(pvec, dtype=np.complex128)
        a, b = ctypes.c_double(), ctypes.c_double()
        lib().orc_cross_sections(self.h, _dp(p), _dp(np.asarray(prop, dtype=np.float64)), pol,
                                 ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def jones(self, pol1, pol2, prop, theta, phi):
        """Jones matrices [count][2][2] for polarisation-1/2 solutions."""
        p1 = np.ascontiguousarray(pol1, dtype=np.complex128)
        p2 = np.ascontiguousarray(pol2, dtype=np.complex128)
        th = np.ascontiguousarray(theta, dtype=np.float64)
        ph = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros((len(th), 2, 2), dtype=np.complex128)
        lib().orc_jones(self.h, _dp(p1), _dp(p2), _dp(np.asarray(prop, dtype=np.float64)), _dp(th),
                        _dp(ph), len(th), _dp(out))
        return out

    def solve(self, einc, solver="qmr", eps=1e-5, max_iter=0, start=None, stop_after=0,
              history_cap=100000, precision="fp64"):
        """getPolVec of the reference's CPU path: precision "fp64" (--ftype
        double) or "fp32" (--ftype float: D, matvec, vectors and scalars in
        float).  Returns (status, polarisations, stats, residual history)."""
        e = np.ascontiguousarray(einc, dtype=np.complex128)
        pol = np.zeros(self.vec_size, dtype=np.complex128)
        st = OrcStats()
        hist = np.zeros(history_cap)
        s = None if start is None else np.ascontiguousarray(start, dtype=np.complex128)
        fn = lib().orc_solve_f32 if precision == "fp32" else lib().orc_solve
        rc = fn(self.h, SOLVERS[solver], _dp(e), eps, max_iter,
                             None if s is None else _dp(s), _dp(pol), ctypes.byref(st),
                             stop_after, _dp(hist), history_cap)
        return rc, pol, st, hist[:min(st.iterations, history_cap)].copy()


def mie(x, m):
    """Bohren-Huffman efficiencies (Qext, Qsca, Qabs) of a sphere."""
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().orc_mie(x, complex(m).real, complex(m).imag, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def set_threads(n):
    lib().orc_set_threads(n)


def max_threads():
    return int(lib().orc_max_threads())
