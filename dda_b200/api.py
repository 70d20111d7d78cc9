"""ctypes binding of libdda_b200.so and the reference-shaped host classes."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_HERE, "libdda_b200.so")

SOLVERS = {"qmr": 0, "bicgstab": 1, "bicg": 2, "cgnr": 3}
PRECISIONS = {"fp64": 0, "fp32": 1, "mixed": 2}
POLARIZABILITIES = {"cm": 0, "ldr": 1, "ldr-avgpol": 2}
GRID_POLICIES = {"reference": 0, "tuned": 1}
ERRORS = {-1: "invalid argument", -2: "CUDA failure", -3: "out of device memory",
          -4: "unsupported size", -5: "Krylov breakdown", -6: "Too many iterations",
          -7: "Too many iterations w/o increase", -8: "cancelled"}


class DDAError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


class Problem(ctypes.Structure):
    _fields_ = [("nv", ctypes.c_uint32), ("box", ctypes.c_uint32 * 3),
                ("grid", ctypes.c_uint32 * 3), ("positions", ctypes.POINTER(ctypes.c_uint32)),
                ("materials", ctypes.POINTER(ctypes.c_uint8)), ("nmat", ctypes.c_uint32),
                ("kd", ctypes.c_double), ("grid_unit", ctypes.c_double),
                ("dmatrix", ctypes.POINTER(ctypes.c_double)), ("max_rhs", ctypes.c_int32),
                ("device", ctypes.c_int32), ("flags", ctypes.c_uint32)]

FLAG_SPLIT_YZ = 1
FLAG_YZ_GROUPS2 = 32
FLAG_YZ_GROUPS4 = 64
FLAG_YZ_PAIR = 128


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("matvecs", ctypes.c_int64),
                ("refinements", ctypes.c_int64), ("rel_residual", ctypes.c_double),
                ("res_scale", ctypes.c_double), ("status", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


_lib = None


def lib():
    """Loads libdda_b200.so (building it first when nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(lib_path):
        from . import build
        build.build()
    L = ctypes.CDLL(lib_path)
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    cp = ctypes.c_char_p
    sig = {
        "dda_create": ([ctypes.POINTER(Problem), ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_destroy": ([vp], ctypes.c_int),
        "dda_last_error": ([vp], cp),
        "dda_vec_stride": ([vp], ctypes.c_int64),
        "dda_set_cc": ([vp, ctypes.c_int, dp], ctypes.c_int),
        "dda_matvec": ([vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
        "dda_matvec_host": ([vp, dp, dp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "dda_solve": ([vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, ctypes.c_int64, dp, dp,
                       dp, ctypes.c_int64, ctypes.POINTER(Stats)], ctypes.c_int),
        "dda_solve_f32": ([vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_double, ctypes.c_int64, vp, vp,
                           dp, ctypes.c_int64, ctypes.POINTER(Stats)], ctypes.c_int),
        "dda_get_dmatrix": ([vp, dp], ctypes.c_int),
        "dda_solve_device": ([vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_double, ctypes.c_int64, vp, vp,
                              ctypes.POINTER(Stats)], ctypes.c_int),
        "dda_stream": ([vp], vp),
        "dda_cancel": ([vp], ctypes.c_int),
        "dda_launch_count": ([vp], ctypes.c_int64),
        "dda_matvec_layout": ([vp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "dda_profile_matvec": ([vp, ctypes.c_int, ctypes.c_int, dp], ctypes.c_int),
        "dda_synchronize": ([vp], ctypes.c_int),
        "dda_far_field": ([vp, ctypes.c_int, dp, ctypes.c_int64, dp, dp], ctypes.c_int),
        "dda_far_field_noalloc": ([vp, ctypes.c_int, ctypes.c_int64, dp, dp], ctypes.c_int),
        "dda_frontend_error": ([], cp),
        "dda_fft_fit": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int], ctypes.c_uint32),
        "dda_parse_length_m": ([cp, dp], ctypes.c_int),
        "dda_geom_sphere": ([cp, cp, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_geom_cylinder": ([cp, cp, cp, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_geom_box": ([cp, cp, cp, cp, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_geom_load": ([cp, cp, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_geom_from_arrays": ([u32p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint32, cp,
                                  ctypes.POINTER(vp)], ctypes.c_int),
        "dda_geom_free": ([vp], None),
        "dda_geom_nv": ([vp], ctypes.c_uint32),
        "dda_geom_nmat": ([vp], ctypes.c_uint32),
        "dda_geom_box_size": ([vp, u32p], None),
        "dda_geom_grid_unit": ([vp], ctypes.c_double),
        "dda_geom_positions": ([vp], u32p),
        "dda_geom_materials": ([vp], ctypes.POINTER(ctypes.c_uint8)),
        "dda_beam_pol": ([dp, ctypes.c_int, dp, dp], None),
        "dda_couple_constants": ([ctypes.c_int, ctypes.c_uint32, dp, ctypes.c_double, ctypes.c_double,
                                  dp, ctypes.c_int, dp, dp, dp], ctypes.c_int),
        "dda_einc_plane": ([vp, ctypes.c_double, dp, ctypes.c_int, dp], ctypes.c_int),
        "dda_einc_gaussian": ([vp, ctypes.c_double, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp],
                              ctypes.c_int),
        "dda_beam_frame": ([dp, dp, dp, dp, dp, dp, dp], None),
        "dda_einc_plane_frame": ([vp, ctypes.c_double, dp, dp, dp], ctypes.c_int),
        "dda_einc_gaussian_frame": ([vp, ctypes.c_double, dp, dp, dp, ctypes.c_int, ctypes.c_double, dp, dp],
                                    ctypes.c_int),
        "dda_couple_constants_frame": ([ctypes.c_int, ctypes.c_uint32, dp, ctypes.c_double, ctypes.c_double,
                                        dp, dp, dp, dp, dp], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _cbuf(a):
    """complex128 array -> contiguous, returns (array, double*)"""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a, _dp(a.view(np.float64))


def _front_check(rc):
    if rc != 0:
        raise DDAError(-1, lib().dda_frontend_error().decode())


def fft_fit(x, override=0, support_nonpot=True):
    """DDA/DDAParams.cpp:45-90."""
    return int(lib().dda_fft_fit(x, override, 1 if support_nonpot else 0))


def beam_pol(prop, pol):
    out = np.zeros(3)
    pn = np.zeros(3)
    lib().dda_beam_pol(_dp(np.asarray(prop, dtype=np.float64)), pol, _dp(out), _dp(pn))
    return out, pn


def beam_frame(prop, orient=None, center=None):
    """(prop_p, pol1_p, pol2_p, center_p): the beam's propagation direction,
    polarisation vectors and a point (the Gaussian beam's centre) in the
    frame of a particle oriented by the ZYZ Euler angles `orient` in degrees
    (--orient; DipoleGeometry::orientationInverse, DDA/DipoleGeometry.cpp:
    149-152, applied as in DDA/Beam.hpp:69-81)."""
    out = [np.zeros(3) for _ in range(4)]
    o = None if orient is None else _dp(np.asarray(orient, dtype=np.float64))
    c = None if center is None else _dp(np.asarray(center, dtype=np.float64))
    lib().dda_beam_frame(_dp(np.asarray(prop, dtype=np.float64)), o, _dp(out[0]), _dp(out[1]), _dp(out[2]), c,
                         _dp(out[3]))
    return tuple(out)


def oriented(orient):
    """True for a particle orientation other than the identity."""
    return orient is not None and any(float(x) != 0.0 for x in orient)


def parse_length(s):
    v = ctypes.c_double()
    _front_check(lib().dda_parse_length_m(s.encode(), ctypes.byref(v)))
    return v.value


GAUSSIAN_BEAMS = {"lminus": 0, "davis3": 1, "barton5": 2}


class Beam:
    """The incident beam of the reference's --beam option: "plane", or
    "gaussian:<lminus|davis3|barton5>,<waist>[,(x,y,z)]" with EMSim lengths
    ("2um"; the centre relative to the target's centre) -- Beam::parseBeam and
    Beams::Gaussian::parse (DDA/Beam.cpp:68-98, 139-181).  lminus is the
    fundamental Gaussian mode, davis3 and barton5 add the third- and
    fifth-order corrections (DDA/Beam.hpp:126-129)."""

    def __init__(self, spec="plane"):
        self.spec = spec
        i = 0
        while i < len(spec) and "a" <= spec[i] <= "z":
            i += 1
        name = spec[:i]
        while i < len(spec) and spec[i] in " \t:":
            i += 1
        rest = spec[i:]
        self.kind, self.waist, self.center = None, None, (0.0, 0.0, 0.0)
        if name == "plane":
            if rest:
                raise ValueError("the plane beam takes no parameters: " + spec)
        elif name == "gaussian":
            j = 0
            while j < len(rest) and (rest[j].isdigit() or "a" <= rest[j] <= "z"):
                j += 1
            kind = rest[:j]
            while j < len(rest) and rest[j] in " \t,":
                j += 1
            value = rest[j:]
            if kind not in GAUSSIAN_BEAMS:
                raise ValueError("unknown gaussian beam type `%s'" % kind)
            size, _, center = value.partition(",")
            self.kind = kind
            self.waist = parse_length(size.strip())
            if not self.waist > 0:
                raise ValueError("the waist must be positive: " + spec)
            if center.strip():
                c = center.strip()
                if not (c.startswith("(") and c.endswith(")")):
                    raise ValueError("beam centre must read (x,y,z): " + spec)
                parts = [x.strip() for x in c[1:-1].split(",")]
                if len(parts) != 3:
                    raise ValueError("beam centre must read (x,y,z): " + spec)
                self.center = tuple(parse_length(x) for x in parts)
        else:
            raise ValueError("unknown beam `%s'" % name)

    @property
    def plane(self):
        return self.kind is None

    def einc(self, params, prop=(0, 0, 1), pol=1, orient=None):
        """Incident field [3 nvs] complex of polarisation pol (orient: the
        particle orientation, ZYZ Euler angles in degrees)."""
        if self.plane:
            return params.einc(prop, pol, orient=orient)
        out = np.zeros(params.vec_size, dtype=np.complex128)
        if oriented(orient):
            pp, p1, p2, cp = beam_frame(prop, orient, self.center)
            ex, ey = (p1, -p2) if pol == 1 else (p2, p1)
            _front_check(lib().dda_einc_gaussian_frame(params.geometry.h, ctypes.c_double(params.wave_num), _dp(pp),
                                                       _dp(ex), _dp(ey), GAUSSIAN_BEAMS[self.kind],
                                                       ctypes.c_double(self.waist), _dp(cp),
                                                       _dp(out.view(np.float64))))
            return out
        center = np.asarray(self.center, dtype=np.float64)
        _front_check(lib().dda_einc_gaussian(params.geometry.h, ctypes.c_double(params.wave_num),
                                             _dp(np.asarray(prop, dtype=np.float64)), pol,
                                             GAUSSIAN_BEAMS[self.kind], ctypes.c_double(self.waist), _dp(center),
                                             _dp(out.view(np.float64))))
        return out


class Geometry:
    """Dipole list: positions (nv x 3, sorted by z) and material indices."""

    def __init__(self, handle):
        self.h = handle
        L = lib()
        self.nv = int(L.dda_geom_nv(handle))
        b = (ctypes.c_uint32 * 3)()
        L.dda_geom_box_size(handle, b)
        self.box = tuple(b)
        self.nmat = int(L.dda_geom_nmat(handle))
        self.grid_unit = float(L.dda_geom_grid_unit(handle))
        self.positions = np.ctypeslib.as_array(L.dda_geom_positions(handle), shape=(self.nv, 3)).copy()
        self.materials = np.ctypeslib.as_array(L.dda_geom_materials(handle), shape=(self.nv,)).copy()

    @staticmethod
    def _make(fn, *args):
        h = ctypes.c_void_p()
        _front_check(fn(*[a.encode() if isinstance(a, str) else a for a in args], ctypes.byref(h)))
        return Geometry(h)

    @classmethod
    def sphere(cls, radius, grid_unit):
        return cls._make(lib().dda_geom_sphere, radius, grid_unit)

    @classmethod
    def cylinder(cls, length, radius, grid_unit):
        return cls._make(lib().dda_geom_cylinder, length, radius, grid_unit)

    @classmethod
    def box_shape(cls, sx, sy, sz, grid_unit):
        return cls._make(lib().dda_geom_box, sx, sy, sz, grid_unit)

    @classmethod
    def load(cls, path, grid_unit):
        return cls._make(lib().dda_geom_load, path, grid_unit)

    @classmethod
    def from_arrays(cls, positions, materials, grid_unit):
        pos = np.ascontiguousarray(positions, dtype=np.uint32).reshape(-1, 3)
        mat = np.ascontiguousarray(materials, dtype=np.uint8)
        h = ctypes.c_void_p()
        _front_check(lib().dda_geom_from_arrays(
            pos.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            mat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(mat), grid_unit.encode(),
            ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.dda_geom_free(self.h)
            self.h = None


class DDAParams:
    """Grid and vector layout of one target (DDA/DDAParams.cpp:93-214)."""

    def __init__(self, geometry, materials, wavelength, grid=None, support_nonpot=True, grid_policy="reference"):
        self.geometry = geometry
        self.materials = [m if isinstance(m, (list, tuple)) else (m, m, m) for m in materials]
        if len(self.materials) < geometry.nmat:
            raise DDAError(-1, "fewer refractive indices than material indices")
        self.wavelength = parse_length(wavelength) if isinstance(wavelength, str) else float(wavelength)
        self.nv = geometry.nv
        self.nvs = (self.nv + 15) // 16 * 16
        self.box = geometry.box
        g = grid or (0, 0, 0)
        self.grid = tuple(fft_fit(2 * b, o, support_nonpot) for b, o in zip(self.box, g))
        if grid is None and grid_policy != "reference":
            # dda_choose_grid: lengths with compile-time FFT plans (same
            # matvec up to rounding, the zero padding being exact)
            box = (ctypes.c_uint32 * 3)(*self.box)
            out = (ctypes.c_uint32 * 3)()
            L = lib()
            L.dda_choose_grid.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_uint32)]
            if L.dda_choose_grid(box, GRID_POLICIES[grid_policy], out) != 0:
                raise DDAError(-1, "bad grid policy")
            self.grid = tuple(out)
        self.grid_unit = geometry.grid_unit
        self.wave_num = 2 * np.pi / self.wavelength
        self.kd = self.wave_num * self.grid_unit

    @property
    def vec_size(self):
        return 3 * self.nvs

    def einc(self, prop=(0, 0, 1), pol=1, beam=None, orient=None):
        """Incident field [3 nvs] complex: the plane wave, or `beam` (a Beam
        or its --beam string); orient: the particle orientation (ZYZ Euler
        angles in degrees, --orient)."""
        if beam is not None:
            b = beam if isinstance(beam, Beam) else Beam(beam)
            if not b.plane:
                return b.einc(self, prop, pol, orient=orient)
        out = np.zeros(self.vec_size, dtype=np.complex128)
        if oriented(orient):
            pp, p1, p2, _ = beam_frame(prop, orient)
            _front_check(lib().dda_einc_plane_frame(self.geometry.h, self.wave_num, _dp(pp),
                                                    _dp(p1 if pol == 1 else p2), _dp(out.view(np.float64))))
            return out
        _front_check(lib().dda_einc_plane(self.geometry.h, self.wave_num,
                                          _dp(np.asarray(prop, dtype=np.float64)), pol,
                                          _dp(out.view(np.float64))))
        return out


class CoupleConstants:
    """cc, sqrt(cc), chi_inv per material and axis (DDA/DDAParams.cpp:315-331)."""

    def __init__(self, params, prop=(0, 0, 1), pol=1, kind="ldr", orient=None):
        n = len(params.materials) * 3
        refr = np.array([c for m in params.materials for c in m], dtype=np.complex128)
        self.cc = np.zeros(n, dtype=np.complex128)
        self.cc_sqrt = np.zeros(n, dtype=np.complex128)
        self.chi_inv = np.zeros(n, dtype=np.complex128)
        if oriented(orient):  # LDR sees the beam in the particle frame
            pp, p1, p2, _ = beam_frame(prop, orient)
            _front_check(lib().dda_couple_constants_frame(
                POLARIZABILITIES[kind], len(params.materials), _dp(refr.view(np.float64)),
                params.grid_unit, params.wave_num, _dp(pp), _dp(p1 if pol == 1 else p2),
                _dp(self.cc.view(np.float64)), _dp(self.cc_sqrt.view(np.float64)),
                _dp(self.chi_inv.view(np.float64))))
            return
        _front_check(lib().dda_couple_constants(
            POLARIZABILITIES[kind], len(params.materials), _dp(refr.view(np.float64)),
            params.grid_unit, params.wave_num, _dp(np.asarray(prop, dtype=np.float64)), pol,
            _dp(self.cc.view(np.float64)), _dp(self.cc_sqrt.view(np.float64)),
            _dp(self.chi_inv.view(np.float64))))


class CudaMatVec:
    """The device context: D matrix, FFT plans and the matvec.

    apply() follows MatVec<T>::apply (host vectors in, host vector out);
    apply_device() follows GpuMatVec<T>::apply on device pointers.
    """

    def __init__(self, params, precision="fp64", max_rhs=1, dmatrix=None, device=0, flags=0):
        self.params = params
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else precision
        self.max_rhs = max_rhs
        geom = params.geometry
        self._pos = np.ascontiguousarray(geom.positions, dtype=np.uint32)
        self._mat = np.ascontiguousarray(geom.materials, dtype=np.uint8)
        p = Problem()
        p.nv = params.nv
        p.box = (ctypes.c_uint32 * 3)(*params.box)
        p.grid = (ctypes.c_uint32 * 3)(*params.grid)
        p.positions = self._pos.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        p.materials = self._mat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        p.nmat = len(params.materials)
        p.kd = params.kd
        p.grid_unit = params.grid_unit
        self._d = None
        if dmatrix is not None:
            self._d, p.dmatrix = _cbuf(dmatrix)
        p.max_rhs = max_rhs
        p.device = device
        p.flags = flags
        h = ctypes.c_void_p()
        rc = lib().dda_create(ctypes.byref(p), self.precision, ctypes.byref(h))
        if rc != 0:
            raise DDAError(rc, lib().dda_last_error(None).decode())
        self.h = h
        self.nvs = int(lib().dda_vec_stride(h))

    def _check(self, rc):
        if rc != 0:
            raise DDAError(rc, lib().dda_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            lib().dda_destroy(self.h)
            self.h = None

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.dda_destroy(self.h)
            self.h = None

    def set_couple_constants(self, cc, rhs=0):
        """MatVec<T>::setCoupleConstants (DDA/MatVec.hpp:46)."""
        s = cc.cc_sqrt if isinstance(cc, CoupleConstants) else cc
        a, p = _cbuf(s)
        self._check(lib().dda_set_cc(self.h, rhs, p))

    setCoupleConstants = set_couple_constants

    def apply(self, arg, conj=False):
        """MatVec<T>::apply (DDA/MatVec.hpp:54) on host vectors [nrhs][3 nvs]."""
        a, ap = _cbuf(arg)
        nrhs = a.size // (3 * self.nvs)
        out = np.zeros_like(a)
        self._check(lib().dda_matvec_host(self.h, ap, _dp(out.view(np.float64)), 1 if conj else 0, nrhs))
        return out

    def apply_device(self, arg_ptr, res_ptr, conj=False, nrhs=1, precision=None, stream=None):
        """GpuMatVec<T>::apply (DDA/GpuMatVec.hpp:99) on device buffers."""
        prec = self.precision if precision is None else (PRECISIONS[precision] if isinstance(precision, str) else precision)
        if prec == PRECISIONS["mixed"]:
            prec = PRECISIONS["fp32"]
        self._check(lib().dda_matvec(self.h, ctypes.c_void_p(arg_ptr), ctypes.c_void_p(res_ptr),
                                     1 if conj else 0, nrhs, prec,
                                     ctypes.c_void_p(stream) if stream else None))

    def dmatrix(self):
        gx, gy, gz = self.params.grid
        out = np.zeros((gx, gz, gy, 6), dtype=np.complex128)
        self._check(lib().dda_get_dmatrix(self.h, _dp(out.view(np.float64))))
        return out

    def synchronize(self):
        self._check(lib().dda_synchronize(self.h))

    def far_field(self, dirs, nrhs=1, pol=None):
        """Scattered far field E(n) for directions dirs [ndir][3] (particle
        frame) of `pol` ([nrhs][3 nvs]) or of the last solve: [ndir][nrhs][3]."""
        d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(d), nrhs, 3), dtype=np.complex128)
        pp = None
        if pol is not None:
            pa, pp = _cbuf(pol)
        self._check(lib().dda_far_field(self.h, nrhs, pp, len(d), _dp(d), _dp(out.view(np.float64))))
        return out

    def far_field_noalloc(self, dirs, nrhs=1):
        """far_field() of the last solve through dda_far_field_noalloc: no
        allocation, at most 1 MiB of directions and fields per call."""
        d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(d), nrhs, 3), dtype=np.complex128)
        self._check(lib().dda_far_field_noalloc(self.h, nrhs, len(d), _dp(d), _dp(out.view(np.float64))))
        return out

    def cancel(self):
        """dda_cancel: the solve running on this context (in another thread)
        stops after its current round and raises DDAError code -8."""
        self._check(lib().dda_cancel(self.h))

    @property
    def stream(self):
        """The context's cudaStream_t as an integer."""
        return lib().dda_stream(self.h) or 0

    @property
    def launches(self):
        """Kernels launched by this context so far."""
        return int(lib().dda_launch_count(self.h))

    @property
    def layout(self):
        """dda_matvec_layout as a dict."""
        v = (ctypes.c_int64 * 8)()
        self._check(lib().dda_matvec_layout(self.h, v))
        keys = ("yz_path", "clusters", "cluster_size", "rows_per_batch", "smem_yz", "lines_per_x_tile",
                "compile_time_plans", "device_bytes")
        d = dict(zip(keys, (int(x) for x in v)))
        d["yz_path"] = ("fused", "cluster", "split")[d["yz_path"]]
        if d["yz_path"] == "fused":  # slots 1, 2: CTAs per plane and thread groups
            d["groups"] = d.pop("cluster_size")
            d["ctas_per_plane"] = d.pop("clusters")
        return d

    def profile(self, nrhs=1, reps=10):
        """Mean ms of the matvec stages: x forward, y/z, x inverse, total."""
        ms = np.zeros(4)
        self._check(lib().dda_profile_matvec(self.h, nrhs, reps, _dp(ms)))
        return ms


class CudaSolver:
    """IterativeSolverBase<T>::getPolVec (DDA/IterativeSolverBase.cpp:40-103)
    with the solver chosen by its --iter name."""

    def __init__(self, matvec, solver="qmr", max_iter=0):
        self.mv = matvec
        self.solver = SOLVERS[solver]
        self.max_iter = max_iter
        self.last_stats = None
        self.last_history = None

    def get_pol_vec(self, einc, eps, start=None, history_cap=100000, raise_on_error=True, out=None):
        """Solves for one or more right-hand sides; einc is [nrhs][3 nvs].
        `out`, when given, is the C-contiguous array of einc's size and type
        that receives the polarisations (for instance a pinned host buffer,
        which makes both bus copies asynchronous DMA).  A complex64 einc
        (the reference's --ftype float vectors) goes through dda_solve_f32 and
        gives complex64 polarisations: on an FP32 context half the bytes
        cross the bus."""
        if isinstance(einc, np.ndarray) and einc.dtype == np.complex64:
            return self._get_pol_vec_f32(einc, eps, start, history_cap, raise_on_error, out)
        e, ep = _cbuf(einc)
        nvs = self.mv.nvs
        nrhs = e.size // (3 * nvs)
        if out is None:
            pol = np.zeros_like(e)
        else:
            if out.dtype != np.complex128 or out.size != e.size or not out.flags["C_CONTIGUOUS"]:
                raise ValueError("out must be a C-contiguous complex128 array of einc's size")
            pol = out
        sp = None
        if start is not None:
            s, sp = _cbuf(start)
        stats = (Stats * nrhs)()
        hist = np.zeros((nrhs, history_cap))
        rc = lib().dda_solve(self.mv.h, self.solver, nrhs, ep, eps, self.max_iter, sp,
                             _dp(pol.view(np.float64)), _dp(hist), history_cap, stats)
        self.last_stats = [stats[i] for i in range(nrhs)]
        self.last_history = [hist[i, :min(stats[i].iterations, history_cap)].copy() for i in range(nrhs)]
        if rc != 0 and raise_on_error:
            raise DDAError(rc, lib().dda_last_error(self.mv.h).decode())
        return pol

    def _get_pol_vec_f32(self, einc, eps, start, history_cap, raise_on_error, out):
        e = np.ascontiguousarray(einc)
        nrhs = e.size // (3 * self.mv.nvs)
        if out is None:
            pol = np.zeros_like(e)
        else:
            if out.dtype != np.complex64 or out.size != e.size or not out.flags["C_CONTIGUOUS"]:
                raise ValueError("out must be a C-contiguous complex64 array of einc's size")
            pol = out
        s = None if start is None else np.ascontiguousarray(start, dtype=np.complex64)
        stats = (Stats * nrhs)()
        hist = np.zeros((nrhs, history_cap))
        rc = lib().dda_solve_f32(self.mv.h, self.solver, nrhs, ctypes.c_void_p(e.ctypes.data), eps, self.max_iter,
                                 None if s is None else ctypes.c_void_p(s.ctypes.data),
                                 ctypes.c_void_p(pol.ctypes.data), _dp(hist), history_cap, stats)
        self.last_stats = [stats[i] for i in range(nrhs)]
        self.last_history = [hist[i, :min(stats[i].iterations, history_cap)].copy() for i in range(nrhs)]
        if rc != 0 and raise_on_error:
            raise DDAError(rc, lib().dda_last_error(self.mv.h).decode())
        return pol

    getPolVec = get_pol_vec

    def get_pol_vec_device(self, einc_ptr, pol_ptr, nrhs, eps, start_ptr=None, raise_on_error=True):
        """Device-resident solve: einc and pol are device buffers of the
        context precision ([nrhs][3 nvs] complex)."""
        stats = (Stats * nrhs)()
        rc = lib().dda_solve_device(self.mv.h, self.solver, nrhs, ctypes.c_void_p(einc_ptr), eps,
                                    self.max_iter, ctypes.c_void_p(start_ptr) if start_ptr else None,
                                    ctypes.c_void_p(pol_ptr), stats)
        self.last_stats = [stats[i] for i in range(nrhs)]
        if rc != 0 and raise_on_error:
            raise DDAError(rc, lib().dda_last_error(self.mv.h).decode())
        return rc
