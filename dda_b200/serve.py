"""Python side of the request loop (include/dda_serve.h).

    srv = Server(max_active=4)
    rid = srv.submit(target, wavelength="1um", prop=(0, 0, 1))
    results = srv.drain()          # list of dicts, one per finished request

A target is (positions [nv][3] uint32 sorted by z, materials [nv] uint8 or
None, refractive indices [nmat] (complex or 3 complex per material), grid
unit string).  Results carry the solve statistics, Cext / Cabs of each
polarisation and the server-clock times of submission, admission and
completion; with keep_pol=True also the polarisations [npol][3 nvs].
"""
import ctypes

import numpy as np

from .api import DDAError, POLARIZABILITIES, PRECISIONS, SOLVERS, Stats, lib

vp = ctypes.c_void_p
GRID_POLICIES = {"reference": 0, "tuned": 1}


class Request(ctypes.Structure):
    _fields_ = [("positions", ctypes.POINTER(ctypes.c_uint32)), ("materials", ctypes.POINTER(ctypes.c_uint8)),
                ("nv", ctypes.c_uint32), ("nmat", ctypes.c_uint32), ("refr", ctypes.POINTER(ctypes.c_double)),
                ("grid_unit", ctypes.c_char_p), ("wavelength", ctypes.c_char_p), ("prop", ctypes.c_double * 3),
                ("npol", ctypes.c_int32), ("polarizability", ctypes.c_int32), ("solver", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("eps", ctypes.c_double), ("max_iter", ctypes.c_int64),
                ("keep_pol", ctypes.c_int32), ("first_pol", ctypes.c_int32), ("grid_policy", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("tag", ctypes.c_uint64)]


class Result(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("tag", ctypes.c_uint64), ("status", ctypes.c_int32),
                ("npol", ctypes.c_int32), ("stats", Stats * 2), ("cext", ctypes.c_double * 2),
                ("cabs", ctypes.c_double * 2), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("t_setup", ctypes.c_double), ("t_solved", ctypes.c_double),
                ("footprint", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("grid", ctypes.c_uint32 * 3), ("nv", ctypes.c_uint32), ("nvs", ctypes.c_int64),
                ("pol", ctypes.POINTER(ctypes.c_double)), ("error", ctypes.c_char * 160)]


def _bind():
    L = lib()
    if getattr(L, "_serve_bound", False):
        return L
    sig = {
        "dda_serve_create": ([ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "dda_serve_submit": ([vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "dda_serve_poll": ([vp, ctypes.POINTER(Result), ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "dda_serve_release": ([vp, ctypes.c_int64], ctypes.c_int),
        "dda_serve_cancel": ([vp, ctypes.c_int64], ctypes.c_int),
        "dda_serve_pending": ([vp], ctypes.c_int64),
        "dda_serve_clock": ([vp], ctypes.c_double),
        "dda_serve_destroy": ([vp], ctypes.c_int),
        "dda_serve_error": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    L._serve_bound = True
    return L


def _refr_array(refr):
    out = []
    for m in refr:
        out.extend(m if isinstance(m, (list, tuple)) else (m, m, m))
    return np.array(out, dtype=np.complex128)


class Server:
    """Continuous-batching request loop on one device (dda_serve_*)."""

    def __init__(self, device=0, budget_bytes=0, max_active=4):
        L = _bind()
        h = vp()
        rc = L.dda_serve_create(device, int(budget_bytes), max_active, ctypes.byref(h))
        if rc != 0:
            raise DDAError(rc, L.dda_serve_error().decode())
        self.h = h
        self.L = L

    def submit(self, positions, materials, refr, grid_unit, wavelength, prop=(0, 0, 1), npol=2,
               polarizability="ldr", solver="qmr", precision="mixed", eps=1e-5, max_iter=0, keep_pol=False,
               tag=0, first_pol=1, grid_policy="tuned"):
        pos = np.ascontiguousarray(positions, dtype=np.uint32).reshape(-1, 3)
        mat = None if materials is None else np.ascontiguousarray(materials, dtype=np.uint8)
        r = _refr_array(refr)
        q = Request()
        q.positions = pos.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        q.materials = mat.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if mat is not None else None
        q.nv = len(pos)
        q.nmat = len(r) // 3
        q.refr = r.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        q.grid_unit = grid_unit.encode()
        q.wavelength = wavelength.encode()
        q.prop = (ctypes.c_double * 3)(*prop)
        q.npol = npol
        q.polarizability = POLARIZABILITIES[polarizability]
        q.solver = SOLVERS[solver]
        q.precision = PRECISIONS[precision]
        q.eps = eps
        q.max_iter = max_iter
        q.keep_pol = 1 if keep_pol else 0
        q.first_pol = first_pol
        q.grid_policy = GRID_POLICIES[grid_policy]
        q.tag = tag
        rid = ctypes.c_int64()
        rc = self.L.dda_serve_submit(self.h, ctypes.byref(q), ctypes.byref(rid))
        if rc != 0:
            raise DDAError(rc, self.L.dda_serve_error().decode())
        return rid.value

    def poll(self, max_results=64, timeout_ms=-1):
        buf = (Result * max_results)()
        n = self.L.dda_serve_poll(self.h, buf, max_results, timeout_ms)
        out = []
        for i in range(n):
            r = buf[i]
            d = {"id": r.id, "tag": r.tag, "status": r.status, "npol": r.npol,
                 "iterations": [r.stats[k].iterations for k in range(r.npol)],
                 "refinements": [r.stats[k].refinements for k in range(r.npol)],
                 "rel_residual": [r.stats[k].rel_residual for k in range(r.npol)],
                 "cext": list(r.cext)[:r.npol], "cabs": list(r.cabs)[:r.npol],
                 "t_submit": r.t_submit, "t_admit": r.t_admit, "t_done": r.t_done, "t_setup": r.t_setup,
                 "t_solved": r.t_solved,
                 "footprint": r.footprint, "device_bytes": r.device_bytes, "grid": tuple(r.grid),
                 "nv": r.nv, "nvs": r.nvs, "error": r.error.decode(errors="replace")}
            if r.pol:
                n_d = r.npol * 3 * r.nvs * 2
                d["pol"] = np.ctypeslib.as_array(r.pol, shape=(n_d,)).view(np.complex128).copy().reshape(r.npol, -1)
                self.L.dda_serve_release(self.h, r.id)
            out.append(d)
        return out

    def cancel(self, rid):
        """dda_serve_cancel: a queued request leaves the queue, a running one
        stops after its current round; its result has status -8."""
        rc = self.L.dda_serve_cancel(self.h, rid)
        if rc != 0:
            raise DDAError(rc, "request %d is neither queued nor running" % rid)

    @property
    def pending(self):
        return int(self.L.dda_serve_pending(self.h))

    def clock(self):
        return float(self.L.dda_serve_clock(self.h))

    def drain(self):
        """Waits for every queued and running request; returns their results."""
        out = []
        while True:
            got = self.poll(timeout_ms=-1)
            out.extend(got)
            if not got and self.pending == 0:
                return out

    def close(self):
        if getattr(self, "h", None):
            self.L.dda_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
