"""CPU tests of the serving front end: the footprint bound used for
admission, and the target generators of the batched and served workloads."""
import ctypes

import numpy as np

from dda_b200 import api, targets


def _footprint(grid, box, nv, max_rhs, precision):
    p = api.Problem()
    p.nv = nv
    p.box = (ctypes.c_uint32 * 3)(*box)
    p.grid = (ctypes.c_uint32 * 3)(*grid)
    p.nmat = 1
    p.max_rhs = max_rhs
    res, peak = ctypes.c_int64(), ctypes.c_int64()
    L = api.lib()
    L.dda_footprint.argtypes = [ctypes.POINTER(api.Problem), ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_int64)]
    assert L.dda_footprint(ctypes.byref(p), api.PRECISIONS[precision], ctypes.byref(res), ctypes.byref(peak)) == 0
    return res.value, peak.value


def test_footprint_grows_with_rhs_and_precision():
    r1, p1 = _footprint((200, 100, 100), (100, 50, 50), 250000, 1, "fp32")
    r2, p2 = _footprint((200, 100, 100), (100, 50, 50), 250000, 2, "fp32")
    r3, _ = _footprint((200, 100, 100), (100, 50, 50), 250000, 1, "mixed")
    assert 0 < r1 < r2 and r1 < r3
    assert p1 - r1 == 200 * 100 * 100 * 16  # FP64 grid of the D-matrix generation
    # the plane-major x spectrum alone: Gx * 3 * by * bz complex FP32 per rhs
    assert r1 > 200 * 3 * 50 * 50 * 8


def test_spheroid_matches_cell_centre_count():
    # semi-axes 48 x 32 x 32 dipoles: 206 192 cells with centres inside
    p = targets.spheroid(48, 32, 32)
    assert len(p) == 206192
    assert tuple(p.max(axis=0)) == (95, 63, 63)
    assert np.all(np.diff(p[:, 2].astype(np.int64)) >= 0)


def test_served_requests_are_valid_targets():
    rng = np.random.default_rng(3)
    for _ in range(20):
        r = targets.served_request(rng, (6, 20))
        pos = r["positions"]
        assert len(pos) > 0 and pos.dtype == np.uint32
        assert np.all(np.diff(pos[:, 2].astype(np.int64)) >= 0)
        assert len(np.unique(pos, axis=0)) == len(pos)
        m = r["refr"][0]
        assert 1.05 <= m.real <= 2.0 and 0 <= m.imag <= 0.5
        assert abs(np.linalg.norm(r["prop"]) - 1) < 1e-12


TUNED = {32, 48, 56, 64, 80, 96, 100, 112, 120, 128, 144, 160, 168, 192, 200, 224, 240, 256, 288, 320, 384, 512}


def test_choose_grid_policies():
    L = api.lib()
    L.dda_choose_grid.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]
    for box in [(7, 6, 5), (35, 40, 45), (70, 81, 72), (100, 50, 50), (96, 64, 64), (256, 256, 256), (300, 10, 10)]:
        b = (ctypes.c_uint32 * 3)(*box)
        ref, tun = (ctypes.c_uint32 * 3)(), (ctypes.c_uint32 * 3)()
        assert L.dda_choose_grid(b, 0, ref) == 0 and L.dda_choose_grid(b, 1, tun) == 0
        assert tuple(ref) == tuple(api.fft_fit(2 * x) for x in box)
        if tuple(tun) != tuple(ref):
            assert all(g >= 2 * x and g in TUNED for g, x in zip(tun, box))
            assert tun[1] == tun[2]
            assert tun[0] * tun[1] * tun[2] <= 2 * ref[0] * ref[1] * ref[2]
