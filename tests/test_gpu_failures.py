"""Failure detection on the host side, with no fault on the GPU.

The failures are made on the host: incident fields with NaN or zero
entries, an incidence whose bilinear residual product vanishes (the
BiCG-CS rho guard of DDA/BicgCs.cpp:65-74 fires, as in the oracle), a cancel
request from another thread, and a failing request in the middle of the
request loop.  Every case ends with a defined status, and the context (or
the server) stays usable: later solves give the same bits as on a fresh
context."""
import threading
import time

import numpy as np
import pytest

import dda_b200
from dda_b200 import targets
from dda_b200.serve import Server
from tests.pairs import Pair, aniso_arrays

pytestmark = pytest.mark.gpu

MATS = [1.5 + 0.1j, (1.33 + 0.01j, 1.4 + 0.02j, 1.6 + 0.0j)]


def _problem(prec, max_rhs=2):
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", prec, max_rhs=max_rhs, oracle_d=False)
    es = []
    for r, (prop, pol) in enumerate([((0.3, 0.4, 0.866), 1), ((0, 1, 0), 2)][:max_rhs]):
        pr.set_cc(prop, pol, "ldr", rhs=r)
        es.append(pr.p.einc(prop, pol))
    return pr, es


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_nan_incident_field_fails_alone(prec):
    pr, es = _problem(prec)
    s = dda_b200.CudaSolver(pr.mv, "qmr")
    bad = es[0].copy()
    bad[3] = np.nan
    t0 = time.time()
    with pytest.raises(dda_b200.DDAError) as ei:
        s.get_pol_vec(np.concatenate([bad, es[1]]), 1e-8)
    assert ei.value.code == -1 and time.time() - t0 < 30
    st = s.last_stats
    assert st[0].status == -1 and st[0].iterations == 0
    assert st[1].status == 0 and st[1].rel_residual < 1e-8
    # the device entry point reports the same
    import torch
    dt = torch.complex128 if prec != "fp32" else torch.complex64
    e_dev = torch.from_numpy(np.concatenate([bad, es[1]])).to(dt).cuda()
    p_dev = torch.zeros_like(e_dev)
    torch.cuda.synchronize()
    rc = s.get_pol_vec_device(e_dev.data_ptr(), p_dev.data_ptr(), 2, 1e-8, raise_on_error=False)
    assert rc == -1 and s.last_stats[0].status == -1 and s.last_stats[1].status == 0
    # the context is still usable: a clean two-rhs solve gives a fresh
    # context's bits
    both = s.get_pol_vec(np.concatenate(es), 1e-8)
    pr2, _ = _problem(prec)
    ref = dda_b200.CudaSolver(pr2.mv, "qmr").get_pol_vec(np.concatenate(es), 1e-8)
    assert np.array_equal(both, ref)
    with pytest.raises(dda_b200.DDAError) as ei:
        pr.mv.set_couple_constants(np.full(len(MATS) * 3, np.nan + 0j))
    assert ei.value.code == -1


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_zero_incident_field_gives_zero_polarisation(prec):
    pr, es = _problem(prec, max_rhs=1)
    s = dda_b200.CudaSolver(pr.mv, "bicgstab")
    pol = s.get_pol_vec(np.zeros_like(es[0]), 1e-6)
    assert s.last_stats[0].status == 0 and s.last_stats[0].iterations == 0
    assert not np.any(pol)


def test_bicg_rho_breakdown_matches_oracle():
    # Clausius-Mossotti constants of a real index are real; an incident
    # field (a, i a, 0) then has r.r = 0 in the bilinear product of
    # BiCG-CS (DDA/BicgCs.cpp:65-74), whose rho guard fires on the first
    # iteration.  Start value 0, so r0 = b.
    pr = Pair("arrays", aniso_arrays(), [1.5, 1.5], "0.9um", "fp64")
    pr.set_cc((0, 0, 1), 1, "cm")
    n, nv, nvs = pr.p.vec_size, pr.p.nv, pr.p.nvs
    e = np.zeros(n, dtype=np.complex128)
    a = np.linspace(0.5, 1.5, nv)
    e[:nv] = a
    e[nvs:nvs + nv] = 1j * a
    zero = np.zeros(n, dtype=np.complex128)
    rc_o, _, st_o, _ = pr.op.solve(e, "bicg", 1e-8, start=zero)
    s = dda_b200.CudaSolver(pr.mv, "bicg")
    with pytest.raises(dda_b200.DDAError) as ei:
        s.get_pol_vec(e, 1e-8, start=zero)
    assert rc_o == -5 and ei.value.code == -5
    assert s.last_stats[0].iterations == st_o.iterations == 0


def test_cancel_stops_a_running_solve():
    g = dda_b200.Geometry.sphere("10um", "0.5um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    mv = dda_b200.CudaMatVec(p, "fp64", max_rhs=1)
    mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr"))
    e = p.einc((0, 0, 1), 1)
    # QMR-CS to an unreachable target: the residual stagnates at rounding
    # level and the solve would only end after 50 000 iterations without
    # improvement (DDA/IterativeSolverBase.cpp:62-64), minutes from now
    s = dda_b200.CudaSolver(mv, "qmr", max_iter=10 ** 7)
    box = {}

    def run():
        t0 = time.time()
        try:
            s.get_pol_vec(e, 1e-300)
        except dda_b200.DDAError as ex:
            box["code"] = ex.code
        box["t"] = time.time() - t0

    th = threading.Thread(target=run)
    th.start()
    time.sleep(1.0)
    t_cancel = time.time()
    mv.cancel()
    th.join(60)
    assert not th.is_alive()
    assert box["code"] == -8 and s.last_stats[0].status == -8
    assert s.last_stats[0].iterations > 8
    assert time.time() - t_cancel < 5
    # the cancel request is consumed: the next solve runs normally and
    # gives a fresh context's bits
    s2 = dda_b200.CudaSolver(mv, "bicgstab")
    pol = s2.get_pol_vec(e, 1e-6)
    mv2 = dda_b200.CudaMatVec(p, "fp64", max_rhs=1)
    mv2.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr"))
    assert np.array_equal(pol, dda_b200.CudaSolver(mv2, "bicgstab").get_pol_vec(e, 1e-6))


def _requests(n):
    rng = np.random.default_rng(5)
    return [targets.served_request(rng, (16, 28)) for _ in range(n)]


def _submit(srv, r, **kw):
    return srv.submit(r["positions"], r["materials"], r["refr"], r["grid_unit"], r["wavelength"],
                      prop=r["prop"], keep_pol=True, **kw)


def test_failing_request_fails_alone_in_the_mix():
    reqs = _requests(8)
    bad = 3
    reqs[bad] = dict(reqs[bad], refr=[complex(np.nan, 0.0)] * len(reqs[bad]["refr"]))
    alone = {}
    srv = Server(max_active=1)
    for i, r in enumerate(reqs):
        if i == bad:
            continue
        _submit(srv, r, tag=i)
        res = srv.drain()
        assert len(res) == 1 and res[0]["status"] == 0
        alone[i] = res[0]["pol"]
    srv.close()
    srv = Server(max_active=4)
    for i, r in enumerate(reqs):
        _submit(srv, r, tag=i)
    res = {x["tag"]: x for x in srv.drain()}
    srv.close()
    assert len(res) == 8
    assert res[bad]["status"] == -1 and "not finite" in res[bad]["error"]
    for i in alone:
        assert res[i]["status"] == 0
        assert np.array_equal(res[i]["pol"], alone[i])


def test_serve_cancel_queued_and_running():
    reqs = _requests(4)
    srv = Server(max_active=1)
    # request 0 cannot converge (eps far below rounding) and runs until cancelled
    r0 = _submit(srv, reqs[0], tag=0, eps=1e-300, solver="qmr", precision="fp64", max_iter=10 ** 7)
    ids = [r0] + [_submit(srv, r, tag=i + 1) for i, r in enumerate(reqs[1:])]
    srv.cancel(ids[2])  # still queued behind request 0
    time.sleep(1.0)
    srv.cancel(ids[0])  # running
    res = {x["tag"]: x for x in srv.drain()}
    assert res[2]["status"] == -8 and "before admission" in res[2]["error"]
    assert res[0]["status"] == -8
    assert res[1]["status"] == 0 and res[3]["status"] == 0
    with pytest.raises(dda_b200.DDAError):
        srv.cancel(ids[1])  # finished: neither queued nor running
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_single_dipole(prec):
    # one dipole (box 1x1x1, grid 2^3, runtime-planned FFTs): no interaction,
    # A = I, so the solve ends at once with the oracle's polarisation
    import dda_b200
    from oracle import oracle as O
    g = dda_b200.Geometry.from_arrays(np.zeros((1, 3), np.uint32), np.zeros(1, np.uint8), "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    op = O.Problem(O.Geometry.from_arrays(np.zeros((1, 3), np.uint32), np.zeros(1, np.uint8), "0.1um"),
                   [1.5 + 0.1j], "1um")
    op.build_dmatrix()
    mv = dda_b200.CudaMatVec(p, prec, max_rhs=2)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), pol, "ldr"), rhs=r)
    e = np.stack([p.einc((0, 0, 1), pol) for pol in (1, 2)])
    x = np.random.default_rng(3).normal(size=p.vec_size) + 0j
    x.reshape(3, p.nvs)[:, 1:] = 0
    y = mv.apply(x)
    assert np.allclose(y, x, rtol=0, atol=1e-6 if prec == "fp32" else 1e-14)  # A = I
    pol = dda_b200.CudaSolver(mv, "qmr").get_pol_vec(e, 1e-8)
    for r, pv in enumerate((1, 2)):
        op.set_cc((0, 0, 1), pv, "ldr")
        rc, want, _, _ = op.solve(e[r], "qmr", 1e-8)
        assert rc == 0
        assert np.linalg.norm(pol[r] - want) <= (1e-6 if prec == "fp32" else 1e-12) * np.linalg.norm(want)
    mv.close()


@pytest.mark.gpu
def test_argument_and_size_checks():
    # the context and solve entry points reject what they cannot run with a
    # code and a message, before any device work: grids that are odd, smaller
    # than twice the box, not 2,3,5,7-smooth or above the 4096 edge limit;
    # more right-hand sides than the context holds, a solve before its couple
    # constants, a non-positive tolerance
    import dda_b200
    from dda_b200.api import DDAError
    g = dda_b200.Geometry.box_shape("0.5um", "0.4um", "0.3um", "0.1um")
    cases = [((11, 8, 6), -1, "even"), ((8, 8, 6), -1, "twice"), ((22, 8, 6), -4, "smooth"),
             ((4098, 8, 6), -4, "4096")]
    for grid, code, words in cases:
        p = dda_b200.DDAParams(g, [1.5], "1um", grid=grid)
        with pytest.raises(DDAError) as ei:
            dda_b200.CudaMatVec(p, "fp32")
        assert ei.value.code == code and words in str(ei.value), (grid, str(ei.value))
    p = dda_b200.DDAParams(g, [1.5], "1um")
    mv = dda_b200.CudaMatVec(p, "fp32", max_rhs=1)
    s = dda_b200.CudaSolver(mv, "qmr")
    e = p.einc((0, 0, 1), 1)
    with pytest.raises(DDAError, match="couple constants"):
        s.get_pol_vec(e, 1e-5)
    mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr"))
    with pytest.raises(DDAError) as ei:
        s.get_pol_vec(np.stack([e, e]), 1e-5)  # two rhs on a one-rhs context
    assert ei.value.code == -1
    with pytest.raises(DDAError, match="eps"):
        s.get_pol_vec(e, 0.0)
    assert np.all(np.isfinite(s.get_pol_vec(e, 1e-5)))  # the context still works
    mv.close()
