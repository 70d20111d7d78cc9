"""The request loop on the GPU: results of requests solved together equal
their results solved alone, cross sections equal the direct API's, and
admission keeps to the HBM budget."""
import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess as PP
from dda_b200 import targets
from dda_b200.serve import Server

pytestmark = pytest.mark.gpu


def _requests(n, seed, edges=(6, 16)):
    rng = np.random.default_rng(seed)
    return [targets.served_request(rng, edges) for _ in range(n)]


def _submit(srv, r, tag, **kw):
    return srv.submit(r["positions"], r["materials"], r["refr"], r["grid_unit"], r["wavelength"],
                      prop=r["prop"], tag=tag, **kw)


def test_results_same_alone_and_in_the_mix():
    reqs = _requests(8, 11)
    mix = Server(max_active=4)
    for i, r in enumerate(reqs):
        _submit(mix, r, i, keep_pol=True)
    together = {d["tag"]: d for d in mix.drain()}
    mix.close()
    # overlap actually happened: some request was admitted before another finished
    spans = sorted((d["t_admit"], d["t_done"]) for d in together.values())
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    alone = Server(max_active=1)
    for i, r in enumerate(reqs):
        _submit(alone, r, i, keep_pol=True)
        (d,) = alone.drain()
        t = together[i]
        assert d["status"] == 0 and t["status"] == 0, (d["error"], t["error"])
        assert d["iterations"] == t["iterations"]
        assert np.array_equal(d["pol"], t["pol"])
        assert d["cext"] == t["cext"] and d["cabs"] == t["cabs"]
        assert max(t["rel_residual"]) <= 1e-5
    alone.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_served_request_matches_direct_api(precision):
    rng = np.random.default_rng(5)
    r = targets.served_request(rng, (10, 12))
    srv = Server(max_active=2)
    _submit(srv, r, 7, keep_pol=True, precision=precision, solver="bicgstab")
    (d,) = srv.drain()
    srv.close()
    assert d["status"] == 0, d["error"]
    g = dda_b200.Geometry.from_arrays(r["positions"], np.zeros(len(r["positions"]), np.uint8), r["grid_unit"])
    p = dda_b200.DDAParams(g, r["refr"], r["wavelength"])
    mv = dda_b200.CudaMatVec(p, precision, max_rhs=2)
    ccs = []
    for k, pol in enumerate((1, 2)):
        ccs.append(dda_b200.CoupleConstants(p, r["prop"], pol, "ldr"))
        mv.set_couple_constants(ccs[-1], rhs=k)
    einc = np.stack([p.einc(r["prop"], 1), p.einc(r["prop"], 2)])
    pol = dda_b200.CudaSolver(mv, "bicgstab").get_pol_vec(einc, 1e-5)
    assert np.array_equal(pol, d["pol"])
    for k, polno in enumerate((1, 2)):
        _, pn = dda_b200.beam_pol(r["prop"], 1)
        ef = mv.far_field(pn[None, :], nrhs=2)[0, k]
        cext, cabs, _, _ = PP.cross_sections(p, ccs[k], pol[k], ef, r["prop"], polno)
        assert abs(cext - d["cext"][k]) <= 1e-12 * abs(cext)
        assert abs(cabs - d["cabs"][k]) <= 1e-12 * abs(cabs)
    assert d["device_bytes"] <= d["footprint"]


def test_budget_admits_one_at_a_time():
    # one target under four incidences: equal footprints, and a budget of
    # 1.5 footprints admits one request at a time
    base = _requests(1, 21)[0]
    rng = np.random.default_rng(22)
    reqs = [dict(base, prop=tuple(targets.random_direction(rng))) for _ in range(4)]
    probe = Server(max_active=1)
    _submit(probe, reqs[0], 0)
    (d0,) = probe.drain()
    probe.close()
    srv = Server(budget_bytes=int(d0["footprint"] * 1.5), max_active=4)
    for i, r in enumerate(reqs):
        _submit(srv, r, i)
    res = srv.drain()
    srv.close()
    assert all(d["status"] == 0 for d in res)
    spans = sorted((d["t_admit"], d["t_done"]) for d in res)
    for a, b in zip(spans, spans[1:]):
        assert b[0] >= a[1]


def test_request_beyond_budget_is_rejected():
    r = _requests(1, 31)[0]
    srv = Server(budget_bytes=1 << 20, max_active=1)
    with pytest.raises(dda_b200.DDAError) as e:
        _submit(srv, r, 0)
    assert "exceeds the budget" in str(e.value)
    srv.close()
