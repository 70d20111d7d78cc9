"""GPU parity of the four Krylov solvers against the oracle's restatement of
the reference CPU solvers (DDA/QmrCs.cpp, DDA/BicgStab.cpp, DDA/BicgCs.cpp,
DDA/Cgnr.cpp, loop of DDA/IterativeSolverBase.cpp:40-103)."""
import numpy as np
import pytest

import dda_b200
from tests.pairs import Pair, aniso_arrays, rel

pytestmark = pytest.mark.gpu

SOLVERS = ["qmr", "bicgstab", "bicg", "cgnr"]
MATS = [1.5 + 0.1j, (1.33 + 0.01j, 1.4 + 0.02j, 1.6 + 0.0j)]


@pytest.fixture(scope="module")
def aniso64():
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", "fp64")
    pr.set_cc((0.3, 0.4, 0.866), 1, "ldr")
    return pr


@pytest.mark.parametrize("solver", SOLVERS)
def test_fp64_solver_tracks_oracle(aniso64, solver):
    pr = aniso64
    e = pr.p.einc((0.3, 0.4, 0.866), 1)
    s = dda_b200.CudaSolver(pr.mv, solver)
    pol = s.get_pol_vec(e, 1e-10)
    rc, opol, ost, ohist = pr.op.solve(e, solver, 1e-10)
    assert rc == 0
    st = s.last_stats[0]
    assert st.status == 0 and st.rel_residual < 1e-10
    assert abs(st.iterations - ost.iterations) <= 1
    h = s.last_history[0]
    k = min(len(h), len(ohist), 8)
    assert np.allclose(h[:k], ohist[:k], rtol=1e-8, atol=0)
    assert rel(pol, opol) < 1e-8


@pytest.mark.parametrize("solver", SOLVERS)
def test_fp32_solver_converges(aniso64, solver):
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", "fp32")
    pr.set_cc((0.3, 0.4, 0.866), 1, "ldr")
    e = pr.p.einc((0.3, 0.4, 0.866), 1)
    s = dda_b200.CudaSolver(pr.mv, solver)
    pol = s.get_pol_vec(e, 1e-5)
    assert s.last_stats[0].status == 0
    rc, opol, _, _ = pr.op.solve(e, solver, 1e-9)
    assert rel(pol, opol) < 1e-4


def test_fp32_host_path_matches_device_path():
    # dda_solve converts the host FP64 fields to FP32 on the device (rounding
    # to nearest, as a host cast does) and the polarisations back: the result
    # is the device-resident solve's, bit for bit, also into a pinned buffer
    import torch
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", "fp32")
    pr.set_cc((0.3, 0.4, 0.866), 1, "ldr")
    e = np.ascontiguousarray(pr.p.einc((0.3, 0.4, 0.866), 1).reshape(-1))
    s = dda_b200.CudaSolver(pr.mv, "bicgstab")
    out = torch.empty(e.size, dtype=torch.complex128, pin_memory=True).numpy()
    pol = s.get_pol_vec(e, 1e-5, out=out)
    assert pol is out and s.last_stats[0].status == 0
    paged = s.get_pol_vec(e, 1e-5)
    assert np.array_equal(paged, out)
    ed = torch.from_numpy(e).to(torch.complex64).cuda()
    pd = torch.zeros_like(ed)
    torch.cuda.synchronize()
    s.get_pol_vec_device(ed.data_ptr(), pd.data_ptr(), 1, 1e-5)
    assert np.array_equal(pd.cpu().numpy().astype(np.complex128), out)
    with pytest.raises(ValueError):
        s.get_pol_vec(e, 1e-5, out=np.zeros(e.size, dtype=np.complex64))


def test_cfg1_qmr_fp64_iterations():
    # README workload 1: sphere r = 10 um, d = 0.5 um, m = 1.5+0.1i, 6 um, QMR, 1e-5
    pr = Pair("sphere", ("10um", "0.5um"), [1.5 + 0.1j], "6um", "fp64")
    pr.set_cc((0, 0, 1), 1, "ldr")
    e = pr.p.einc((0, 0, 1), 1)
    s = dda_b200.CudaSolver(pr.mv, "qmr")
    pol = s.get_pol_vec(e, 1e-5)
    rc, opol, ost, ohist = pr.op.solve(e, "qmr", 1e-5)
    st = s.last_stats[0]
    assert st.status == 0 and abs(st.iterations - ost.iterations) <= 2
    assert np.allclose(s.last_history[0][:20], ohist[:20], rtol=1e-7)
    assert rel(pol, opol) < 1e-5


def test_batched_solve_equals_single(aniso64):
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", "fp64", max_rhs=2)
    cases = [((0.3, 0.4, 0.866), 1), ((0, 1, 0), 2)]
    es = []
    for r, (prop, pol) in enumerate(cases):
        pr.set_cc(prop, pol, "ldr", rhs=r)
        es.append(pr.p.einc(prop, pol))
    s = dda_b200.CudaSolver(pr.mv, "bicgstab")
    both = s.get_pol_vec(np.concatenate(es), 1e-8).reshape(2, -1)
    it_both = [st.iterations for st in s.last_stats]
    # rhs 0 alone (same context, cc slot 0) reproduces the batched bits
    one = s.get_pol_vec(es[0], 1e-8)
    assert s.last_stats[0].iterations == it_both[0]
    assert np.array_equal(one, both[0])


def test_start_value(aniso64):
    pr = aniso64
    e = pr.p.einc((0.3, 0.4, 0.866), 1)
    s = dda_b200.CudaSolver(pr.mv, "qmr")
    pol = s.get_pol_vec(e, 1e-6)
    s2 = dda_b200.CudaSolver(pr.mv, "qmr")
    pol2 = s2.get_pol_vec(e, 1e-9, start=pol)
    rc, opol, ost, _ = pr.op.solve(e, "qmr", 1e-9, start=pol)
    assert rc == 0 and abs(s2.last_stats[0].iterations - ost.iterations) <= 1
    assert rel(pol2, opol) < 1e-8


def test_max_iter_reports_error(aniso64):
    pr = aniso64
    e = pr.p.einc((0.3, 0.4, 0.866), 1)
    s = dda_b200.CudaSolver(pr.mv, "qmr", max_iter=3)
    with pytest.raises(dda_b200.DDAError) as ei:
        s.get_pol_vec(e, 1e-10)
    assert ei.value.code == -6
    assert s.last_stats[0].iterations == 3


@pytest.mark.parametrize("solver", ["qmr", "bicgstab"])
def test_mixed_refinement_reaches_fp64_accuracy(solver):
    # FP32 inner solves refined by FP64 residuals reach residuals FP32 alone cannot
    pr = Pair("arrays", aniso_arrays(), MATS, "0.9um", "mixed")
    pr.set_cc((0.3, 0.4, 0.866), 1, "ldr")
    e = pr.p.einc((0.3, 0.4, 0.866), 1)
    s = dda_b200.CudaSolver(pr.mv, solver)
    pol = s.get_pol_vec(e, 1e-9)
    st = s.last_stats[0]
    assert st.status == 0 and st.rel_residual < 1e-9 and st.refinements >= 2
    rc, opol, _, _ = pr.op.solve(e, solver, 1e-11)
    assert rel(pol, opol) < 1e-7


def test_mixed_cfg1_both_pols_batched():
    pr = Pair("sphere", ("10um", "0.5um"), [1.5 + 0.1j], "6um", "mixed", max_rhs=2)
    es = []
    for r, pol in enumerate((1, 2)):
        pr.set_cc((0, 0, 1), pol, "ldr", rhs=r)
        es.append(pr.p.einc((0, 0, 1), pol))
    s = dda_b200.CudaSolver(pr.mv, "qmr")
    pol = s.get_pol_vec(np.concatenate(es), 1e-5).reshape(2, -1)
    for r, p in enumerate((1, 2)):
        assert s.last_stats[r].status == 0 and s.last_stats[r].rel_residual < 1e-5
        pr.op.set_cc((0, 0, 1), p, "ldr")
        rc, opol, _, _ = pr.op.solve(es[r], "qmr", 1e-7)
        assert rel(pol[r], opol) < 2e-5


@pytest.mark.parametrize("solver", ["qmr", "bicgstab", "bicg", "cgnr"])
@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_graph_replay_gives_identical_solutions(solver, prec):
    # rounds of eight iterations replayed from a captured CUDA graph run the
    # same kernels in the same order as launching them one by one
    import dda_b200
    g = dda_b200.Geometry.sphere("10um", "0.5um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    out = []
    for flags in (0, 16):
        mv = dda_b200.CudaMatVec(p, prec, max_rhs=2, flags=flags)
        for r, pol in enumerate((1, 2)):
            mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), pol, "ldr"), rhs=r)
        s = dda_b200.CudaSolver(mv, solver, max_iter=400)
        einc = np.stack([p.einc((0, 0, 1), 1), p.einc((0, 0, 1), 2)])
        pol = s.get_pol_vec(einc, 1e-6, raise_on_error=False)
        out.append((pol, [(x.iterations, x.status) for x in s.last_stats]))
        mv.close()
    assert out[0][1] == out[1][1]
    assert max(it for it, _ in out[0][1]) > 16  # replayed rounds were used
    assert np.array_equal(out[0][0], out[1][0])


def test_fp32_bench_solution_meets_tolerance_in_fp64():
    # the default benchmark solves in FP32 (complex64 vectors, FP64 scalars)
    # and stops on the recurrence residual; the FP64 residual of its answer
    # must meet the same 1e-5
    import dda_b200
    g = dda_b200.Geometry.box_shape("10um", "5um", "5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    prop = (0.0, 1.0, 0.0)
    mv32 = dda_b200.CudaMatVec(p, "fp32", max_rhs=2)
    mv64 = dda_b200.CudaMatVec(p, "fp64")
    ccs = []
    for r, pol in enumerate((1, 2)):
        ccs.append(dda_b200.CoupleConstants(p, prop, pol, "ldr"))
        mv32.set_couple_constants(ccs[-1], rhs=r)
    einc = np.stack([p.einc(prop, 1), p.einc(prop, 2)])
    P = dda_b200.CudaSolver(mv32, "bicgstab").get_pol_vec(einc, 1e-5)
    mat = p.geometry.materials.astype(np.int64)
    for r in range(2):
        mv64.set_couple_constants(ccs[r])
        cs = np.zeros(p.vec_size, dtype=np.complex128)
        for c in range(3):
            cs[c * p.nvs:c * p.nvs + p.nv] = ccs[r].cc_sqrt[mat * 3 + c]
        live = cs != 0
        x = np.zeros_like(P[r])
        x[live] = P[r][live] / cs[live]
        b = cs * einc[r]
        res = np.linalg.norm(b - mv64.apply(x)) / np.linalg.norm(b)
        assert res < 1e-5, res
