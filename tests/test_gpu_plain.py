"""The straightforward FP64 baseline of the benchmark (bench_plain.py) solves
the same system as the library."""
import numpy as np
import pytest

import dda_b200

pytestmark = pytest.mark.gpu


def test_plain_baseline_matches_library_solution():
    import bench_plain
    g = dda_b200.Geometry.sphere("10um", "0.5um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    mv = dda_b200.CudaMatVec(p, "fp64")
    cc = dda_b200.CoupleConstants(p, (0, 1, 0), 1, "ldr")
    mv.set_couple_constants(cc)
    e = p.einc((0, 1, 0), 1)
    want = dda_b200.CudaSolver(mv, "bicgstab").get_pol_vec(e, 1e-9)
    sp = bench_plain.PlainSolver(mv, p, cc.cc_sqrt)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    import torch
    y = sp.matvec(torch.from_numpy(x).cuda()).cpu().numpy()
    yl = mv.apply(x)
    assert np.linalg.norm(y - yl) / np.linalg.norm(yl) < 1e-12
    got, its = sp.solve(e, 1e-9)
    got = got.cpu().numpy()
    assert its > 5
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-7


def test_plain_qmr_matches_library_solution():
    import bench_plain
    g = dda_b200.Geometry.sphere("10um", "0.5um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    mv = dda_b200.CudaMatVec(p, "fp64")
    cc = dda_b200.CoupleConstants(p, (0, 0, 1), 2, "ldr")
    mv.set_couple_constants(cc)
    e = p.einc((0, 0, 1), 2)
    s = dda_b200.CudaSolver(mv, "qmr")
    want = s.get_pol_vec(e, 1e-9)
    got, its = bench_plain.PlainSolver(mv, p, cc.cc_sqrt).solve_qmr(e, 1e-9)
    got = got.cpu().numpy()
    assert abs(its - s.last_stats[0].iterations) <= 2
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-7
