"""GPU parity of the D-matrix setup and the FFT matvec against the oracle
(MatVecCpu restated, DDA/MatVecCpu.cpp:67-150).  Tolerances: FP64 1e-12 and
FP32 2e-6, relative in the 2-norm of the result."""
import numpy as np
import pytest

from tests.pairs import Pair, aniso_arrays, scrambled_arrays, rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-6

CASES = {
    "aniso": ("arrays", aniso_arrays(), [1.5 + 0.1j, (1.33 + 0.01j, 1.4 + 0.02j, 1.6 + 0.0j)], "0.9um"),
    "scrambled": ("arrays", scrambled_arrays(), [1.5 + 0.1j, (1.33 + 0.01j, 1.4 + 0.02j, 1.6 + 0.0j)], "0.9um"),
    "sphere_small": ("sphere", ("1um", "0.1um"), [1.6 + 0.05j], "1.1um"),
    "cfg1": ("sphere", ("10um", "0.5um"), [1.5 + 0.1j], "6um"),
    "cylinder": ("cylinder", ("1.4um", "0.35um", "0.1um"), [2.0 + 0.3j], "1.5um"),
}


@pytest.mark.parametrize("case", ["aniso", "sphere_small", "cylinder"])
def test_dmatrix_generated_on_gpu(case):
    kind, args, mats, lam = CASES[case]
    pr = Pair(kind, args, mats, lam, "fp64")
    D = pr.mv.dmatrix()
    Do = pr.op.dmatrix()
    assert np.abs(D - Do).max() < 1e-12 * np.abs(Do).max()


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_matches_oracle(case, prec, tol):
    kind, args, mats, lam = CASES[case]
    pr = Pair(kind, args, mats, lam, prec)
    pr.set_cc((0.3, 0.4, 0.866), 2, "ldr")
    x = pr.rand_vec(11)
    y = pr.mv.apply(x)
    yo = pr.op.matvec(x)
    assert rel(y, yo) < tol
    # padding of the result is zeroed
    for c in range(3):
        assert not np.any(y[c * pr.p.nvs + pr.p.nv:(c + 1) * pr.p.nvs])
    yc = pr.mv.apply(x, conj=True)
    assert rel(yc, pr.op.matvec(x, conj=True)) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_split_yz_path(prec, tol):
    kind, args, mats, lam = CASES["aniso"]
    pr = Pair(kind, args, mats, lam, prec, flags=1)
    pr.set_cc((0, 0, 1), 1, "cm")
    x = pr.rand_vec(5)
    assert rel(pr.mv.apply(x), pr.op.matvec(x)) < tol


@pytest.mark.parametrize("flags", [0, 1, 2, 3, 4, 6])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_kernel_paths(flags, prec, tol):
    # README workload 1 (grid 80^3) has compile-time FFT plans; flags select
    # the split y/z path (1), the runtime-planned kernels (2) and the cluster
    # plane kernel (4).
    kind, args, mats, lam = CASES["cfg1"]
    pr = Pair(kind, args, mats, lam, prec, flags=flags)
    pr.set_cc((0, 0, 1), 2, "ldr")
    x = pr.rand_vec(17)
    assert rel(pr.mv.apply(x), pr.op.matvec(x)) < tol
    assert rel(pr.mv.apply(x, conj=True), pr.op.matvec(x, conj=True)) < tol


@pytest.mark.parametrize("case", ["aniso", "scrambled", "cylinder"])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_cluster_path_small_grids(case, prec, tol):
    # runtime-planned grids (odd sizes) through the cluster plane kernel
    kind, args, mats, lam = CASES[case]
    pr = Pair(kind, args, mats, lam, prec, flags=4)
    assert pr.mv.layout["yz_path"] == "cluster"
    pr.set_cc((0.6, 0.0, 0.8), 1, "ldr")
    x = pr.rand_vec(23)
    assert rel(pr.mv.apply(x), pr.op.matvec(x)) < tol
    assert rel(pr.mv.apply(x, conj=True), pr.op.matvec(x, conj=True)) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_plane_beyond_shared_memory(prec, tol):
    # sphere of radius 40 dipoles: grid 160^3, a kx plane (160 x 3 x 80
    # complex) does not fit one CTA, so the default path is the cluster
    # kernel; two right-hand sides with different couple constants
    pr = Pair("sphere", ("2um", "0.05um"), [1.5 + 0.1j], "1.2um", prec, max_rhs=2)
    assert pr.p.grid == (160, 160, 160)
    assert pr.mv.layout["yz_path"] == "cluster"
    xs = [pr.rand_vec(31), pr.rand_vec(32)]
    want = []
    for r, pol in enumerate((1, 2)):
        pr.set_cc((0, 0, 1), pol, "ldr", rhs=r)
        want.append(pr.op.matvec(xs[r]))
    y = pr.mv.apply(np.concatenate(xs))
    n = pr.p.vec_size
    for r in range(2):
        assert rel(y[r * n:(r + 1) * n], want[r]) < tol
    # one right-hand side of a two-rhs context
    assert rel(pr.mv.apply(xs[0]), want[0]) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_tuned_grid_matches_reference_grid(prec, tol):
    # box 35 x 40 x 45 with holes: reference grid 70 x 80 x 90 (runtime
    # plans), tuned grid 80 x 96 x 96 (compile-time plans, fused y/z); the
    # matvec restricted to the dipoles is the same linear convolution
    import dda_b200
    from oracle import oracle as O
    pos = np.array([(x, y, z) for z in range(45) for y in range(40) for x in range(35) if (x * 7 + y * 3 + z) % 11],
                   dtype=np.uint32)
    mat = np.zeros(len(pos), np.uint8)
    g = dda_b200.Geometry.from_arrays(pos, mat, "0.05um")
    p = dda_b200.DDAParams(g, [1.4 + 0.2j], "0.8um", grid_policy="tuned")
    assert p.grid == (80, 96, 96)
    mv = dda_b200.CudaMatVec(p, prec)
    assert mv.layout["compile_time_plans"] == 1
    og = O.Geometry.from_arrays(pos, mat, "0.05um")
    op = O.Problem(og, [1.4 + 0.2j], "0.8um")
    assert op.grid == (70, 80, 90)
    op.build_dmatrix()
    mv.set_couple_constants(dda_b200.CoupleConstants(p, (0.6, 0, 0.8), 2, "ldr"))
    op.set_cc((0.6, 0, 0.8), 2, "ldr")
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    assert rel(mv.apply(x), op.matvec(x)) < tol


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", ["box", "sphere"])
def test_autotuned_layout_gives_identical_results(prec, shape):
    # the autotuner changes only the batching of the y/z passes: the
    # product is bit-for-bit the same as with the default layout
    import dda_b200
    if shape == "box":  # grid 200 x 100 x 100, fused plane kernel
        g = dda_b200.Geometry.box_shape("5um", "2.5um", "2.5um", "0.05um")
    else:  # grid 160^3, cluster kernel
        g = dda_b200.Geometry.sphere("2um", "0.05um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1.2um")
    mvs = [dda_b200.CudaMatVec(p, prec, flags=f) for f in (0, 8)]
    for mv in mvs:
        mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr"))
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    assert np.array_equal(mvs[0].apply(x), mvs[1].apply(x))
    print(mvs[0].layout, mvs[1].layout)


@pytest.mark.parametrize("groups,pair", [(2, False), (4, False), (1, True), (2, True), (4, True)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["cfg1", "half", "aniso_tuned"])
def test_grouped_plane_kernel_is_identical(prec, case, groups, pair):
    # the fused plane kernel run as two groups of half the CTA (named
    # barriers, columns and row batches split between the groups) does the
    # same arithmetic per butterfly: bit-identical to one group, and equal to
    # the oracle
    import dda_b200
    from tests.pairs import Pair
    if case == "cfg1":  # grid 80^3, Plan<10,8>, not half padded
        kind, args, mats, lam = CASES["cfg1"]
    elif case == "half":  # box 40 x 24 x 24 on 80 x 48 x 48: the HALF variant
        pos = np.array([(x, y, z) for z in range(24) for y in range(24) for x in range(40) if (x + y + 2 * z) % 7],
                       dtype=np.uint32)
        kind, args, mats, lam = "arrays", (pos, np.zeros(len(pos), np.uint8), "0.05um"), [1.4 + 0.2j], "0.8um"
    else:  # 35 x 40 x 45 with holes on its tuned grid 80 x 96 x 96
        pos = np.array([(x, y, z) for z in range(45) for y in range(40) for x in range(35) if (x * 7 + y * 3 + z) % 11],
                       dtype=np.uint32)
        kind, args, mats, lam = "arrays", (pos, np.zeros(len(pos), np.uint8), "0.05um"), [1.4 + 0.2j], "0.8um"
    out = []
    # the same plane kernel with thread groups and/or as a two-CTA cluster
    # per plane (k_yz_pair: half the plane per CTA, exchanged through
    # distributed shared memory)
    gflag = {1: 0, 2: dda_b200.api.FLAG_YZ_GROUPS2, 4: dda_b200.api.FLAG_YZ_GROUPS4}[groups]
    gflag |= dda_b200.api.FLAG_YZ_PAIR if pair else 0
    for flags in (8, 8 | gflag):
        if case == "aniso_tuned":
            g = dda_b200.Geometry.from_arrays(*args)
            p = dda_b200.DDAParams(g, mats, lam, grid_policy="tuned")
            mv = dda_b200.CudaMatVec(p, prec, max_rhs=2, flags=flags)
            op = None
        else:
            pr = Pair(kind, args, mats, lam, prec, max_rhs=2, flags=flags)
            p, mv, op = pr.p, pr.mv, pr.op
        lay = mv.layout
        assert lay["yz_path"] == "fused" and lay["groups"] == (groups if flags & gflag else 1)
        assert lay["ctas_per_plane"] == (2 if pair and flags & gflag else 1)
        for r, pol in enumerate((1, 2)):
            mv.set_couple_constants(dda_b200.CoupleConstants(p, (0.6, 0.0, 0.8), pol, "ldr"), rhs=r)
        rng = np.random.default_rng(4)
        x = rng.uniform(-1, 1, 2 * p.vec_size) + 1j * rng.uniform(-1, 1, 2 * p.vec_size)
        for rr in range(2):
            for c in range(3):
                x[rr * p.vec_size + c * p.nvs + p.nv:rr * p.vec_size + (c + 1) * p.nvs] = 0
        out.append((mv.apply(x), mv.apply(x, conj=True)))
        if op is not None and flags & gflag:
            op.set_cc((0.6, 0.0, 0.8), 1, "ldr")
            assert rel(out[-1][0][:p.vec_size], op.matvec(x[:p.vec_size])) < (FP64_TOL if prec == "fp64" else FP32_TOL)
        mv.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
@pytest.mark.parametrize("flags,path", [(0, "fused"), (4, "cluster")])
def test_matvec_half_padded_box_matches_oracle(prec, tol, flags, path):
    # box 40 x 24 x 24 with holes on its own grid 80 x 48 x 48: y and z are
    # exactly twice the box, so the fused and the cluster plane kernels take
    # their variants with the zero half of the first FFT stage known at
    # compile time
    import dda_b200
    from oracle import oracle as O
    pos = np.array([(x, y, z) for z in range(24) for y in range(24) for x in range(40)
                    if (x * 5 + y * 3 + z) % 13 or (x, y, z) in ((39, 23, 23), (0, 0, 0))], dtype=np.uint32)
    mat = (pos[:, 1] % 2).astype(np.uint8)
    mats = [1.4 + 0.2j, 1.7 + 0.05j]
    g = dda_b200.Geometry.from_arrays(pos, mat, "0.05um")
    p = dda_b200.DDAParams(g, mats, "0.8um")
    assert p.grid == (80, 48, 48) and p.box == (40, 24, 24)
    mv = dda_b200.CudaMatVec(p, prec, flags=flags)
    assert mv.layout["yz_path"] == path and mv.layout["compile_time_plans"] == 1
    og = O.Geometry.from_arrays(pos, mat, "0.05um")
    op = O.Problem(og, mats, "0.8um")
    op.build_dmatrix()
    mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0.6, 0.8), 1, "ldr"))
    op.set_cc((0, 0.6, 0.8), 1, "ldr")
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    assert rel(mv.apply(x), op.matvec(x)) < tol
    mv.close()


def test_x_tile_fills_whole_waves():
    # the x-pass tile is chosen by the count of CTA waves: for the 250 000
    # dipole box (2 500 grid lines, grid x 200) with two right-hand sides in
    # FP32 both x passes take one wave of at most three CTAs per SM
    import torch
    import dda_b200
    g = dda_b200.Geometry.box_shape("10um", "5um", "5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    mv = dda_b200.CudaMatVec(p, "fp32", max_rhs=2)
    tl = mv.layout["lines_per_x_tile"]
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    tmax = min(64, 73728 // (8 * 201))
    assert tmax // 2 <= tl <= tmax
    assert -(-2500 // tl) * 3 * 2 <= 3 * nsm
    mv.close()


def test_matvec_host_dmatrix():
    kind, args, mats, lam = CASES["aniso"]
    pr = Pair(kind, args, mats, lam, "fp64", host_d=True)
    pr.set_cc((0, 1, 0), 1, "ldr")
    x = pr.rand_vec(8)
    assert rel(pr.mv.apply(x), pr.op.matvec(x)) < FP64_TOL


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_batched_rhs(prec, tol):
    kind, args, mats, lam = CASES["sphere_small"]
    pr = Pair(kind, args, mats, lam, prec, max_rhs=3)
    props = [((0, 0, 1), 1), ((0, 1, 0), 2), ((0.6, 0, 0.8), 1)]
    xs, ys = [], []
    for r, (prop, pol) in enumerate(props):
        pr.set_cc(prop, pol, "ldr", rhs=r)
        x = pr.rand_vec(20 + r)
        xs.append(x)
        ys.append(pr.op.matvec(x))
    y = pr.mv.apply(np.concatenate(xs)).reshape(3, -1)
    for r in range(3):
        assert rel(y[r], ys[r]) < tol
    # one rhs alone gives the same bits as inside the batch
    y0 = pr.mv.apply(xs[0])
    assert np.array_equal(y0, y[0])


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_matvec_cfg2_box(prec, tol):
    # README workload 2: box 10x5x5 um, d = 0.1 um, grid 200x100x100.  The FP64
    # kx plane (240 KB) exceeds shared memory, so this exercises the split path.
    pr = Pair("box", ("10um", "5um", "5um", "0.1um"), [1.5 + 0.1j], "6um", prec)
    pr.set_cc((0, 1, 0), 1, "ldr")
    x = pr.rand_vec(3)
    assert rel(pr.mv.apply(x), pr.op.matvec(x)) < tol


def test_matvec_device_pointers():
    torch = pytest.importorskip("torch")
    kind, args, mats, lam = CASES["sphere_small"]
    pr = Pair(kind, args, mats, lam, "fp32")
    pr.set_cc((0, 0, 1), 1, "ldr")
    x = pr.rand_vec(2)
    xd = torch.from_numpy(x.astype(np.complex64)).cuda()
    yd = torch.zeros_like(xd)
    pr.mv.apply_device(xd.data_ptr(), yd.data_ptr(), nrhs=1)
    pr.mv.synchronize()
    assert rel(yd.cpu().numpy(), pr.op.matvec(x)) < FP32_TOL
