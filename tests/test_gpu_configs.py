"""GPU parity on the shapes of the benchmark workloads, against the oracle.

* the 128-rhs spheroid's grid (192 x 128 x 128, fused half-padded plane
  kernel) on four right-hand sides with their own LDR couple constants;
* the 512^3 sphere's grid through its production path (cluster plane kernel,
  compile-time 512-point plans), against the oracle's matvec and against the
  split y/z path of the same context shape;
* the README sphere (cfg1) Jones matrices on the --efield-grid angle set of
  the reference (theta 0..180/91, phi 0..360/61, DDA/DDAMain.cpp:346-347)
  from FP32 and mixed-precision solves against the oracle's FP64 solve, with
  the normalised RMS difference of DDA/FieldDiff.cpp:192;
* the README box (cfg2) FP32 benchmark solution against the oracle's FP64
  system and solution.

Tolerances: matvec FP64 1e-12, FP32 2e-6 (relative 2-norm); Jones 1e-4
(FieldDiff); solutions at relative residual 1e-5.
"""
import math

import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess as PP
from dda_b200 import targets
from oracle import oracle as O
from tests.pairs import rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-6
SEED = 20261203


def _cc_vector(p, cc):
    """sqrt(cc) per vector entry ([x: nvs][y: nvs][z: nvs]); 0 on padding."""
    mat = p.geometry.materials.astype(np.int64)
    cs = np.zeros(p.vec_size, dtype=np.complex128)
    for c in range(3):
        cs[c * p.nvs:c * p.nvs + p.nv] = cc.cc_sqrt[mat * 3 + c]
    return cs


# ------------------------------------------------------------ spheroid ----
@pytest.fixture(scope="module")
def spheroid_oracle():
    d_um = 0.05
    kd = 15.0 / (48 * 32 * 32) ** (1.0 / 3)
    lam = "%.17gum" % (2 * math.pi * d_um / kd)
    pos = targets.spheroid(48, 32, 32)
    mat = np.zeros(len(pos), np.uint8)
    og = O.Geometry.from_arrays(pos, mat, "%gum" % d_um)
    op = O.Problem(og, [1.33 + 0.01j], lam)
    op.build_dmatrix()
    rng = np.random.default_rng(SEED)
    dirs = rng.normal(size=(2, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rhs = [(tuple(dirs[r // 2]), 1 + r % 2) for r in range(4)]
    return pos, mat, "%gum" % d_um, lam, op, rhs


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_spheroid_block_matvec_matches_oracle(spheroid_oracle, prec, tol):
    pos, mat, gu, lam, op, rhs = spheroid_oracle
    g = dda_b200.Geometry.from_arrays(pos, mat, gu)
    p = dda_b200.DDAParams(g, [1.33 + 0.01j], lam)
    assert p.grid == (192, 128, 128) and p.box == (96, 64, 64)
    mv = dda_b200.CudaMatVec(p, prec, max_rhs=4)
    # FP32: the fused half-padded plane kernel in one CTA; FP64: the plane
    # (395 KB) is beyond one CTA's shared memory, so two CTAs share it
    lay = mv.layout
    assert lay["yz_path"] == "fused" and lay["ctas_per_plane"] == (1 if prec == "fp32" else 2)
    rng = np.random.default_rng(3)
    xs, want = [], []
    for r, (prop, pol) in enumerate(rhs):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
        x = rng.uniform(-1, 1, p.vec_size) + 1j * rng.uniform(-1, 1, p.vec_size)
        for c in range(3):
            x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
        xs.append(x)
        op.set_cc(prop, pol, "ldr")
        want.append(op.matvec(x))
    y = mv.apply(np.concatenate(xs)).reshape(4, -1)
    for r in range(4):
        assert rel(y[r], want[r]) < tol, (r, rel(y[r], want[r]))
    mv.close()


# --------------------------------------------------------- 512^3 sphere ----
@pytest.fixture(scope="module")
def sphere512():
    g = dda_b200.Geometry.sphere("12.8um", "0.1um")
    p = dda_b200.DDAParams(g, [1.6 + 0.01j], "1.3404um")
    assert p.grid == (512, 512, 512) and p.nv == 8783848
    x = np.random.default_rng(41).uniform(-1, 1, p.vec_size) + 0j
    x.imag = np.random.default_rng(42).uniform(-1, 1, p.vec_size)
    for c in range(3):
        x[c * p.nvs + p.nv:(c + 1) * p.nvs] = 0
    return p, x


@pytest.fixture(scope="module")
def sphere512_oracle(sphere512):
    """The oracle's matvec of the 512^3 sphere (FP64, all host threads; the
    D matrix alone is 12.9 GB of host memory)."""
    p, x = sphere512
    og = O.Geometry.sphere("12.8um", "0.1um")
    op = O.Problem(og, [1.6 + 0.01j], "1.3404um")
    op.build_dmatrix()
    op.set_cc((0, 0, 1), 1, "ldr")
    y = op.matvec(x)
    del op
    return y


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_sphere512_cluster_matvec_matches_oracle(sphere512, sphere512_oracle, prec, tol):
    p, x = sphere512
    mv = dda_b200.CudaMatVec(p, prec)
    lay = mv.layout
    assert lay["yz_path"] == "cluster" and lay["compile_time_plans"] == 1
    mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 1, "ldr"))
    y = mv.apply(x)
    assert rel(y, sphere512_oracle) < tol, rel(y, sphere512_oracle)
    mv.close()


def test_sphere512_cluster_path_equals_split_path(sphere512):
    # the production cluster kernel and the split y/z path (tested against
    # the oracle on small grids) on the same input, both FP64
    p, x = sphere512
    out = []
    for flags in (0, dda_b200.api.FLAG_SPLIT_YZ):
        mv = dda_b200.CudaMatVec(p, "fp64", flags=flags)
        assert mv.layout["yz_path"] == ("cluster" if flags == 0 else "split")
        mv.set_couple_constants(dda_b200.CoupleConstants(p, (0, 0, 1), 2, "ldr"))
        out.append(mv.apply(x))
        mv.close()
    assert rel(out[0], out[1]) < FP64_TOL


# ----------------------------------------------- Jones gate, README sphere ----
from dda_b200.fielddiff import normalised_rms as field_diff  # DDA/FieldDiff.cpp:189-192


@pytest.fixture(scope="module")
def cfg1_oracle_jones():
    og = O.Geometry.sphere("10um", "0.5um")
    op = O.Problem(og, [1.5 + 0.1j], "6um")
    op.build_dmatrix()
    prop = (0.0, 0.0, 1.0)
    pols = []
    for pol in (1, 2):
        op.set_cc(prop, pol, "ldr")
        rc, pv, st, _ = op.solve(op.einc(prop, pol), "qmr", 1e-5)
        assert rc == 0
        pols.append(pv)
    theta, phi = PP.grid_angles("0..180/91", "0..360/61")
    return op.jones(pols[0], pols[1], prop, theta, phi), theta, phi


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
def test_cfg1_jones_against_oracle_fp64(cfg1_oracle_jones, prec):
    want, theta, phi = cfg1_oracle_jones
    assert len(theta) == 91 * 61
    g = dda_b200.Geometry.sphere("10um", "0.5um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    assert p.nv == 33552 and p.grid == (80, 80, 80)
    prop = (0.0, 0.0, 1.0)
    mv = dda_b200.CudaMatVec(p, prec, max_rhs=2)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
    s = dda_b200.CudaSolver(mv, "qmr")
    s.get_pol_vec(np.stack([p.einc(prop, 1), p.einc(prop, 2)]), 1e-5)
    assert all(st.status == 0 for st in s.last_stats)
    j = PP.jones_far_field(mv, prop, theta, phi)
    err = field_diff(j, want)
    assert err < 1e-4, err
    mv.close()


# ----------------------------------------- README box, FP32 bench solution ----
def test_cfg2_fp32_solution_against_oracle_fp64():
    # the default benchmark's FP32 solve (both polarisations as one block,
    # BiCGStab to 1e-5): its relative residual in the oracle's FP64 system,
    # and its distance to the oracle's own FP64 solution
    g = dda_b200.Geometry.box_shape("10um", "5um", "5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    prop = (0.0, 1.0, 0.0)
    mv = dda_b200.CudaMatVec(p, "fp32", max_rhs=2)
    ccs = []
    for r, pol in enumerate((1, 2)):
        ccs.append(dda_b200.CoupleConstants(p, prop, pol, "ldr"))
        mv.set_couple_constants(ccs[-1], rhs=r)
    einc = np.stack([p.einc(prop, 1), p.einc(prop, 2)])
    P = dda_b200.CudaSolver(mv, "bicgstab").get_pol_vec(einc, 1e-5)
    mv.close()
    og = O.Geometry.box("10um", "5um", "5um", "0.1um")
    op = O.Problem(og, [1.5 + 0.1j], "6um")
    op.build_dmatrix()
    for r, pol in enumerate((1, 2)):
        op.set_cc(prop, pol, "ldr")
        cs = _cc_vector(p, ccs[r])
        live = cs != 0
        x = np.zeros_like(P[r])
        x[live] = P[r][live] / cs[live]
        b = cs * einc[r]
        res = np.linalg.norm(b - op.matvec(x)) / np.linalg.norm(b)
        assert res < 1.5e-5, (pol, res)
        rc, opol, _, _ = op.solve(op.einc(prop, pol), "bicgstab", 1e-5)
        assert rc == 0
        assert rel(P[r], opol) < 1e-4, (pol, rel(P[r], opol))


def test_cfg2_fp64_histories_match_oracle_fixture():
    # the oracle's iteration counts and residual histories of this workload
    # (tests/golden/cfg2_oracle_bicgstab.json, made by make_cfg2_iterations.py)
    import json
    import os
    ref = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cfg2_oracle_bicgstab.json")))
    g = dda_b200.Geometry.box_shape("10um", "5um", "5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "6um")
    prop = (0.0, 1.0, 0.0)
    mv = dda_b200.CudaMatVec(p, "fp64", max_rhs=2)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
    s = dda_b200.CudaSolver(mv, "bicgstab")
    s.get_pol_vec(np.stack([p.einc(prop, 1), p.einc(prop, 2)]), 1e-5)
    for r, pol in enumerate(("1", "2")):
        want = np.array(ref["pols"][pol]["history"])
        assert s.last_stats[r].iterations == ref["pols"][pol]["iterations"]
        got = s.last_history[r]
        assert np.max(np.abs(got - want) / want) < 1e-7
    mv.close()
