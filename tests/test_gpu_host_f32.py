"""dda_solve_f32: the solve on single-precision host arrays (the vectors of the
reference's --ftype float path, IterativeSolverBase<float>::getPolVec,
DDA/IterativeSolverBase.hpp:59) gives dda_solve's result rounded to float, with
the same iterations, in every context precision."""
import numpy as np
import pytest

import dda_b200


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64", "mixed"])
def test_single_precision_host_arrays_match_dda_solve(prec):
    g = dda_b200.Geometry.sphere("0.6um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "2um")
    mv = dda_b200.CudaMatVec(p, prec, max_rhs=2)
    prop = (0.0, 0.6, 0.8)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
    e32 = np.stack([p.einc(prop, 1), p.einc(prop, 2)]).astype(np.complex64)
    s = dda_b200.CudaSolver(mv, "bicgstab")
    p32 = s.get_pol_vec(e32, 1e-5)
    assert p32.dtype == np.complex64
    its32 = [st.iterations for st in s.last_stats]
    p64 = s.get_pol_vec(e32.astype(np.complex128), 1e-5)
    its64 = [st.iterations for st in s.last_stats]
    assert its32 == its64
    # the inputs widen exactly; the device arithmetic is the same
    assert np.array_equal(p32, p64.astype(np.complex64))
    # into a caller's buffer, from the solution as start value
    out = np.empty_like(e32)
    s.get_pol_vec(e32, 1e-5, start=p32, out=out)
    assert max(st.iterations for st in s.last_stats) <= 2
    assert np.abs(out - p32).max() <= 1e-3 * np.abs(p32).max()
    mv.close()
