"""dda_far_field_noalloc (far field through a fixed device scratch, no
allocation) against dda_far_field on the same context.  Collected last so
that it also runs after every other test has used the device."""
import numpy as np
import pytest

import dda_b200
from dda_b200 import postprocess as PP

pytestmark = pytest.mark.gpu

PROP = (0.0, 0.6, 0.8)


def _solved(precision):
    g = dda_b200.Geometry.sphere("0.5um", "0.1um")
    p = dda_b200.DDAParams(g, [1.5 + 0.1j], "1um")
    mv = dda_b200.CudaMatVec(p, precision, max_rhs=2)
    for r, pol in enumerate((1, 2)):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, PROP, pol, "ldr"), rhs=r)
    einc = np.stack([p.einc(PROP, 1), p.einc(PROP, 2)])
    dda_b200.CudaSolver(mv, "qmr").get_pol_vec(einc, 1e-8)
    return mv


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_far_field_matches_far_field_twice(precision):
    mv = _solved(precision)
    theta, phi = PP.grid_angles("0..180/19", "0..360/13")
    dirs, _, _ = PP.scattering_frame(PROP, theta, phi)
    want = mv.far_field(dirs, nrhs=2)
    scale = np.abs(want).max()
    for _ in range(2):
        got = mv.far_field_noalloc(dirs, nrhs=2)
        assert np.abs(got - want).max() <= 1e-12 * scale
    # a smaller request after a larger one reads only what it wrote
    got1 = mv.far_field_noalloc(dirs[:5], nrhs=1)
    assert np.abs(got1[:, 0] - want[:5, 0]).max() <= 1e-12 * scale


def test_noalloc_far_field_rejects_beyond_scratch():
    mv = _solved("fp64")
    dirs = np.tile([[0.0, 0.0, 1.0]], (8737, 1))  # 209,920 + 838,752 bytes > 1 MiB
    with pytest.raises(dda_b200.DDAError) as err:
        mv.far_field_noalloc(dirs, nrhs=2)
    assert "scratch" in str(err.value)
    # the largest request that fits still works
    out = mv.far_field_noalloc(dirs[:8736], nrhs=2)  # 1,048,320 bytes
    want = mv.far_field(dirs[:1], nrhs=2)
    assert np.abs(out[-1] - want[0]).max() <= 1e-12 * np.abs(want).max()
