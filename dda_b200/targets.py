"""Dipole-list targets for the batched and served workloads.

Spheres use the reference's own shape (DDA/Shapes.cpp:53-143 through the
front end); spheroids, boxes and aggregates of spheres are dipole lists built
with the same cell-centre rule (a cell belongs to the body when its centre,
x + 0.5 in grid units, lies inside), in z-major order as DipoleGeometry
requires (DDA/DDAParams.cpp:441-445).  The spheroid and aggregate shapes are
not reference shapes; the reference takes them as loaded dipole lists
(--geometry load:file=, DDA/DDAMain.cpp:156-249).
"""
import math

import numpy as np

from . import api


def _cells(shape):
    z, y, x = np.meshgrid(np.arange(shape[2]), np.arange(shape[1]), np.arange(shape[0]), indexing="ij")
    return x.ravel(), y.ravel(), z.ravel()


def _as_list(mask_xyz, x, y, z):
    keep = mask_xyz
    pos = np.stack([x[keep], y[keep], z[keep]], axis=1).astype(np.uint32)
    return pos  # z-major order is kept by the meshgrid layout


def spheroid(ax, ay, az):
    """Ellipsoid with semi-axes (ax, ay, az) in dipoles, box 2a x 2b x 2c."""
    x, y, z = _cells((int(round(2 * ax)), int(round(2 * ay)), int(round(2 * az))))
    r = ((x + 0.5 - ax) / ax) ** 2 + ((y + 0.5 - ay) / ay) ** 2 + ((z + 0.5 - az) / az) ** 2
    return _as_list(r <= 1.0, x, y, z)


def box(ex, ey, ez):
    x, y, z = _cells((ex, ey, ez))
    return _as_list(np.ones(len(x), dtype=bool), x, y, z)


def aggregate(centres, radii, extent):
    """Union of spheres (centres and radii in dipoles) inside a box `extent`."""
    x, y, z = _cells(extent)
    inside = np.zeros(len(x), dtype=bool)
    for c, r in zip(centres, radii):
        inside |= (x + 0.5 - c[0]) ** 2 + (y + 0.5 - c[1]) ** 2 + (z + 0.5 - c[2]) ** 2 <= r * r
    pos = _as_list(inside, x, y, z)
    # shift to the occupied bounding box
    return (pos - pos.min(axis=0)).astype(np.uint32)


def sphere(diameter, grid_unit_um):
    """Reference sphere (DDA/Shapes.cpp) of `diameter` dipoles."""
    g = api.Geometry.sphere("%.17gum" % (diameter * grid_unit_um / 2), "%.17gum" % grid_unit_um)
    return g.positions.astype(np.uint32)


def random_direction(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def served_request(rng, edge_range=(16, 160), grid_unit_um=0.05):
    """One request of the served workload: a random target (sphere, spheroid,
    box or an aggregate of 2-20 overlapping spheres) with its edge
    log-uniform in `edge_range` dipoles, refractive index Re U[1.05, 2.0],
    Im U[0, 0.5], an isotropic incidence and both polarisations.  The
    wavelength puts |m| k d in [0.3, 0.8]."""
    lo, hi = edge_range
    e = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
    e = max(e, 4)
    kind = rng.choice(["sphere", "spheroid", "box", "aggregate"])
    if kind == "sphere":
        pos = sphere(e, grid_unit_um)
    elif kind == "spheroid":
        f = rng.uniform(0.5, 1.0, size=2)
        pos = spheroid(e / 2, max(2.0, e * f[0] / 2), max(2.0, e * f[1] / 2))
    elif kind == "box":
        f = rng.uniform(0.5, 1.0, size=2)
        pos = box(e, max(2, int(e * f[0])), max(2, int(e * f[1])))
    else:
        n = int(rng.integers(2, 21))
        r = rng.uniform(0.15, 0.3, size=n) * e
        c = rng.uniform(0.3, 0.7, size=(n, 3)) * e
        pos = aggregate(c, r, (e, e, e))
    m = complex(rng.uniform(1.05, 2.0), rng.uniform(0.0, 0.5))
    kd = rng.uniform(0.3, 0.8) / abs(m)
    lam_um = 2 * math.pi * grid_unit_um / kd
    return {"kind": str(kind), "edge": e, "positions": pos, "materials": None, "refr": [m],
            "grid_unit": "%.17gum" % grid_unit_um, "wavelength": "%.17gum" % lam_um,
            "prop": tuple(random_direction(rng))}
