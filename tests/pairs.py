"""Builds the same DDA problem in the CUDA library and in the oracle."""
import numpy as np

import dda_b200
from oracle import oracle as O


def geometry(kind, args):
    if kind == "sphere":
        return dda_b200.Geometry.sphere(*args), O.Geometry.sphere(*args)
    if kind == "box":
        return dda_b200.Geometry.box_shape(*args), O.Geometry.box(*args)
    if kind == "cylinder":
        return dda_b200.Geometry.cylinder(*args), O.Geometry.cylinder(*args)
    if kind == "load":
        return dda_b200.Geometry.load(*args), O.Geometry.load_text(*args)
    if kind == "arrays":
        pos, mat, gu = args
        return dda_b200.Geometry.from_arrays(pos, mat, gu), O.Geometry.from_arrays(pos, mat, gu)
    raise ValueError(kind)


def aniso_arrays():
    """Small two-material target with holes (lines of uneven length)."""
    pos = [(x, y, z) for z in range(5) for y in range(6) for x in range(7) if (x + 2 * y + 3 * z) % 5]
    pos = np.array(pos, dtype=np.uint32)
    mat = (pos[:, 0] % 2).astype(np.uint8)
    return pos, mat, "0.1um"


def scrambled_arrays():
    """Same target with dipoles shuffled inside each z layer (z order kept),
    so the library's line ordering differs from the caller's."""
    pos, mat, gu = aniso_arrays()
    rng = np.random.default_rng(7)
    order = np.lexsort((rng.random(len(pos)), pos[:, 2]))
    return pos[order], mat[order], gu


class Pair:
    def __init__(self, kind, args, mats, lam, precision="fp64", max_rhs=1, flags=0,
                 host_d=False, oracle_d=True):
        self.g, self.og = geometry(kind, args)
        self.p = dda_b200.DDAParams(self.g, mats, lam)
        self.op = O.Problem(self.og, mats, lam)
        assert self.p.grid == self.op.grid and self.p.nvs == self.op.nvs
        if oracle_d or host_d:
            self.op.build_dmatrix()
        d = self.op.dmatrix() if host_d else None
        self.mv = dda_b200.CudaMatVec(self.p, precision, max_rhs=max_rhs, dmatrix=d, flags=flags)

    def set_cc(self, prop=(0, 0, 1), pol=1, kind="ldr", rhs=0):
        cc = dda_b200.CoupleConstants(self.p, prop, pol, kind)
        self.mv.set_couple_constants(cc, rhs)
        self.op.set_cc(prop, pol, kind)
        return cc

    def rand_vec(self, seed):
        rng = np.random.default_rng(seed)
        n = self.p.vec_size
        x = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        for c in range(3):
            x[c * self.p.nvs + self.p.nv:(c + 1) * self.p.nvs] = 0
        return x


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))
