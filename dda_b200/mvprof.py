"""Times the matvec passes of one of the README workloads on the GPU.

    python -m dda_b200.mvprof --shape box --precision fp32 --nrhs 2 --reps 20 [--flags N]

Shapes: `sphere` (radius 10 um, d 0.5 um, lambda 6 um: grid 80^3), `box`
(10 x 5 x 5 um, d 0.1 um: grid 200 x 100 x 100), `sphere256` (radius 12.8 um,
d 0.1 um, lambda 1.3404 um: grid 512^3).  Prints the mean milliseconds of the
x forward, y/z and x inverse passes and of the whole matvec as one JSON line
(dda_profile_matvec, CUDA events on the context stream).
"""
import argparse
import json

import dda_b200 as D

SHAPES = {
    "sphere": (lambda: D.Geometry.sphere("10um", "0.5um"), 1.5 + 0.1j, "6um"),
    "box": (lambda: D.Geometry.box_shape("10um", "5um", "5um", "0.1um"), 1.5 + 0.1j, "6um"),
    "sphere256": (lambda: D.Geometry.sphere("12.8um", "0.1um"), 1.6 + 0.01j, "1.3404um"),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", default="box", choices=sorted(SHAPES))
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--flags", type=int, default=0)
    a = ap.parse_args()
    geom, m, lam = SHAPES[a.shape]
    p = D.DDAParams(geom(), [m], lam)
    mv = D.CudaMatVec(p, a.precision, max_rhs=a.nrhs, flags=a.flags)
    for r in range(a.nrhs):
        mv.set_couple_constants(D.CoupleConstants(p, (0, 0, 1), 1 + r % 2, "ldr"), rhs=r)
    ms = mv.profile(nrhs=a.nrhs, reps=a.reps)
    print(json.dumps({"shape": a.shape, "grid": list(p.grid), "nv": p.nv, "precision": a.precision,
                      "nrhs": a.nrhs, "flags": a.flags, "layout": mv.layout,
                      "ms": {"x_forward": ms[0], "yz": ms[1], "x_inverse": ms[2], "total": ms[3]}}))


if __name__ == "__main__":
    main()
