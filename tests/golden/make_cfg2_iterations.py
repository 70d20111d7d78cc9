"""Runs the oracle's BiCGStab solve of the box workload (10 x 5 x 5 um box,
d = 0.1 um, m = 1.5+0.1i, lambda = 6 um, propagation (0,1,0), LDR, relative
residual 1e-5) for both polarisations and records the iteration counts and
residual histories in cfg2_oracle_bicgstab.json.  The GPU tests compare the
library's FP64 solve of the same workload with these counts and histories
(tests/test_gpu_configs.py)."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def main():
    g = O.Geometry.box("10um", "5um", "5um", "0.1um")
    p = O.Problem(g, [1.5 + 0.1j], "6um")
    t0 = time.time()
    p.build_dmatrix()
    out = {"workload": "box 10x5x5um d=0.1um m=1.5+0.1i lambda=6um prop=(0,1,0) ldr bicgstab eps=1e-5",
           "nv": p.nv, "grid": list(p.grid), "dmatrix_seconds": time.time() - t0,
           "threads": O.max_threads(), "pols": {}}
    for pol in (1, 2):
        p.set_cc((0, 1, 0), pol, "ldr")
        e = p.einc((0, 1, 0), pol)
        t0 = time.time()
        rc, pv, st, hist = p.solve(e, "bicgstab", 1e-5)
        out["pols"][str(pol)] = {"status": rc, "iterations": int(st.iterations),
                                 "rel_residual": st.relResidual, "seconds": time.time() - t0,
                                 "history": [float(h) for h in hist]}
        print(pol, rc, st.iterations, time.time() - t0, flush=True)
    with open(os.path.join(HERE, "cfg2_oracle_bicgstab.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
