"""The other workloads of bench.py (--workload batched | mixed512 | serve).

Each prints one JSON line like the default one.  All inputs are synthetic
and generated in-process with fixed seeds.

  batched   prolate spheroid, semi-axes 48 x 32 x 32 dipoles (box 96 x 64 x
            64, 206 192 dipoles, grid 192 x 128 x 128), m = 1.33+0.01i,
            size parameter k a_eq = 15 with a_eq = (48*32*32)^(1/3) d; 64
            incidences N(0, I3)/|.| from numpy default_rng(20261203) x 2
            polarisations = 128 right-hand sides solved as one block, FP32
            complex QMR-CS with FP64 residual refinement to 1e-5 (plain FP32
            QMR stagnates near 7e-5 on 2 of the 128 right-hand sides).
  mixed512  sphere of diameter 256 dipoles (radius 12.8 um, d 0.1 um, grid
            512^3, 8 783 848 dipoles), m = 1.6+0.01i, lambda 1.3404 um
            (x = k r = 60), incidence (0,0,1), both polarisations: FP32
            QMR-CS inner solves with FP64 residual refinement to 1e-6,
            against the FP64 solve (Cext, Cabs, Jones matrices) and the Mie
            series.
  serve     Poisson stream (mean --rate per second) of --requests random
            targets (spheres, spheroids, boxes, aggregates of 2-20 spheres,
            edge log-uniform 16-160 dipoles, Re m U[1.05, 2], Im m U[0, 0.5],
            isotropic incidence, both polarisations), FP32 with FP64
            refinement to 1e-5, through the request loop (dda_serve_*).
"""
import json
import math
import os
import sys
import time

import numpy as np

import bench
from bench import ClockSampler, dist_env

SEED = 20261203


def _peaks():
    try:
        return json.load(open(os.path.join(bench.ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def _roofline(p, mv, nrhs, s_bytes, reps=5):
    ms = mv.profile(nrhs=nrhs, reps=reps)
    sb = bench.stage_bytes(p, mv, nrhs, s_bytes)
    names = ["x_forward", "yz_planes", "x_inverse"]
    dom = int(np.argmax(ms[:3]))
    peaks = _peaks()
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = sb[names[dom]] / (ms[dom] * 1e-3) / 1e9
    total = sum(sb.values())
    return ({"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
             "frac": achieved / peak, "traffic": None,
             "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
             "algorithmic_bytes_per_launch": sb[names[dom]], "ms_per_launch": float(ms[dom])},
            {"ms": float(ms[3]), "stages_ms": dict(zip(names, map(float, ms[:3]))),
             "GB_per_s": total / (ms[3] * 1e-3) / 1e9, "frac_of_hbm": total / (ms[3] * 1e-3) / 1e9 / peak,
             "nrhs": nrhs, "algorithmic_bytes": total})


def _line(metric, value, unit, args, ms_per_step, dtype, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
         "vs_baseline": None, "dtype": dtype, "data": "synthetic (generated in-process, fixed seeds)",
         "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


# ------------------------------------------------------------- batched ----
def spheroid_problem(nrhs=128):
    """The 128-rhs spheroid workload: params, incident fields [nrhs][3 nvs],
    the (direction, polarisation) of each right-hand side."""
    import dda_b200
    from dda_b200 import targets
    d_um = 0.05
    kd = 15.0 / (48 * 32 * 32) ** (1.0 / 3)
    lam = "%.17gum" % (2 * math.pi * d_um / kd)
    pos = targets.spheroid(48, 32, 32)
    g = dda_b200.Geometry.from_arrays(pos, np.zeros(len(pos), np.uint8), "%gum" % d_um)
    p = dda_b200.DDAParams(g, [1.33 + 0.01j], lam)
    rng = np.random.default_rng(SEED)
    dirs = rng.normal(size=(64, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rhs = [(tuple(dirs[r // 2]), 1 + r % 2) for r in range(nrhs)]
    einc = np.empty((nrhs, p.vec_size), dtype=np.complex128)
    for r, (prop, pol) in enumerate(rhs):
        einc[r] = p.einc(prop, pol)
    return p, einc, rhs


def spheroid_cpu_sample(p, rhs0, n_iter, precision="fp32", iters=4):
    """Bounded CPU sample of one right-hand side of the spheroid block: the
    oracle's QMR-CS set-up plus `iters` iterations, timed, then scaled to
    `n_iter` iterations (the mean the GPU block needed).  Extrapolated: a
    full oracle solve of one right-hand side takes minutes."""
    from oracle import oracle as O
    og = O.Geometry.from_arrays(p.geometry.positions, p.geometry.materials, "0.05um")
    op = O.Problem(og, [1.33 + 0.01j], p.wavelength)
    t0 = time.perf_counter()
    op.build_dmatrix()
    t_d = time.perf_counter() - t0
    prop, pol = rhs0
    op.set_cc(prop, pol, "ldr")
    e = op.einc(prop, pol)
    t0 = time.perf_counter()
    op.solve(e, "qmr", 1e-5, stop_after=1, precision=precision)
    t1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    op.solve(e, "qmr", 1e-5, stop_after=1 + iters, precision=precision)
    tn = time.perf_counter() - t0
    per_it = (tn - t1) / iters
    per_solve = (t1 - per_it) + n_iter * per_it
    return {"value": 1.0 / per_solve, "unit": "solves/s", "cores": O.max_threads(), "kind": "port",
            "precision": precision, "extrapolated": True, "seconds_per_iteration": per_it,
            "sample": "oracle QMR-CS (%s), rhs 0: set-up + 1 and %d iterations timed, scaled to %.0f "
                      "iterations (the GPU block's mean); D matrix %.1f s beforehand"
                      % (precision, 1 + iters, n_iter, t_d)}


def batched_block(steps, warmup, local=0, nrhs=128, cpu=True):
    """The 128-rhs spheroid block measured on this GPU; returns the line's
    fields (value, latency, e2e, roofline, matvec, FP64 comparisons, CPU
    sample)."""
    import torch
    import dda_b200
    p, einc, rhs = spheroid_problem(nrhs)
    mv = dda_b200.CudaMatVec(p, "mixed", max_rhs=nrhs)
    for r, (prop, pol) in enumerate(rhs):
        mv.set_couple_constants(dda_b200.CoupleConstants(p, prop, pol, "ldr"), rhs=r)
    solver = dda_b200.CudaSolver(mv, "qmr")
    e_dev = torch.from_numpy(einc).cuda()  # FP64 pairs: the refinement's outer residual is FP64
    pol_dev = torch.zeros_like(e_dev)
    stream = torch.cuda.ExternalStream(mv.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step():
        solver.get_pol_vec_device(e_dev.data_ptr(), pol_dev.data_ptr(), nrhs, 1e-5)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    iters = [st.iterations for st in solver.last_stats]
    refs = [st.refinements for st in solver.last_stats]
    resid = max(st.rel_residual for st in solver.last_stats)
    sampler = ClockSampler(local)
    sampler.start()
    l0 = mv.launches
    lat = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        step()
        b.record(stream)
        b.synchronize()
        lat.append(a.elapsed_time(b))
        sampler.sample()
    total = sum(lat)
    launches = mv.launches - l0
    clocks = sampler.stop()
    value = nrhs * steps / (total / 1000.0)
    # e2e through the host API, from and into pinned host memory
    einc_host = torch.empty(einc.size, dtype=torch.complex128, pin_memory=True).numpy()
    einc_host[:] = einc.reshape(-1)
    pol_host = torch.empty(einc.size, dtype=torch.complex128, pin_memory=True).numpy()
    e2e_ms = 0.0
    n_e2e = max(1, steps // 2)
    for _ in range(n_e2e):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.get_pol_vec(einc_host, 1e-5, history_cap=1, out=pol_host)
        b.record(stream)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
    e2e = {"value": nrhs * n_e2e / (e2e_ms / 1000.0), "unit": "solves/s",
           "h2d_bytes_per_step": int(einc.nbytes), "d2h_bytes_per_step": int(einc.nbytes)}
    roof, matvec = _roofline(p, mv, nrhs, 8, reps=3)
    roof["traffic"] = bench.traffic_per_launch("spheroid", nrhs)
    layout = mv.layout
    mv.close()
    del e_dev, pol_dev, einc_host, pol_host
    torch.cuda.empty_cache()
    # FP64 single-rhs solves of the first incidence, both polarisations: this
    # library's FP64 path, and the straightforward restatement (cuFFT,
    # unfused vector operations, host-side scalars; the plain denominator)
    import bench_plain
    mv64 = dda_b200.CudaMatVec(p, "fp64", max_rhs=1)
    s64 = dda_b200.CudaSolver(mv64, "qmr")
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    st64 = torch.cuda.ExternalStream(mv64.stream)
    its64 = []
    a.record(st64)
    for r in range(2):
        mv64.set_couple_constants(dda_b200.CoupleConstants(p, rhs[r][0], rhs[r][1], "ldr"))
        s64.get_pol_vec(einc[r], 1e-5, history_cap=1)
        its64.append(s64.last_stats[0].iterations)
    b.record(st64)
    b.synchronize()
    ours64 = {"value": 2 / (a.elapsed_time(b) / 1000.0), "unit": "solves/s", "iterations": its64,
              "sample": "incidence 0, both polarisations, one FP64 solve each (this library)"}
    sps = [bench_plain.PlainSolver(mv64, p, dda_b200.CoupleConstants(p, rhs[r][0], rhs[r][1], "ldr").cc_sqrt)
           for r in range(2)]
    sps[0].solve_qmr(einc[0], 1e-5, max_iter=5)  # cuFFT plans
    torch.cuda.synchronize()
    a.record()
    itp = [sp.solve_qmr(einc[r], 1e-5)[1] for r, sp in enumerate(sps)]
    b.record()
    b.synchronize()
    plain = {"value": 2 / (a.elapsed_time(b) / 1000.0), "unit": "solves/s", "iterations": itp,
             "sample": "incidence 0, both polarisations: straightforward FP64 QMR-CS (cuFFT, unfused "
                       "vector operations, host-side scalars, bench_plain.py)"}
    del sps
    mv64.close()
    cpu_b = None
    if cpu:
        try:
            cpu_b = spheroid_cpu_sample(p, rhs[0], float(np.mean(iters)))
        except Exception as ex:  # the CPU baseline is reported, never required
            cpu_b = {"value": None, "error": str(ex)}
    return {"value": value, "unit": "solves/s", "ms_per_step": total / steps, "steps": steps, "warmup": warmup,
            "config": {"workload": "spheroid 48x32x32 dipoles, m=1.33+0.01i, k a_eq=15, 64 directions x 2 pols "
                                   "= 128 rhs, qmr eps=1e-5, fp32 convolution + fp64 refinement",
                       "nv": p.nv, "grid": list(p.grid), "rhs_per_step": nrhs, "precision": "mixed"},
            "iterations_max": max(iters), "iterations_mean": float(np.mean(iters)), "max_rel_residual": resid,
            "refinements_max": max(refs), "l2": "flushed between steps (256 MB write)", "layout": layout,
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "matvec": matvec,
            "plain_fp64_single_rhs": plain, "ours_fp64_single_rhs": ours64,
            "speedup_vs_plain": value / plain["value"],
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "per": "block of %d rhs" % nrhs, "samples": len(lat)},
            "cpu_baseline": cpu_b, "clocks": clocks}


def run_batched(args):
    import torch
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    d = batched_block(args.steps, args.warmup, local, cpu=not args.no_cpu)
    extra = {k: v for k, v in d.items() if k not in ("value", "unit", "ms_per_step", "steps", "warmup", "config")}
    _line("solves/s at relative residual 1e-5 (128-rhs spheroid block, QMR-CS)", d["value"], "solves/s", args,
          d["ms_per_step"], "c64+f64", d["config"], **extra)


# ------------------------------------------------------------ mixed512 ----
def run_mixed512(args):
    import torch
    import dda_b200
    from dda_b200 import postprocess as PP
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    g = dda_b200.Geometry.sphere("12.8um", "0.1um")
    p = dda_b200.DDAParams(g, [1.6 + 0.01j], "1.3404um")
    prop = (0.0, 0.0, 1.0)
    einc = np.stack([p.einc(prop, 1), p.einc(prop, 2)])
    theta, phi = PP.grid_angles("0..180/19", "0..360/13")
    out = {}
    for prec, eps in (("mixed", 1e-6), ("fp64", 1e-6)):
        mv = dda_b200.CudaMatVec(p, prec, max_rhs=2)
        ccs = []
        for r, pol in enumerate((1, 2)):
            ccs.append(dda_b200.CoupleConstants(p, prop, pol, "ldr"))
            mv.set_couple_constants(ccs[-1], rhs=r)
        solver = dda_b200.CudaSolver(mv, "qmr", max_iter=args.max_iter)
        stream = torch.cuda.ExternalStream(mv.stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pol = solver.get_pol_vec(einc, eps, history_cap=1, raise_on_error=False)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        _, pn = dda_b200.beam_pol(prop, 1)
        ef = mv.far_field(pn[None, :], nrhs=2)[0]
        cs = [PP.cross_sections(p, ccs[r], pol[r], ef[r], prop, r + 1) for r in range(2)]
        jones = PP.jones_far_field(mv, prop, theta, phi)
        print("mixed512 %s: %.1f s" % (prec, ms / 1000), file=sys.stderr, flush=True)
        out[prec] = {"ms": ms, "stats": [dict(iterations=s.iterations, refinements=s.refinements,
                                              rel_residual=s.rel_residual, status=s.status)
                                         for s in solver.last_stats],
                     "cext": [c[0] for c in cs], "cabs": [c[1] for c in cs], "qext": [c[2] for c in cs],
                     "qabs": [c[3] for c in cs], "jones": jones, "launches": mv.launches,
                     "layout": mv.layout}
        if prec == "mixed":
            roof, matvec = _roofline(p, mv, 2, 8, reps=2)
        mv.close()
        del pol
    mx, f64 = out["mixed"], out["fp64"]
    jr = np.sqrt(np.sum(np.abs(mx["jones"] - f64["jones"]) ** 2) / np.sum(np.abs(f64["jones"]) ** 2))
    x = 2 * math.pi * 12.8 / 1.3404
    qe, _, qa = PP.mie(x, 1.6 + 0.01j)
    area = math.pi * (12.8e-6) ** 2
    acc = {"jones_rel_rms_vs_fp64": float(jr),
           "cext_rel_vs_fp64": [abs(a - b) / abs(b) for a, b in zip(mx["cext"], f64["cext"])],
           "cabs_rel_vs_fp64": [abs(a - b) / abs(b) for a, b in zip(mx["cabs"], f64["cabs"])],
           "mie_qext": qe, "mie_qabs": qa,
           "dda_qext_r12.8um": [c / area for c in mx["cext"]], "dda_qabs_r12.8um": [c / area for c in mx["cabs"]]}
    value = 2 / (mx["ms"] / 1000.0)
    plain = 2 / (f64["ms"] / 1000.0)
    for d in (mx, f64):
        d.pop("jones")
    _line("solves/s at relative residual 1e-6 (512^3 sphere, FP32 QMR-CS + FP64 refinement)", value, "solves/s",
          args, mx["ms"], "c64+f64",
          {"workload": "sphere r=12.8um d=0.1um (diameter 256 dipoles) m=1.6+0.01i lambda=1.3404um prop=(0,0,1), "
                       "both pols, qmr, eps=1e-6", "nv": p.nv, "grid": list(p.grid), "rhs_per_step": 2,
           "max_iter": args.max_iter},
          mixed=mx, fp64_gpu=f64, accuracy=acc, speedup_vs_fp64_gpu=value / plain, roofline=roof,
          matvec=matvec, gpu_launches=mx["launches"])


# --------------------------------------------------------------- serve ----
def run_serve(args):
    import torch
    import dda_b200
    from dda_b200 import targets
    from dda_b200.serve import Server
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(SEED)
    reqs = [targets.served_request(rng, (16, 160)) for _ in range(args.requests)]
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=args.requests))
    # warm-up: one small request through the loop (context set-up paths)
    warm = Server(max_active=1)
    w = targets.served_request(np.random.default_rng(1), (16, 20))
    warm.submit(w["positions"], None, w["refr"], w["grid_unit"], w["wavelength"], prop=w["prop"])
    warm.drain()
    warm.close()
    srv = Server(max_active=args.slots)
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        delay = arrivals[i] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        srv.submit(r["positions"], r["materials"], r["refr"], r["grid_unit"], r["wavelength"], prop=r["prop"],
                   tag=i)
    res = srv.drain()
    clocks = sampler.stop()
    srv.close()
    ok = [d for d in res if d["status"] == 0]
    lat = np.array([(d["t_done"] - d["t_submit"]) * 1000 for d in ok])
    wait = np.array([(d["t_admit"] - d["t_submit"]) * 1000 for d in ok])
    span = max(d["t_done"] for d in res) - min(d["t_submit"] for d in res)
    solves = 2 * len(ok)
    value = solves / span
    # baselines on every 4th request of the same stream (same size
    # distribution), one solve at a time, reference grids, host wall clock:
    # this library's FP64 path through the server, and the straightforward
    # restatement (D-matrix from the library, then cuFFT, unfused vector
    # operations and host-side scalars, bench_plain.py)
    kinds = {}
    for r in reqs:
        kinds[r["kind"]] = kinds.get(r["kind"], 0) + 1
    config = {"workload": "Poisson %.1f req/s, %d requests, edges log-uniform 16-160 dipoles, spheres/spheroids/"
                          "boxes/aggregates, m Re U[1.05,2] Im U[0,0.5], random prop, both pols, mixed fp32+fp64 "
                          "refinement, qmr eps=1e-5" % (args.rate, args.requests),
              "slots": args.slots, "kinds": kinds, "nv_max": int(max(len(r["positions"]) for r in reqs))}
    latency = {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
               "mean": float(np.mean(lat)), "queue_wait_p50": float(np.percentile(wait, 50)),
               "service_p50": float(np.percentile(lat - wait, 50)), "service_p99": float(np.percentile(lat - wait, 99))}
    e2e = {"value": value, "unit": "solves/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
           "note": "the stream is end to end: host geometry in, cross sections out"}
    if args.no_plain:
        _line("served solves/s and latency at relative residual 1e-5 (Poisson stream of random targets)", value,
              "solves/s", args, float(np.mean(lat)) if len(lat) else None, "c64+f64", config, latency_ms=latency,
              completed=len(ok), failed=len(res) - len(ok), clocks=clocks, e2e=e2e)
        return
    import bench_plain
    sample = reqs[::4]
    nplain = len(sample)
    plain_srv = Server(max_active=1)
    t1 = time.perf_counter()
    for r in sample:
        for pol in (1, 2):
            plain_srv.submit(r["positions"], r["materials"], r["refr"], r["grid_unit"], r["wavelength"],
                             prop=r["prop"], npol=1, first_pol=pol, precision="fp64", solver="qmr",
                             grid_policy="reference")
            plain_srv.drain()
    t_ours64 = time.perf_counter() - t1
    plain_srv.close()
    t1 = time.perf_counter()
    its_plain = []
    for r in sample:
        g = dda_b200.Geometry.from_arrays(r["positions"], np.zeros(len(r["positions"]), np.uint8), r["grid_unit"])
        p = dda_b200.DDAParams(g, r["refr"], r["wavelength"])
        mv = dda_b200.CudaMatVec(p, "fp64")
        for pol in (1, 2):
            sp = bench_plain.PlainSolver(mv, p, dda_b200.CoupleConstants(p, r["prop"], pol, "ldr").cc_sqrt)
            its_plain.append(sp.solve_qmr(p.einc(r["prop"], pol), 1e-5, max_iter=20000)[1])
            del sp
        mv.close()
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t1
    _line("served solves/s and latency at relative residual 1e-5 (Poisson stream of random targets)", value,
          "solves/s", args, float(np.mean(lat)) if len(lat) else None, "c64+f64", config,
          latency_ms=latency, completed=len(ok), failed=len(res) - len(ok),
          plain_fp64_single_rhs={"value": 2 * nplain / t_plain, "unit": "solves/s",
                                 "iterations_mean": float(np.mean(its_plain)),
                                 "sample": "every 4th request (%d), each polarisation one straightforward "
                                           "FP64 QMR-CS solve (bench_plain.py) on the reference grid, one at "
                                           "a time, D-matrix set-up included (host wall clock)" % nplain},
          ours_fp64_single_rhs={"value": 2 * nplain / t_ours64, "unit": "solves/s",
                                "sample": "the same requests through this library's FP64 path"},
          speedup_vs_plain=value / (2 * nplain / t_plain), clocks=clocks, e2e=e2e)
