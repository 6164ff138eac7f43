"""Benchmark of the rooftop-mom solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c1|c2|c3|c4|c5]

A step is one complete plate solve of the workload: generator assembly, spectra, preconditioner,
plane-wave excitation, the iterative solve to the workload's tolerance (the FP64 true residual is
checked) and the monostatic RCS. The default workload is the 256 x 256 plate of cell lambda/20
(130,560 unknowns), plane wave theta = 30 deg, phi = 0, TE, block-Jacobi (2 x 2 faces) GMRES(50)
to 1e-6 in FP64. Inputs are synthetic (the plate and the wave are generated; there is no dataset).

Prints one JSON line (rank 0). `value` is whole-job solves/s with the inputs on the device; `e2e` is
the same through the public API with the right-hand side coming from pinned host memory and the
solution going back to it. Multi-GPU runs are independent replicas (each rank solves its own plates,
no collective on the data path): value = all ranks' solves / max over ranks of the timed span.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0

# Workloads (cell lambda/N, k = 2 pi at lambda = 1 m).
WORKLOADS = {
    "c1": dict(n=32, density=20, theta=0.0, phi=0.0, pol="x", method="cg", tol=1e-8, restart=50, pc=None,
               precision="double"),
    "c2": dict(n=256, density=20, theta=30.0, phi=0.0, pol="TE", method="gmres", tol=1e-6, restart=50,
               pc="blockJacobi", precision="double"),
    # the inner FP32 FGMRES(30) runs without a preconditioner (with the rChan circulant, restarted GMRES
    # did not reach the tolerance within 20000 iterations on this plate); the error against an FP64 GPU
    # solve of the same plate is reported beside the line
    "c3": dict(n=1024, density=15, theta=30.0, phi=0.0, pol="TE", method="fgmres", tol=1e-8, restart=30,
               pc=None, precision="mixed"),
    # 64 plane waves, theta ~ U[0, 80] deg, phi ~ U[0, 360) deg, TE / TM ~ Bernoulli(1/2), seed 0; COCG
    # preconditioned by the rChan circulant (the reference's default) in FP64 for all right-hand sides at
    # once. FP32 COCG inside FP64 refinement diverges on this plate (its FP32 recurrences break down
    # within the first inner solve, while FP64 COCG converges in about 1100 iterations), and restarted
    # FP32 GMRES(30) needs more than 20000 iterations, so the precision form is measured on c3.
    "c4": dict(n=512, density=20, rhs=64, seed=0, method="cg", tol=1e-6, restart=30, pc="rChan",
               precision="double", theta="U[0,80]", phi="U[0,360)", pol="TE/TM"),
    # plates of uneven size solved as one plate batch: Nx, Ny ~ U[lo, n] faces (all on one n x n power-of-two
    # transform grid), cell lambda/20, one plane wave each (theta ~ U[0, 80] deg, phi ~ U[0, 360) deg, TE / TM),
    # block-Jacobi (2 x 2 faces) GMRES(50) to 1e-6 in FP64 (the C2 method); against the same plates one by one
    "c4u": dict(n=64, lo=33, density=20, plates=64, seed=0, method="gmres", tol=1e-6, restart=50, pc="blockJacobi",
                precision="double", theta="U[0,80]", phi="U[0,360)", pol="TE/TM"),
    # request stream of plate solves (see serving_requests)
    "c5": dict(n=0, density=0, seed=0, method="cg", tol=1e-6, restart=50, pc="rChan", precision="double",
               theta="U[0,80]", phi="U[0,360)", pol="TE/TM"),
}

SPEED_OF_LIGHT = 299792458.0


def random_waves(count, rng):
    """Directions and polarisations of `count` plane waves: theta ~ U[0, 80] deg, phi ~ U[0, 360) deg, TE or
    TM with probability 1/2 each."""
    dirs, pols = [], []
    for _ in range(count):
        t, p = rng.uniform(0.0, 80.0), rng.uniform(0.0, 360.0)
        d, e = plane_wave_vectors(t, p, "TE" if rng.random() < 0.5 else "TM")
        dirs.append(d)
        pols.append(e)
    return np.array(dirs), np.array(pols)


def batch_rhs(R, prob, dirs, pols):
    """The plane waves of dirs / pols as one device tensor of nrhs * N complex doubles (rtm_plane_wave)."""
    import ctypes as C

    import torch
    from rooftop_mom_b200 import _lib as L

    cx, cy = prob.mesh().count()
    a, b = prob.mesh().faceSize()
    nrhs, n = len(dirs), prob.rooftopCount()
    out = torch.empty(nrhs * n, dtype=torch.complex128, device="cuda")
    d = np.ascontiguousarray(dirs, dtype=np.float64)
    p = np.ascontiguousarray(pols, dtype=np.float64)
    inten = np.ones(nrhs)
    L.call("rtm_plane_wave", cx, cy, a, b, prob.quadratureOrder()[1], prob.wavenumber(),
           d.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p), inten.ctypes.data_as(C.c_void_p), nrhs,
           C.c_void_p(out.data_ptr()), L.DEVICE, None)
    return out


def solve_batch(R, w, b=None, mixed=False):
    """One batched solve of the c4 workload, all right-hand sides in one solve: FP64 COCG preconditioned by the
    rChan circulant; or (mixed) FP32 flexible GMRES(MIXED_RESTART) with the FP32 product and FP32 block-Jacobi
    inside FP64 iterative refinement to the same FP64 true residual (FP32 COCG diverges on this plate)."""
    prob = build_plate(R, w)
    dirs, pols = random_waves(w["rhs"], np.random.default_rng(w["seed"]))
    op = R.Operator(prob, maxRhs=w["rhs"])
    if b is None:
        b = batch_rhs(R, prob, dirs, pols)
    if mixed:
        inner = R.Operator(prob, precision="single", maxRhs=w["rhs"])
        pc = R.Preconditioner.blockJacobi(prob, (2, 2), precision="single")
        res = R.Solver(method="fgmres", tolerance=w["tol"], restart=MIXED_RESTART, innerTolerance=INNER_FLOOR,
                       gramSchmidtPasses=INNER_GS_PASSES,
                       maxIterationCount=20000).solve(op, b, innerOperator=inner, innerPreconditioner=pc,
                                                      nrhs=w["rhs"])
    else:
        pc = R.Preconditioner(prob, kernel="rChan")
        res = R.Solver(method=w["method"], tolerance=w["tol"], maxIterationCount=20000).solve(
            op, b, preconditioner=pc, nrhs=w["rhs"])
    return prob, res


def uneven_plates(R, w):
    """The c4u plates: face counts, plane waves (seed w["seed"])."""
    rng = np.random.default_rng(w["seed"])
    sizes = rng.integers(w["lo"], w["n"] + 1, size=(w["plates"], 2))
    dirs, pols = random_waves(w["plates"], rng)
    return [(int(cx), int(cy)) for cx, cy in sizes], dirs, pols


def plate_batch_step(R, w, batched, device=True):
    """One c4u step: every plate's assembly, spectra, preconditioner and plane wave, then the solves (one
    plate batch, or one plate after another) and each plate's RCS. Returns (results, RCS values, fused,
    seconds of the solves alone)."""
    import torch

    sizes, dirs, pols = uneven_plates(R, w)
    h = 1.0 / w["density"]
    plates = []
    for (cx, cy), d, p in zip(sizes, dirs, pols):
        mesh = R.Mesh(cx, cy, h, h)
        R.setTransformSize(mesh, (w["n"], w["n"]))
        prob = R.Problem(mesh, 2 * math.pi)
        op = R.Operator(prob)
        pc = (R.Preconditioner.blockJacobi(prob, (2, 2)) if w["pc"] == "blockJacobi"
              else R.Preconditioner(prob, kernel=w["pc"]))
        plates.append((op, pc, R.Excitation.planeWave(prob, direction=d, polarization=p, device=device)))
    solver = R.Solver(method=w["method"], tolerance=w["tol"], restart=w["restart"], maxIterationCount=20000,
                      side="right")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if batched:
        batch = R.PlateBatch([op for op, _, _ in plates], [pc for _, pc, _ in plates])
        res = solver.solveBatch(batch, [e for _, _, e in plates])
        fused = batch.fused()
    else:
        res = [solver.solve(op, e, preconditioner=pc) for op, pc, e in plates]
        fused = False
    torch.cuda.synchronize()
    return res, [r.radarCrossSection() for r in res], fused, time.perf_counter() - t0


def run_plate_batch(args, w):
    """c4u: value = plates solved per second as one plate batch; beside it the same plates one by one."""
    import torch

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    R.load()
    arms = {}
    with Clocks(0) as clk:
        for name, batched in (("batch", True), ("one_by_one", False)):
            for _ in range(args.warmup):
                plate_batch_step(R, w, batched)
            torch.cuda.synchronize()
            launches0 = L.launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            solve_s = 0.0
            for _ in range(args.steps):
                res, rcs, fused, ts = plate_batch_step(R, w, batched)
                solve_s += ts
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            arms[name] = {"value": w["plates"] * args.steps / t, "unit": "solves/s", "ms_per_step": t / args.steps * 1e3,
                          "iterations": max(r.iterationCount() for r in res),
                          "true_residual": max(r.residualNorm() for r in res),
                          "all_converged_to_tolerance": all(r.converged() and r.residualNorm() <= w["tol"] for r in res),
                          "gpu_launches": int(L.launch_count() - launches0), "fused": fused, "rcs": rcs,
                          "solve_ms_per_step": solve_s / args.steps * 1e3}
        # e2e: the plane waves from host memory through the same public call, the currents back to it
        plate_batch_step(R, w, True, device=False)
        torch.cuda.synchronize()
        e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e2[0].record()
        for _ in range(args.steps):
            res_h, _, _, _ = plate_batch_step(R, w, True, device=False)
        e2[1].record()
        torch.cuda.synchronize()
        t_e2e = e2[0].elapsed_time(e2[1]) / 1e3
    sizes, _, _ = uneven_plates(R, w)
    unknowns = [(cx - 1) * cy + cx * (cy - 1) for cx, cy in sizes]
    rcs_b, rcs_s = arms["batch"].pop("rcs"), arms["one_by_one"].pop("rcs")
    line = {
        "metric": f"batched solves/s of plates of uneven size (one plane wave each) at rel. residual 1e-6, "
                  f"{w['method']} + {w['pc']}, FP64",
        "value": arms["batch"]["value"], "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": arms["batch"]["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic plates and plane waves, seed 0",
        "config": {"workload": f"c4u: {w['plates']} plates, Nx, Ny ~ U[{w['lo']},{w['n']}] faces on one "
                               f"{w['n']}x{w['n']} transform grid, cell lambda/{w['density']}, one plane wave each, "
                               f"{w['pc']} {w['method']}({w['restart']}) to {w['tol']:g}, FP64, one plate batch",
                   "plates": w["plates"],
                   "unknowns": unknowns, "l2": "working set per step re-created every step"},
        "iterations": arms["batch"]["iterations"], "true_residual": arms["batch"]["true_residual"],
        "all_converged_to_tolerance": arms["batch"]["all_converged_to_tolerance"], "fused": arms["batch"]["fused"],
        "solve_ms_per_step": arms["batch"]["solve_ms_per_step"],
        "one_by_one": arms["one_by_one"], "batch_over_one_by_one": arms["batch"]["value"] / arms["one_by_one"]["value"],
        "solves_batch_over_one_by_one": arms["one_by_one"]["solve_ms_per_step"] / arms["batch"]["solve_ms_per_step"],
        "rcs_rel_batch_vs_one_by_one": max(abs(a - b) / abs(b) for a, b in zip(rcs_b, rcs_s)),
        "e2e": {"value": w["plates"] * args.steps / t_e2e, "unit": "solves/s",
                "h2d_bytes_per_step": 16 * sum(unknowns), "d2h_bytes_per_step": 16 * sum(unknowns)},
        "gpu_launches": arms["batch"]["gpu_launches"], "clocks": clk.summary(),
    }
    print(json.dumps(line))


def serving_requests(R, count, seed):
    """The c5 request stream: faces Nx (and Ny) log-uniform in [16, 768]; with probability 1/2 a strip one
    face wide fed by a 1 V delta gap at its middle, else a plate under a random plane wave; cell lambda/N
    with N ~ U[10, 25]; frequency ~ U[0.5, 3] GHz; to 1e-6 by rChan-preconditioned COCG."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(16), math.log(768)
    out = []
    for _ in range(count):
        nx = int(round(math.exp(rng.uniform(lo, hi))))
        strip = rng.random() < 0.5
        ny = 1 if strip else int(round(math.exp(rng.uniform(lo, hi))))
        cells = rng.uniform(10.0, 25.0)
        f = rng.uniform(0.5e9, 3e9)
        h = SPEED_OF_LIGHT / f / cells
        k = 2 * math.pi * f / SPEED_OF_LIGHT
        # COCG with the rChan circulant, the reference's default preconditioner (face counts with a large
        # prime factor transform by Bluestein convolutions)
        kw = dict(method="cg", preconditioner="rChan", tolerance=1e-6, maxIterationCount=20000)
        if strip:
            out.append(R.Request.deltaGap(nx, 1, h, h, k, portDirection="x", voltage=1.0, **kw))
        else:
            d, p = random_waves(1, rng)
            out.append(R.Request.planeWave(nx, ny, h, h, k, direction=d[0], polarization=p[0], **kw))
    return out


def serve_stream(R, count, slots, precision, sizes, seed=0, batch=0):
    """The c5 stream on a server: a closed-loop burst measures capacity (a tenth of the stream, at least four
    requests a slot), then the stream arrives as a Poisson process at 0.8 x capacity; per-request latency
    (submission to result) gives p50 / p99. precision "double" (FP64) or "mixed" (FP32 inner solves, FP64
    refinement); sizes: the servers' transform-size policy."""
    import torch

    reqs = serving_requests(R, count, seed)
    prec = "single" if precision == "mixed" else "double"
    with R.Server(budgetBytes=150e9, maxActive=slots, precision=prec, transformSizes=sizes, maxBatch=batch) as srv:
        warm = serving_requests(R, 4, seed + 1)
        for r in [srv.submit(q) for q in warm]:
            srv.wait(r, release=True)
        burst = reqs[: min(len(reqs), max(slots * 4, len(reqs) // 10))]
        ids = [srv.submit(q) for q in burst]
        res = [srv.wait(r, release=True) for r in ids]
        span = max(x["finished"] for x in res) - min(x["submitted"] for x in res)
        capacity = len(burst) / span
        rate = 0.8 * capacity
        rng = np.random.default_rng(seed + 2)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ids = []
        for q, ta in zip(reqs, arrivals):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids.append(srv.submit(q))
        res = [srv.wait(r, release=True) for r in ids]
    done = [x for x in res if x["state"] == "done"]
    lat = np.array([x["latency"] for x in done])
    span = max(x["finished"] for x in res) - min(x["submitted"] for x in res)
    ok = [x for x in done if x["converged"] and x["residual"] <= 1e-6]
    return {"value": len(ok) / span, "unit": "solves/s", "requests": len(reqs), "slots": slots,
            "precision": precision, "transform_sizes": sizes, "capacity_solves_per_s": capacity,
            "arrival_rate": rate, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "converged": len(ok), "failed": len(res) - len(done),
            "max_unknowns": int(max(x["unknowns"] for x in res)), "span_s": span}


def run_serving(args):
    """c5: the request stream on one server (serve_stream), one JSON line."""
    import rooftop_mom_b200 as R

    R.load()
    with Clocks(0) as clk:
        out = serve_stream(R, args.requests, args.slots, args.serving_precision, args.serving_sizes,
                           batch=args.serving_batch)
    prec = "single" if args.serving_precision == "mixed" else "double"
    line = {
        "metric": "serving: solves/s and p50/p99 latency of a Poisson request stream at 0.8 x measured capacity",
        "value": out["value"], "unit": "solves/s", "n_gpus": 1, "steps": out["requests"], "warmup": 4,
        "ms_per_step": out["span_s"] / out["requests"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128" if prec == "double" else "c64/c128",
        "data": "synthetic request stream, seed 0",
        "config": {"workload": f"c5: {out['requests']} requests, Nx, Ny log-U[16,768] (half strips, delta gap), "
                               f"cell lambda/U[10,25], f U[0.5,3] GHz, COCG + rChan to 1e-6, "
                               f"{args.serving_precision}, {args.serving_sizes} transform sizes"
                               + (f", plate batches of up to {args.serving_batch}" if args.serving_batch > 1 else ""),
                   "slots": args.slots, "max_batch": args.serving_batch, "budget_bytes": 150e9, "capacity_solves_per_s": out["capacity_solves_per_s"],
                   "arrival_rate": out["arrival_rate"]},
        "p50_ms": out["p50_ms"], "p99_ms": out["p99_ms"], "converged": out["converged"], "failed": out["failed"],
        "max_unknowns": out["max_unknowns"], "clocks": clk.summary(),
    }
    print(json.dumps(line))


def run_batched(args, w):
    """c4: K batched solves of 64 right-hand sides; value = right-hand sides solved per second."""
    import torch

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    R.load()
    for _ in range(args.warmup):
        solve_batch(R, w)
    torch.cuda.synchronize()
    launches0 = L.launch_count()
    its, res_max = [], 0.0
    with Clocks(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            prob, res = solve_batch(R, w)
            its.append(max(r.iterationCount() for r in res))
            res_max = max(res_max, max(r.residualNorm() for r in res))
        e1.record()
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    # e2e: the right-hand sides from pinned host memory, the currents back to it
    prob = build_plate(R, w)
    dirs, pols = random_waves(w["rhs"], np.random.default_rng(w["seed"]))
    host = batch_rhs(R, prob, dirs, pols).cpu().pin_memory()
    out = torch.empty_like(host).pin_memory()
    torch.cuda.synchronize()
    e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e2[0].record()
    for _ in range(args.steps):
        b = host.to("cuda", non_blocking=True)
        _, res = solve_batch(R, w, b=b)
        out.copy_(torch.cat([r.solution() for r in res]), non_blocking=True)
    e2[1].record()
    torch.cuda.synchronize()
    t_e2e = e2[0].elapsed_time(e2[1]) / 1e3
    # the precision form of the batch: FP32 inner FGMRES(50) + block-Jacobi, FP64 refinement
    mixed = {}
    if not args.no_arms:
        solve_batch(R, w, mixed=True)
        torch.cuda.synchronize()
        e3 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e3[0].record()
        for _ in range(args.steps):
            _, mres = solve_batch(R, w, mixed=True)
        e3[1].record()
        torch.cuda.synchronize()
        t_mix = e3[0].elapsed_time(e3[1]) / 1e3
        mixed = {"value": w["rhs"] * args.steps / t_mix, "unit": "solves/s", "ms_per_step": t_mix / args.steps * 1e3,
                 "method": f"FP32 flexible GMRES({MIXED_RESTART}), FP32 product and block-Jacobi (2 x 2 faces), "
                           f"FP64 refinement",
                 "inner_iterations": max(r.iterationCount() for r in mres),
                 "true_residual": max(r.residualNorm() for r in mres),
                 "all_converged_to_tolerance": all(r.converged() and r.residualNorm() <= w["tol"] for r in mres)}
    n, N = w["n"], prob.rooftopCount()
    line = {
        "metric": "batched solves/s (right-hand sides) at rel. residual 1e-6, rChan-preconditioned COCG, FP64",
        "value": w["rhs"] * args.steps / t, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic plate and 64 plane waves, seed 0",
        "config": {"workload": f"c4: {n}x{n} plate, cell lambda/{w['density']}, {N} unknowns, {w['rhs']} plane "
                               f"waves theta U[0,80] phi U[0,360) TE/TM, COCG + rChan circulant, FP64, all right-hand "
                               f"sides in one solve, to {w['tol']:g}", "unknowns": N, "rhs": w["rhs"],
                   "l2": "working set per batch re-created every step"},
        "iterations": its[0], "true_residual": res_max, "all_converged_to_tolerance": res_max <= w["tol"],
        "e2e": {"value": w["rhs"] * args.steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": 16 * N * w["rhs"],
                "d2h_bytes_per_step": 16 * N * w["rhs"]},
        "gpu_launches": int(L.launch_count() - launches0), "clocks": clk.summary(),
    }
    if mixed:
        line["mixed"] = mixed
        line["mixed_over_fp64"] = mixed["value"] / line["value"]
    print(json.dumps(line))


def plane_wave_vectors(theta_deg, phi_deg, pol):
    """d = [sin t cos p, sin t sin p, -cos t]; TE p = [-sin p, cos p, 0]; TM p = [cos t cos p, cos t sin p, sin t]."""
    t, p = math.radians(theta_deg), math.radians(phi_deg)
    d = np.array([math.sin(t) * math.cos(p), math.sin(t) * math.sin(p), -math.cos(t)])
    if pol == "x":
        e = np.array([1.0, 0.0, 0.0])
    elif pol == "TE":
        e = np.array([-math.sin(p), math.cos(p), 0.0])
    else:
        e = np.array([math.cos(t) * math.cos(p), math.cos(t) * math.sin(p), math.sin(t)])
    return d, e


def matvec_bytes(n_unknowns, P, Q, elem):
    """Algorithmic bytes of one split-FFT product (2-pass schedule): e (2N + 16 PQ + 12 PQ)."""
    return elem * (2 * n_unknowns + 16 * P * Q + 12 * P * Q)


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons in the background."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "500"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 3 + k and r[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def build_plate(R, w, device_rhs=True):
    n = w["n"]
    h = 1.0 / w["density"]
    prob = R.Problem(R.Mesh(n, n, h, h), 2 * math.pi)
    return prob


def solve_plate(R, w, rhs_host=None):
    """One full plate solve. rhs_host: pinned host copy of the excitation for the e2e leg."""
    import torch

    prob = build_plate(R, w)
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    if w["precision"] == "mixed":
        op = R.Operator(prob)
        inner = R.Operator(prob, precision="single")
        exc = R.Excitation.planeWave(prob, direction=d, polarization=p, device=rhs_host is None)
        b = rhs_host if rhs_host is not None else exc.vector()
        pc = R.Preconditioner(prob, kernel=w["pc"], precision="single") if w["pc"] else None
        res = R.Solver(method="fgmres", tolerance=w["tol"], restart=w["restart"], innerTolerance=1e-4,
                       maxIterationCount=20000).solve(op, b, innerOperator=inner, innerPreconditioner=pc)
    else:
        op = R.Operator(prob)
        pc = R.Preconditioner.blockJacobi(prob, (2, 2)) if w["pc"] == "blockJacobi" else None
        exc = R.Excitation.planeWave(prob, direction=d, polarization=p, device=rhs_host is None)
        b = rhs_host if rhs_host is not None else exc.vector()
        res = R.Solver(method=w["method"], tolerance=w["tol"], restart=w["restart"], maxIterationCount=20000,
                       side="right").solve(op, b, preconditioner=pc)
    res._excitation = exc
    rcs = res.radarCrossSection()
    return prob, op, res, rcs


# The precision form's inner solves aim no lower than this relative residual (an FP32 solve reaches it
# safely); each refinement step's inner solve otherwise stops once the outer tolerance will be met.
INNER_FLOOR = 1e-3
# Restart of the precision form's FP32 flexible GMRES in the c2 and c4 arms: the FP64 arm's 50, so that only
# the precision differs (restart 30 measured more inner iterations, 3163 against 2162 on the C2 plate, and
# fewer solves/s at one and at 16 right-hand sides).
MIXED_RESTART = 50
# Classical Gram-Schmidt passes of the precision form's FP32 inner Arnoldi steps (0: the library's default,
# one pass; the FP64 arms keep the reference's two).
INNER_GS_PASSES = 0
# Right-hand sides of the batched arms: the workload's own wave and the rest drawn as the batching form
# draws its waves (theta ~ U[0, 80] deg, phi ~ U[0, 360), TE / TM ~ Bernoulli(1/2), seed 0).
BATCH_RHS = 16


def batch_waves(w, count):
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    if count == 1:
        return d[None], p[None]
    dirs, pols = random_waves(count - 1, np.random.default_rng(0))
    return np.vstack([d[None], dirs]), np.vstack([p[None], pols])


def rcs_of(R, prob, b, x, k, n):
    """Monostatic RCS of right-hand side k of a batched device solve (computeRadarCrossSection.m:18-19)."""
    import ctypes as C

    from rooftop_mom_b200 import _lib as L

    out = C.c_double()
    L.call("rtm_radar_cross_section", prob.wavenumber(), C.c_void_p(b[k * n:(k + 1) * n].data_ptr()),
           C.c_void_p(x[k * n:(k + 1) * n].data_ptr()), n, 1.0, L.DEVICE, C.byref(out))
    return out.value


def solve_arm(R, w, mixed, dirs, pols):
    """One step of an arm on the workload's plate: assembly, spectra, block-Jacobi (2 x 2 faces), the plane
    waves on the device, the solve of all right-hand sides at once to the workload's FP64 true residual, and
    the RCS of each. mixed: FP32 flexible GMRES(MIXED_RESTART) with an FP32 product and FP32 block-Jacobi
    inside FP64 iterative refinement; else FP64 right-preconditioned GMRES(restart) of the workload. Returns (solutions as one
    device tensor, results, RCS values)."""
    import torch

    prob = build_plate(R, w)
    nrhs, n = len(dirs), prob.rooftopCount()
    op = R.Operator(prob, maxRhs=nrhs)
    b = batch_rhs(R, prob, dirs, pols)
    if mixed:
        inner = R.Operator(prob, precision="single", maxRhs=nrhs)
        pc = R.Preconditioner.blockJacobi(prob, (2, 2), precision="single")
        res = R.Solver(method="fgmres", tolerance=w["tol"], restart=MIXED_RESTART, innerTolerance=INNER_FLOOR,
                       gramSchmidtPasses=INNER_GS_PASSES,
                       maxIterationCount=20000).solve(op, b, innerOperator=inner, innerPreconditioner=pc, nrhs=nrhs)
    else:
        pc = R.Preconditioner.blockJacobi(prob, (2, 2))
        res = R.Solver(method="gmres", tolerance=w["tol"], restart=w["restart"], maxIterationCount=20000,
                       side="right").solve(op, b, preconditioner=pc, nrhs=nrhs)
    res = res if isinstance(res, list) else [res]
    x = torch.cat([r.solution().reshape(-1) for r in res]) if nrhs > 1 else res[0].solution().reshape(-1)
    rcs = [rcs_of(R, prob, b, x, k, n) for k in range(nrhs)]
    return x, res, rcs


def time_arm(R, w, mixed, dirs, pols, steps, warmup):
    """Solves/s of an arm (right-hand sides solved per second), CUDA events around `steps` steps."""
    import torch

    for _ in range(warmup):
        solve_arm(R, w, mixed, dirs, pols)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = []
    for _ in range(steps):
        out.append(solve_arm(R, w, mixed, dirs, pols))
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    x, res, rcs = out[-1]
    return {"value": len(dirs) * steps / t, "unit": "solves/s", "rhs": len(dirs), "steps": steps,
            "ms_per_step": t / steps * 1e3,
            "iterations": max(r.iterationCount() for r in res),
            "refinements": max(r.refinements() for r in res) if mixed else 0,
            "true_residual": max(r.residualNorm() for r in res),
            "all_converged_to_tolerance": all(r.converged() and r.residualNorm() <= w["tol"] for r in res)}, x, rcs


def precision_arms(R, w, steps, warmup):
    """The metric's "mixed vs FP64" on the workload's plate: FP64 and mixed, one right-hand side and a batch
    of BATCH_RHS, each to the FP64 true residual of the workload. Errors of the currents and RCS are taken
    against an FP64 solve of the same right-hand sides driven to 1e-10."""
    import torch

    d1, p1 = batch_waves(w, 1)
    dB, pB = batch_waves(w, BATCH_RHS)
    arms = {}
    sols = {}
    for name, mixed, (dd, pp) in (("fp64", False, (d1, p1)), ("mixed", True, (d1, p1)),
                                  ("fp64_batched", False, (dB, pB)), ("mixed_batched", True, (dB, pB))):
        arms[name], x, rcs = time_arm(R, w, mixed, dd, pp, steps, warmup)
        sols[name] = (x, rcs)
    ref_w = dict(w, tol=1e-10)
    xr, _, rcs_r = solve_arm(R, ref_w, False, dB, pB)
    n = xr.numel() // BATCH_RHS
    for name, (x, rcs) in sols.items():
        cur = max(float((x[k * n:(k + 1) * n] - xr[k * n:(k + 1) * n]).norm() / xr[k * n:(k + 1) * n].norm())
                  for k in range(len(rcs)))
        rc = max(abs(a - b) / abs(b) for a, b in zip(rcs, rcs_r))
        arms[name]["error_vs_fp64_1e-10"] = {"current_rel": cur, "rcs_rel": rc}
    torch.cuda.synchronize()
    return arms


def precision_error(R, w):
    """The precision form's error: the mixed solve against an FP64 GPU solve of the same plate (FP64
    GMRES with the same restart to a residual 10 times below the form's)."""
    prob, op, res, rcs = solve_plate(R, w)
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    exc = R.Excitation.planeWave(prob, direction=d, polarization=p, device=True)
    ref = R.Solver(method="gmres", tolerance=w["tol"] / 10, restart=w["restart"], maxIterationCount=40000).solve(
        op, exc.vector())
    ref._excitation = exc
    x, x64 = res.solution(), ref.solution()
    err = float((x - x64).norm() / x64.norm()) if hasattr(x, "norm") else float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
    rcs64 = ref.radarCrossSection()
    return {"current_rel": err, "rcs_rel": abs(rcs - rcs64) / abs(rcs64), "fp64_residual": ref.residualNorm(),
            "fp64_iterations": ref.iterationCount(), "mixed_residual": res.residualNorm()}


def roofline_matvec(R, w, steps, stream_ptr=None):
    """Average device time of the split-FFT product of the workload: `per_graph` back-to-back applies captured
    in one CUDA graph on a side stream, the graph replayed `reps` times between CUDA events on that stream
    (a loop of library calls would time the host's launch overhead at small grids). Also returns the time
    of the same applies launched one by one from the host (`host_loop_seconds`)."""
    import ctypes as C

    import torch

    from rooftop_mom_b200 import _lib as L

    prob = build_plate(R, w)
    prec = "double" if w["precision"] == "double" else "single"
    op = R.Operator(prob, precision=prec)
    inf = op.info()
    N = prob.rooftopCount()
    dt = torch.complex128 if prec == "double" else torch.complex64
    x = torch.randn(N, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    side = torch.cuda.Stream()

    def one():
        L.call("rtm_operator_apply", op.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), N, 1, L.DEVICE,
               C.c_void_p(side.cuda_stream))

    with torch.cuda.stream(side):
        for _ in range(5):
            one()
    torch.cuda.synchronize()
    reps = max(20, steps * 10)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(side):
        e0.record(side)
        for _ in range(reps):
            one()
        e1.record(side)
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1) / 1e3 / reps
    per_graph, t_graph = 20, None
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side, capture_error_mode="relaxed"):
            for _ in range(per_graph):
                one()
        g.replay()
        torch.cuda.synchronize()
        with torch.cuda.stream(side):
            e0.record(side)
            for _ in range(max(3, reps // per_graph)):
                g.replay()
            e1.record(side)
        torch.cuda.synchronize()
        t_graph = e0.elapsed_time(e1) / 1e3 / (max(3, reps // per_graph) * per_graph)
        del g
    except Exception:  # noqa: BLE001 - report the host loop alone
        t_graph = None
    elem = 16 if prec == "double" else 8
    B = matvec_bytes(N, inf["fft_x"], inf["fft_y"], elem)
    return {"seconds": t_graph if t_graph is not None else t_loop, "graph": t_graph is not None,
            "host_loop_seconds": t_loop, "bytes": B, "P": inf["fft_x"], "Q": inf["fft_y"], "N": N,
            "precision": prec}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


# ---------------------------------------------------------------------------------------------
# CPU leg: the oracle (numpy/scipy restatement of the reference's MATLAB path) on the host cores.
def cpu_matvec_ms(apply, v):
    """The oracle's product timed as benchmarks/measureThreadScaling.m:58-74 times it: one warm-up, then the
    median of 5 (milliseconds)."""
    apply(v)
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        apply(v)
        times.append(time.perf_counter() - t0)
    return float(np.median(times)) * 1e3


def cpu_sample(w):
    """Times the oracle's setup (assembly, spectra, block-Jacobi, plane wave) and one whole restart cycle of
    its solver (GMRES: `restart` iterations, so the cost of the Gram-Schmidt passes, which grows with the
    step within a cycle, is averaged over a full cycle; COCG: 50 iterations). Returns (setup s, s per
    iteration, product ms)."""
    from oracle import assembly as A, blockjacobi as BJ, excitation as EX, geometry as G, solvers as OS, spectra as S

    n, h, k = w["n"], 1.0 / w["density"], 2 * math.pi
    t0 = time.perf_counter()
    gen = A.generate(n, n, h, h, k)
    rt = G.Rooftops(n, n, h, h, 8)
    sub = S.subband_spectra(gen, h, h)
    pc = BJ.BlockJacobi(gen, rt, 2, 2).apply if w["pc"] == "blockJacobi" else None
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    b = EX.plane_wave(rt, k, d, p, 1.0)
    t_setup = time.perf_counter() - t0
    apply = lambda v: S.split_apply(rt, sub, rt.content, v)  # noqa: E731
    t0 = time.perf_counter()
    if w["method"] == "cg":
        m = 50
        OS.cocg_iterate(apply, b, None, 1e-300, m, pc)
    else:
        # right preconditioning as the GPU solve: A M u = b
        m = w["restart"]
        Ar = (lambda v: apply(pc(v))) if pc else apply
        OS.gmres_iterate(Ar, b, None, 1e-300, m, m)
    t_iter = (time.perf_counter() - t0) / m
    return t_setup, t_iter, cpu_matvec_ms(apply, b)


def cpu_full_solve(w):
    """A whole oracle solve of a small plate, to its tolerance: (seconds, iterations, product ms)."""
    from oracle import assembly as A, blockjacobi as BJ, excitation as EX, geometry as G, solvers as OS, spectra as S

    n, h, k = w["n"], 1.0 / w["density"], 2 * math.pi
    t0 = time.perf_counter()
    gen = A.generate(n, n, h, h, k)
    rt = G.Rooftops(n, n, h, h, 8)
    sub = S.subband_spectra(gen, h, h)
    pc = BJ.BlockJacobi(gen, rt, 2, 2).apply if w["pc"] == "blockJacobi" else None
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    b = EX.plane_wave(rt, k, d, p, 1.0)
    apply = lambda v: S.split_apply(rt, sub, rt.content, v)  # noqa: E731
    out = OS.solve("cg" if w["method"] == "cg" else "gmres", apply, b, tol=w["tol"], maxit=20000,
                   restart=w["restart"], precond=pc)
    t_solve = time.perf_counter() - t0
    return t_solve, out.iteration_count, cpu_matvec_ms(apply, b)


# Plates small enough for the CPU legs to run whole solves instead of extrapolating a sample.
FULL_SOLVE_MAX_FACES = 64


def run_reference(args, w):
    """--impl reference: the oracle's CPU path (the reference's MATLAB restated) on all host threads. Small
    plates run whole solves per step. Larger ones time, per step, the setup and one whole restart cycle,
    and give solves/s for a solve of the oracle's own iteration count (ORACLE_ITERATIONS, from one whole
    oracle solve of the workload); ms_per_step is the wall time of the step actually run."""
    cores = os.cpu_count() or 1
    full = w["n"] <= FULL_SOLVE_MAX_FACES
    iters = ORACLE_ITERATIONS.get(args.workload)
    solve_times, walls = [], []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if full:
            t_solve, iters, mv_ms = cpu_full_solve(w)
        else:
            t_setup, t_iter, mv_ms = cpu_sample(w)
            t_solve = t_setup + iters * t_iter
        if step >= args.warmup:
            solve_times.append(t_solve)
            walls.append(time.perf_counter() - t0)
    t = float(np.median(solve_times))
    value = 1.0 / t
    if full:
        sample = (f"numpy/scipy oracle (the reference's MATLAB path restated), per step one whole solve: assembly, "
                  f"spectra, plane wave and {iters} iterations to the tolerance (measured, not extrapolated)")
    else:
        sample = (f"numpy/scipy oracle (the reference's MATLAB path restated), per step: assembly + spectra + "
                  f"preconditioner + plane wave timed, plus one whole restart cycle of the solver timed; solves/s "
                  f"is for setup + {iters} iterations at that per-iteration time, {iters} being "
                  f"{ORACLE_ITERATION_SOURCE[args.workload]} (extrapolated: a whole solve takes "
                  f"{t:.0f} s)")
    line = {
        # n_gpus is the N of the launch this line is compared with; the arm itself runs on host cores only
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "device": "host CPU cores (no GPU used)",
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(walls)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": config_of(args, w), "seconds_per_solve": t, "extrapolated": not full,
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample,
                         "matvec_ms": mv_ms},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# Iteration counts of whole oracle solves of the workloads (the oracle's own; c1 runs whole solves per
# step instead). c2: oracle/solvers.gmres_iterate with the block-Jacobi oracle on the right, to 1e-6, as
# `python bench.py --impl reference --workload c2 --full-solve` runs it.
ORACLE_ITERATIONS = {"c2": 2511, "c3": 9220}
ORACLE_ITERATION_SOURCE = {
    "c2": "the count of one whole oracle solve of this plate (block-Jacobi GMRES(50) to 1e-6)",
    # the reference has no precision form; its path for this plate is FP64 GMRES(30), which the oracle
    # cannot run to the end within hours on the host
    "c3": "the count of an FP64 GMRES(30) solve of this plate on the GPU to 1e-9 (a whole oracle solve of "
          "2.1 M unknowns takes hours; the count to the workload's 1e-8 is lower, so the CPU time is an upper "
          "bound)",
}


def run_reference_full(args, w):
    """One whole oracle solve of the workload, to the workload's tolerance: its iteration count is the
    ORACLE_ITERATIONS entry of the workload."""
    t, its, mv = cpu_full_solve(w)
    print(json.dumps({"impl": "reference", "workload": args.workload, "seconds": t, "iterations": its,
                      "matvec_ms": mv, "cores": os.cpu_count()}))


METRIC = "solves/s at rel. residual 1e-6, mixed vs FP64 GPU; matvec HBM GB/s; p99 ms"

# DRAM bytes (read + write) of one product, summed over its three kernels, from one ncu capture each
# (profiles/product_fast_path.md); None where no capture was made.
TRAFFIC = {"c2": 23.2e6, "c3": 200.3e6}


def config_of(args, w):
    n = w["n"]
    return {"workload": f"{args.workload}: {n}x{n} plate, cell lambda/{w['density']}, "
                        f"{(n - 1) * n * 2} unknowns, plane wave theta={w['theta']} phi={w['phi']} {w['pol']}, "
                        f"{w['pc'] or 'no'} preconditioner, {w['method']}({w['restart']}) to {w['tol']:g}, "
                        f"{w['precision']}",
            "unknowns": (n - 1) * n * 2, "grid": [n, n], "tolerance": w["tol"], "method": w["method"],
            "restart": w["restart"], "preconditioner": w["pc"], "precision": w["precision"],
            "parallelism": f"replicas{args.gpus}", "l2": "working set per solve re-created every step"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-arms", action="store_true", help="skip the mixed / batched arms of c2")
    ap.add_argument("--full-solve", action="store_true",
                    help="with --impl reference: one whole oracle solve of the workload (its iteration count)")
    ap.add_argument("--once", action="store_true",
                    help="one untimed solve of the workload, no JSON line (the command profiler captures run)")
    ap.add_argument("--arm", choices=["fp64", "mixed", "fp64_batched", "mixed_batched"],
                    help="with --once: one step of that arm of the workload's plate instead")
    ap.add_argument("--matvec", action="store_true",
                    help="only the product of the workload, applied --steps times (the command profiler captures run)")
    ap.add_argument("--assembly", action="store_true",
                    help="time the generator assembly of the workload's plate (FP64 GFLOP/s of the far lattice)")
    ap.add_argument("--requests", type=int, default=100, help="c5: requests in the stream (2000 in the full form)")
    ap.add_argument("--slots", type=int, default=8, help="c5: requests on the device at once")
    ap.add_argument("--serving-precision", default="double", choices=["double", "mixed"])
    ap.add_argument("--serving-sizes", default="powerOfTwo", choices=["reference", "powerOfTwo", "autotune"],
                    help="c5: the server's transform-size policy")
    ap.add_argument("--serving-batch", type=int, default=0,
                    help="c5: requests a worker solves together as one plate batch (0: each alone)")
    ap.add_argument("--serving-requests", type=int, default=32,
                    help="c2: requests of the short serving stream in the default line (0: none)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.workload == "c4u" and args.once:
        # one batched step of the c4u plates (the profiler captures run)
        import rooftop_mom_b200 as R

        R.load()
        res, _, fused, ts = plate_batch_step(R, w, True)
        print(f"c4u: {len(res)} plates in one batch (fused {fused}), iterations {max(r.iterationCount() for r in res)}, "
              f"residual {max(r.residualNorm() for r in res):.3e}, solves {ts * 1e3:.1f} ms")
        return
    if args.workload in ("c4", "c4u", "c5") and not args.matvec:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": f"the CPU oracle arm times single-plate solves "
                                                                  f"(c1, c2, c3), not {args.workload}"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            {"c4": lambda: run_batched(args, w), "c4u": lambda: run_plate_batch(args, w),
             "c5": lambda: run_serving(args)}[args.workload]()
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference_full(args, w) if args.full_solve else run_reference(args, w)
        return

    import torch

    torch.cuda.set_device(local)
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    R.load()
    L.call("rtm_set_device", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.assembly:
        n = w["n"]
        h = 1.0 / w["density"]
        times = []
        for k in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            R.Problem(R.Mesh(n, n, h, h), 2 * math.pi).generators()
            torch.cuda.synchronize()
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        t = float(np.median(times))
        # 120 FP64 flops per far-lattice kernel value (the 4 x 7 moment multiply-adds and the distance and
        # phase), order_far^2 values per lattice block, (n + 1)^2 blocks
        values = 8 * 8 * (n + 1) ** 2
        print(f"assembly {n}x{n}: {t * 1e3:.2f} ms, {values / 1e6:.1f} M far-lattice values, "
              f"{120 * values / t / 1e9:.0f} GFLOP/s FP64 (algorithmic)")
        return
    if args.matvec:
        rf = roofline_matvec(R, w, args.steps)
        print(f"product {rf['precision']} {rf['P']}x{rf['Q']}: {rf['seconds'] * 1e6:.1f} us "
              f"({'graph' if rf['graph'] else 'host loop'}; host loop {rf['host_loop_seconds'] * 1e6:.1f} us), "
              f"{rf['bytes'] / rf['seconds'] / 1e9:.0f} GB/s")
        return
    if args.once:
        if args.arm:
            # one step of an arm of the workload's plate (the profiler captures run)
            count = BATCH_RHS if args.arm.endswith("batched") else 1
            d, p = batch_waves(w, count)
            _, res, rcs = solve_arm(R, w, args.arm.startswith("mixed"), d, p)
            torch.cuda.synchronize()
            print(f"{args.arm}: {count} right-hand sides, iterations {max(r.iterationCount() for r in res)}, "
                  f"residual {max(r.residualNorm() for r in res):.3e}")
            return
        _, _, res, rcs = solve_plate(R, w)
        torch.cuda.synchronize()
        print(f"iterations {res.iterationCount()} residual {res.residualNorm():.3e} rcs {rcs:.6g}")
        return

    # warm-up: context, FFT tables, kernels; the clock sampler starts before the last warm-up step so that
    # its start-up stays out of the timed region
    for _ in range(max(0, args.warmup - 1)):
        solve_plate(R, w)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        if args.warmup > 0:
            solve_plate(R, w)
        torch.cuda.synchronize()

        # timed region: K full solves with the inputs on the device
        launches0 = L.launch_count()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        its, residuals = [], []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lat = []
        for _ in range(args.steps):
            s0 = time.perf_counter()
            prob, op, res, rcs = solve_plate(R, w)
            lat.append(time.perf_counter() - s0)
            its.append(res.iterationCount())
            residuals.append(res.residualNorm())
        e1.record()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t_dev = e0.elapsed_time(e1) / 1e3
    launches = L.launch_count() - launches0
    t_max = t_dev
    if dist:
        tt = torch.tensor([t_dev], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * args.steps / t_max
    ok = all(r <= w["tol"] for r in residuals)

    # e2e: the public API with the right-hand side from pinned host memory and the solution back to it
    d, p = plane_wave_vectors(w["theta"], w["phi"], w["pol"])
    prob0 = build_plate(R, w)
    b_host = R.Excitation.planeWave(prob0, direction=d, polarization=p).vector()
    pinned = torch.from_numpy(b_host).pin_memory().numpy()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e2[0].record()
    for _ in range(args.steps):
        solve_plate(R, w, rhs_host=pinned)
    e2[1].record()
    torch.cuda.synchronize()
    t_e2e = e2[0].elapsed_time(e2[1]) / 1e3
    if dist:
        tt = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    N = prob0.rooftopCount()

    # roofline of the product (the kernel whose bandwidth the metric names)
    rf = roofline_matvec(R, w, args.steps)
    hbm, kind = peaks()
    achieved = rf["bytes"] / rf["seconds"] / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128" if w["precision"] == "double" else "c64/c128",
        "data": "synthetic plate and plane wave (no dataset)", "config": config_of(args, w),
        "iterations": its[0], "true_residual": max(residuals), "all_converged_to_tolerance": ok,
        "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "matvec_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": kind, "kernel": f"split-FFT product ({rf['precision']}, {rf['P']}x{rf['Q']} grid, "
                                                   f"3 kernels)", "bytes_per_launch": rf["bytes"],
                     "seconds_per_launch": rf["seconds"], "timed_as": "CUDA graph of 20 applies" if rf["graph"]
                     else "host loop", "host_loop_seconds_per_launch": rf["host_loop_seconds"],
                     "traffic": TRAFFIC.get(args.workload)},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": 16 * N,
                "d2h_bytes_per_step": 16 * N},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        if w["n"] <= FULL_SOLVE_MAX_FACES:
            t_cpu, cpu_its, mv_ms = cpu_full_solve(w)
            sample = f"one whole oracle solve: assembly, spectra, plane wave and {cpu_its} iterations (measured)"
        else:
            iters = ORACLE_ITERATIONS[args.workload]
            t_setup, t_iter, mv_ms = cpu_sample(w)
            t_cpu = t_setup + iters * t_iter
            sample = (f"oracle setup (assembly, spectra, preconditioner, plane wave) timed once, plus one whole "
                      f"restart cycle timed, for a solve of {iters} iterations "
                      f"({ORACLE_ITERATION_SOURCE[args.workload]}): {t_setup:.2f} s + {iters} x "
                      f"{t_iter * 1e3:.1f} ms (extrapolated)")
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": sample, "matvec_ms": mv_ms}
    if rank == 0 and world == 1 and w["precision"] == "mixed":
        line["error_vs_fp64"] = precision_error(R, w)
    if args.workload == "c2" and args.serving_requests > 0 and world == 1:
        # the metric's p50 / p99: a short serving stream (c5's mix), FP64 and mixed
        line["serving"] = {p: serve_stream(R, args.serving_requests, args.slots, p, args.serving_sizes)
                           for p in ("double", "mixed")}
    if args.workload == "c2" and not args.no_arms and world == 1:
        # the metric's "mixed vs FP64": both precisions, single and batched, on the same plate (one GPU: the
        # replicas of a multi-GPU run measure the solve rate alone)
        arms = precision_arms(R, w, min(args.steps, 5), min(args.warmup, 2))
        line["arms"] = arms
        # the target's ratio: the mixed-precision batched solver against the plain FP64 GPU path (one
        # right-hand side); then like for like, the same right-hand sides in both precisions
        line["mixed_over_fp64"] = arms["mixed_batched"]["value"] / arms["fp64"]["value"]
        line["mixed_over_fp64_same_batch"] = arms["mixed_batched"]["value"] / arms["fp64_batched"]["value"]
        line["mixed_over_fp64_single_rhs"] = arms["mixed"]["value"] / arms["fp64"]["value"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
