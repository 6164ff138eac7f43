"""Benchmark of the rooftop-mom solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|c3|c4|c1]

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
    "c3": dict(n=1024, density=15, theta=30.0, phi=0.0, pol="TE", method="fgmres", tol=1e-8, restart=30,
               pc=None, precision="mixed"),
}


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
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
        res = R.Solver(method="fgmres", tolerance=w["tol"], restart=w["restart"], innerTolerance=1e-4,
                       maxIterationCount=20000).solve(op, b, innerOperator=inner)
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


def roofline_matvec(R, w, steps, stream_ptr):
    """Average device time of the split-FFT product of the workload (CUDA events on its stream)."""
    import torch

    prob = build_plate(R, w)
    prec = "double" if w["precision"] == "double" else "single"
    op = R.Operator(prob, precision=prec)
    inf = op.info()
    N = prob.rooftopCount()
    dt = torch.complex128 if prec == "double" else torch.complex64
    x = torch.randn(N, dtype=dt, device="cuda")
    y = torch.empty_like(x)
    import ctypes as C

    from rooftop_mom_b200 import _lib as L

    def one():
        L.call("rtm_operator_apply", op.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), N, 1, L.DEVICE,
               C.c_void_p(stream_ptr))

    for _ in range(5):
        one()
    torch.cuda.synchronize()
    reps = max(20, steps * 10)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        one()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    elem = 16 if prec == "double" else 8
    B = matvec_bytes(N, inf["fft_x"], inf["fft_y"], elem)
    return {"seconds": t, "bytes": B, "P": inf["fft_x"], "Q": inf["fft_y"], "N": N, "precision": prec}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


# ---------------------------------------------------------------------------------------------
# CPU leg: the oracle (numpy/scipy restatement of the reference's MATLAB path) on the host cores.
def cpu_sample(w, iterations_gpu, sample_iterations=25):
    """Times the oracle's setup (assembly, spectra, block-Jacobi, plane wave) and a bounded number of
    its GMRES iterations; a full solve is setup + iterations_gpu x per-iteration time."""
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
    apply = lambda v: S.split_apply(rt, sub, rt.content, v)
    m = max(1, sample_iterations)
    t0 = time.perf_counter()
    if w["method"] == "cg":
        OS.cocg_iterate(apply, b, None, 1e-300, m, pc)
    else:
        # right preconditioning as the GPU solve: A M u = b
        Ar = (lambda v: apply(pc(v))) if pc else apply
        OS.gmres_iterate(Ar, b, None, 1e-300, m, w["restart"])
    t_iter = (time.perf_counter() - t0) / m
    return t_setup, t_iter


def run_reference(args, w):
    """--impl reference: the oracle's CPU path, all host threads, bounded sample per step."""
    cores = os.cpu_count() or 1
    iters = REFERENCE_ITERATIONS.get(args.workload)
    times = []
    for step in range(args.warmup + args.steps):
        t_setup, t_iter = cpu_sample(w, iters, sample_iterations=10)
        if step >= args.warmup:
            times.append(t_setup + iters * t_iter)
    t = float(np.median(times))
    value = 1.0 / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": config_of(args, w),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"numpy/scipy oracle (the reference's MATLAB path restated), per step: assembly + "
                                   f"spectra + preconditioner + plane wave timed, plus 10 GMRES/COCG iterations "
                                   f"timed and scaled to the {iters} iterations of the same solve (extrapolated)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# Iteration counts of the default solves (FP64 GPU, same algorithm as the oracle), used to scale the
# CPU leg's bounded sample to a full solve.
REFERENCE_ITERATIONS = {"c2": 2511, "c1": 300, "c3": 300}

METRIC = "solves/s at rel. residual 1e-6, mixed vs FP64 GPU; matvec HBM GB/s; p99 ms"


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
    ap.add_argument("--once", action="store_true",
                    help="one untimed solve of the workload, no JSON line (the command profiler captures run)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, w)
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

    if args.once:
        _, _, res, rcs = solve_plate(R, w)
        torch.cuda.synchronize()
        print(f"iterations {res.iterationCount()} residual {res.residualNorm():.3e} rcs {rcs:.6g}")
        return

    # warm-up: context, FFT tables, kernels
    for _ in range(args.warmup):
        solve_plate(R, w)
    torch.cuda.synchronize()

    # timed region: K full solves with the inputs on the device
    launches0 = L.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    its, residuals = [], []
    with Clocks(local) as clk:
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
    stream = torch.cuda.current_stream().cuda_stream
    rf = roofline_matvec(R, w, args.steps, stream)
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
                     "seconds_per_launch": rf["seconds"], "traffic": None},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": 16 * N,
                "d2h_bytes_per_step": 16 * N},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        t_setup, t_iter = cpu_sample(w, its[0], sample_iterations=20)
        t_cpu = t_setup + its[0] * t_iter
        line["cpu_baseline"] = {
            "value": 1.0 / t_cpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle setup (assembly, spectra, preconditioner, plane wave) timed once, plus 20 iterations "
                      f"timed and scaled to the GPU solve's {its[0]} iterations: {t_setup:.2f} s + "
                      f"{its[0]} x {t_iter * 1e3:.1f} ms (extrapolated)"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
