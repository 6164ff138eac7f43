"""The synthetic workloads of bench.py (no GPU): plane-wave geometry of the configurations, the seeded
64-wave batch, the seeded request stream and its preconditioner choice."""
from __future__ import annotations

import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def test_plane_wave_vectors_are_unit_and_perpendicular():
    import bench

    for pol in ("TE", "TM", "x"):
        for theta, phi in ((0, 0), (30, 0), (55, 130), (80, 359)):
            d, p = bench.plane_wave_vectors(theta, phi, pol)
            assert abs(np.linalg.norm(d) - 1) < 1e-15 and abs(np.linalg.norm(p) - 1) < 1e-15
            if pol != "x" or theta == 0:
                assert abs(d @ p) < 1e-15
    d, p = bench.plane_wave_vectors(30, 0, "TE")  # the C2 wave: d = [0.5, 0, -0.866], p = [0, 1, 0]
    assert np.allclose(d, [0.5, 0, -math.sqrt(0.75)]) and np.allclose(p, [0, 1, 0])


def test_the_batch_of_waves_is_seeded_and_within_its_ranges():
    import bench

    d1, p1 = bench.random_waves(64, np.random.default_rng(0))
    d2, p2 = bench.random_waves(64, np.random.default_rng(0))
    assert np.array_equal(d1, d2) and np.array_equal(p1, p2)
    theta = np.degrees(np.arccos(-d1[:, 2]))
    assert theta.min() >= 0 and theta.max() <= 80 + 1e-9
    assert np.all(np.abs(np.einsum("ij,ij->i", d1, p1)) < 1e-15)


def test_the_request_stream_is_seeded_and_takes_the_rchan_circulant():
    import bench
    import rooftop_mom_b200 as R
    a = bench.serving_requests(R, 50, 0)
    b = bench.serving_requests(R, 50, 0)
    for qa, qb in zip(a, b):
        sa, sb = qa.struct, qb.struct
        assert (sa.count_x, sa.count_y, sa.size_x, sa.wavenumber) == (sb.count_x, sb.count_y, sb.size_x, sb.wavenumber)
        assert 16 <= sa.count_x <= 768 and (sa.count_y == 1 or 16 <= sa.count_y <= 768)
        # strips carry the delta gap, plates the plane wave
        assert (sa.count_y == 1) == (sa.excitation == 1)
        assert sa.preconditioner == 2 and sa.method == 0  # rChan COCG on every face grid
        lam = 2 * math.pi / sa.wavenumber
        assert 10 - 1e-9 <= lam / sa.size_x <= 25 + 1e-9


def test_the_reference_arm_prints_its_line_on_the_host():
    """bench.py --impl reference runs the oracle's CPU path (no GPU) and prints the contract's line: the
    launch's N, the metric and unit of our arm, a cpu_baseline and an e2e object."""
    import json
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0"], check=True, capture_output=True, text=True,
                         timeout=600, cwd=root).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["unit"] == "solves/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_takes_the_oracle_iteration_count_of_each_sampled_workload():
    """The reference arm extrapolates a sampled step to a whole solve with the oracle's own iteration count
    (not the GPU's) for every workload too large to run whole per step, and says where the count comes
    from."""
    import bench

    for name, w in bench.WORKLOADS.items():
        if name in ("c4", "c4u", "c5") or w["n"] <= bench.FULL_SOLVE_MAX_FACES:
            continue
        assert bench.ORACLE_ITERATIONS[name] > 0
        assert bench.ORACLE_ITERATION_SOURCE[name]
