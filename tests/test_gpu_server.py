"""The serving form on the GPU: each request's result is the same alone and in a mix of other requests
running at the same time, equals the direct API solve of the same plate, requests overlap on the device,
the byte budget serialises what does not fit together, queued requests can be cancelled, and the
mixed-precision server stays within 1e-5 of the FP64 currents."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAM = 1.0
K = 2 * math.pi / LAM
TOL = 1e-8


def _plate(cx, cy, d=(0.5, 0.0, -math.sqrt(0.75)), p=(0.0, 1.0, 0.0), **kw):
    import rooftop_mom_b200 as R

    return R.Request.planeWave(cx, cy, LAM / 20, LAM / 20, K, direction=d, polarization=p, tolerance=TOL,
                               keepCurrent=True, **kw)


def _strip(cx, **kw):
    import rooftop_mom_b200 as R

    return R.Request.deltaGap(cx, 1, LAM / 20, LAM / 20, K, portDirection="x", tolerance=TOL, keepCurrent=True,
                              **kw)


def _mix():
    return [_plate(32, 28), _strip(41), _plate(17, 29, method="cg"), _plate(48, 40), _strip(64, method="cg"),
            _plate(20, 20, preconditioner=None), _plate(36, 12)]


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_results_are_the_same_alone_and_in_the_mix():
    import rooftop_mom_b200 as R

    with R.Server(maxActive=4) as srv:
        alone = [srv.wait(srv.submit(q)) for q in (_plate(24, 20), _strip(33))]
        mix = _mix()
        ids = [srv.submit(q) for q in mix[:3]]
        again = [srv.submit(_plate(24, 20))]
        ids += [srv.submit(q) for q in mix[3:]]
        again.append(srv.submit(_strip(33)))
        together = [srv.wait(r) for r in again]
        others = [srv.wait(r) for r in ids]
    for a, b in zip(alone, together):
        assert a["state"] == b["state"] == "done"
        assert a["converged"] and b["converged"]
        assert a["iterations"] == b["iterations"]
        assert _rel(b["current"], a["current"]) < 1e-12
        assert a["rcs"] == pytest.approx(b["rcs"], rel=1e-12)
        assert abs(a["impedance"] - b["impedance"]) <= 1e-12 * max(1.0, abs(a["impedance"]))
    assert all(o["state"] == "done" and o["converged"] and o["residual"] <= TOL for o in others)


def test_served_plate_equals_the_direct_solve():
    import rooftop_mom_b200 as R

    d, p = (0.5, 0.0, -math.sqrt(0.75)), (0.0, 1.0, 0.0)
    with R.Server(maxActive=2) as srv:
        served = srv.wait(srv.submit(_plate(30, 26, d=d, p=p)))
    prob = R.Problem(R.Mesh(30, 26, LAM / 20, LAM / 20), K)
    op = R.Operator(prob)
    pc = R.Preconditioner.blockJacobi(prob)
    exc = R.Excitation.planeWave(prob, direction=d, polarization=p)
    res = R.Solver(method="gmres", tolerance=TOL, restart=50, maxIterationCount=10000, side="right").solve(
        op, exc, preconditioner=pc)
    assert served["iterations"] == res.iterationCount()
    assert _rel(served["current"], res.solution()) < 1e-12
    assert served["rcs"] == pytest.approx(res.radarCrossSection(), rel=1e-10)


def test_admitted_requests_overlap_on_the_device():
    import rooftop_mom_b200 as R

    with R.Server(maxActive=4) as srv:
        ids = [srv.submit(_plate(40, 40)) for _ in range(6)]
        res = [srv.wait(r) for r in ids]
    spans = sorted((r["started"], r["finished"]) for r in res)
    overlaps = sum(1 for a, b in zip(spans, spans[1:]) if b[0] < a[1])
    assert overlaps >= 1


def test_the_budget_serialises_requests_that_do_not_fit_together():
    import rooftop_mom_b200 as R

    with R.Server(budgetBytes=1e9, maxActive=8) as srv:
        probe = srv.poll(srv.submit(_plate(48, 48)), wait=math.inf)["bytes"]
    with R.Server(budgetBytes=1.5 * probe, maxActive=8) as srv:
        res = [srv.wait(r) for r in [srv.submit(_plate(48, 48)) for _ in range(3)]]
    spans = sorted((r["started"], r["finished"]) for r in res)
    assert all(b[0] >= a[1] for a, b in zip(spans, spans[1:]))
    assert all(r["state"] == "done" for r in res)


def test_queued_requests_can_be_cancelled():
    import rooftop_mom_b200 as R

    with R.Server(maxActive=1) as srv:
        ids = [srv.submit(_plate(40, 36)) for _ in range(4)]
        srv.cancel(ids[-1])
        res = [srv.wait(r) for r in ids]
    assert res[-1]["state"] == "cancelled"
    assert all(r["state"] == "done" for r in res[:-1])


def test_mixed_precision_server_stays_close_to_fp64():
    import rooftop_mom_b200 as R

    qs = [_plate(32, 28), _strip(41)]
    with R.Server(maxActive=2) as srv:
        ref = [srv.wait(srv.submit(q)) for q in qs]
    with R.Server(maxActive=2, precision="single") as srv:
        mixed = [srv.wait(srv.submit(q)) for q in qs]
    for a, b in zip(ref, mixed):
        assert b["state"] == "done" and b["converged"] and b["residual"] <= TOL
        assert _rel(b["current"], a["current"]) < 1e-5


def test_a_circulant_request_equals_the_direct_cocg_solve():
    import rooftop_mom_b200 as R

    # exactly unit vectors: the Python excitation normalises them, the request takes them as given
    d, p = (0.0, 0.0, -1.0), (0.0, 1.0, 0.0)
    with R.Server(maxActive=2) as srv:
        served = srv.wait(srv.submit(_plate(32, 28, d=d, p=p, method="cg", preconditioner="rChan")))
    prob = R.Problem(R.Mesh(32, 28, LAM / 20, LAM / 20), K)
    op = R.Operator(prob)
    pc = R.Preconditioner(prob, kernel="rChan")
    exc = R.Excitation.planeWave(prob, direction=d, polarization=p)
    res = R.Solver(method="cg", tolerance=TOL, maxIterationCount=10000).solve(op, exc, preconditioner=pc)
    assert served["state"] == "done" and served["converged"]
    assert served["iterations"] == res.iterationCount()
    assert _rel(served["current"], res.solution()) < 1e-12


@pytest.mark.parametrize("policy", ["powerOfTwo", "autotune"])
def test_transform_size_policies_give_the_reference_sizes_results(policy):
    """A server whose plates take power-of-two or autotuned transform grids (a larger grid gives the same
    product up to rounding) returns the currents of the reference-size server within the solve tolerance,
    for plates whose face counts are not powers of two, and strips unchanged."""
    import rooftop_mom_b200 as R

    reqs = [_plate(37, 30), _plate(45, 23, method="cg"), _strip(41)]
    with R.Server(budgetBytes=50e9, maxActive=3) as ref_srv:
        ref = [ref_srv.wait(ref_srv.submit(q), release=True) for q in reqs]
    R.clearTuning()
    try:
        with R.Server(budgetBytes=50e9, maxActive=3, transformSizes=policy) as srv:
            got = [srv.wait(srv.submit(q), release=True) for q in reqs]
    finally:
        R.clearTuning()
    for a, b in zip(got, ref):
        assert a["state"] == "done" and a["converged"]
        assert _rel(a["current"], b["current"]) < 1e-6


def test_the_mixed_server_converges_on_large_plates():
    """FP32 COCG with the rChan circulant can diverge on large plates; the mixed server's refinement then
    hands the solve to FP64 COCG from its iterate. Every request converges to its FP64 tolerance and its
    current stays within the tolerance's reach of the FP64 server's."""
    import rooftop_mom_b200 as R

    reqs = [R.Request.planeWave(n, m, LAM / 20, LAM / 20, K, direction=(0.5, 0.0, -math.sqrt(0.75)),
                                polarization=(0.0, 1.0, 0.0), tolerance=1e-6, keepCurrent=True, method="cg",
                                preconditioner="rChan", maxIterationCount=20000)
            for n, m in ((384, 320), (300, 260))]
    with R.Server(budgetBytes=100e9, maxActive=2) as ref_srv:
        ref = [ref_srv.wait(ref_srv.submit(q), release=True) for q in reqs]
    with R.Server(budgetBytes=100e9, maxActive=2, precision="single") as srv:
        got = [srv.wait(srv.submit(q), release=True) for q in reqs]
    for a, b in zip(got, ref):
        assert a["state"] == "done" and a["converged"] and a["residual"] <= 1e-6
        assert _rel(a["current"], b["current"]) < 1e-4


def test_batched_requests_match_their_solves_alone():
    """maxBatch: admitted requests whose plates share a power-of-two transform grid (here 64 x 64) and solver
    setting run as one plate batch; each result agrees with the same request served alone to the accuracy of
    its tolerance, and requests of other grids or settings are served beside them."""
    import rooftop_mom_b200 as R

    same = [_plate(60, 50), _plate(64, 64, d=(0, 0, -1), p=(1, 0, 0)), _plate(40, 57),
            R.Request.deltaGap(50, 40, LAM / 20, LAM / 20, K, portDirection="x", tolerance=TOL, keepCurrent=True),
            _plate(33, 63)]
    other = [_strip(41), _plate(20, 20, method="cg")]
    with R.Server(maxActive=2, transformSizes="powerOfTwo") as srv:
        alone = [srv.wait(srv.submit(q)) for q in same]
    with R.Server(maxActive=8, maxBatch=8, transformSizes="powerOfTwo") as srv:
        # the one worker takes the strip first; the requests submitted meanwhile wait admitted for it
        ids = [srv.submit(other[0])] + [srv.submit(q) for q in same] + [srv.submit(other[1])]
        res = [srv.wait(r) for r in ids]
    batched = res[1:1 + len(same)]
    # one worker took every request of the shared grid in one batch: they started and finished together
    assert len({r["finished"] for r in batched}) == 1 and len({r["started"] for r in batched}) == 1
    for a, b in zip(alone, batched):
        assert a["state"] == b["state"] == "done"
        assert b["converged"] and b["residual"] <= TOL
        assert abs(a["iterations"] - b["iterations"]) <= 3
        assert _rel(b["current"], a["current"]) < 1e-6
        if a["rcs"]:
            assert a["rcs"] == pytest.approx(b["rcs"], rel=1e-6)
        assert abs(a["impedance"] - b["impedance"]) <= 1e-6 * max(1.0, abs(a["impedance"]))
    assert all(o["state"] == "done" and o["converged"] for o in (res[0], res[-1]))
