"""Host-side behaviour of the request loop (rtm_server_*) that needs no GPU: validation of requests and
admission by the byte budget (the reference's Budget.require, src/+rooftopMoM/+resources/Budget.m:82-106,
error identifier rooftopMoM:resources:insufficientMemory)."""
from __future__ import annotations

import math

import pytest


def _request(count=(40, 32), **kw):
    import rooftop_mom_b200 as R

    lam = 1.0
    return R.Request.planeWave(count[0], count[1], lam / 20, lam / 20, 2 * math.pi, direction=(0, 0, -1),
                               polarization=(1, 0, 0), **kw)


def test_a_request_above_the_budget_fails_at_submission():
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    with R.Server(budgetBytes=1e6, maxActive=2) as srv:
        rid = srv.submit(_request())
        res = srv.poll(rid)
        assert res["state"] == "failed"
        assert res["status"] == L.ERR_OOM_BUDGET
        assert res["bytes"] > 1e6


def test_invalid_requests_are_rejected():
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    with R.Server(budgetBytes=1e9, maxActive=1) as srv:
        with pytest.raises(L.RtmError):
            srv.submit(_request(count=(1, 1)))
        with pytest.raises(L.RtmError):
            srv.submit(_request(tolerance=0.0))
        with pytest.raises(L.RtmError):
            srv.poll(12345)


def test_request_bytes_grow_with_the_grid_and_the_basis():
    import rooftop_mom_b200 as R

    with R.Server(budgetBytes=1.0, maxActive=1) as srv:  # everything fails at submission: no device work
        small = srv.poll(srv.submit(_request(count=(32, 32))))["bytes"]
        large = srv.poll(srv.submit(_request(count=(64, 64))))["bytes"]
        deep = srv.poll(srv.submit(_request(count=(32, 32), restart=100)))["bytes"]
    assert large > 3.5 * small
    assert deep > small


def test_server_configuration_is_checked():
    import ctypes as C

    from rooftop_mom_b200 import _lib as L

    cfg = L.ServerConfig(1e9, 1, 7, 0)
    h = C.c_void_p()
    with pytest.raises(L.RtmError):
        L.call("rtm_server_create", C.byref(cfg), C.byref(h))


def test_plane_wave_requests_take_perpendicular_unit_vectors():
    """Request normalises the vectors as Excitation.planeWave does; the ABI rejects a request whose vectors are
    not perpendicular unit vectors, before any device work."""
    import ctypes as C

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    req = R.Request.planeWave(40, 32, 0.05, 0.05, 2 * math.pi, direction=(0, 0, -2), polarization=(0, 3, 0))
    assert list(req.struct.direction) == [0, 0, -1] and list(req.struct.polarization) == [0, 1, 0]
    with pytest.raises(L.RtmError) as e:
        R.Request.planeWave(40, 32, 0.05, 0.05, 2 * math.pi, direction=(1, 0, 0), polarization=(1, 1, 0))
    assert e.value.identifier == "rooftopMoM:excitation:notPerpendicular"
    with R.Server(budgetBytes=1e9, maxActive=1) as srv:
        raw = _request().struct
        raw.direction[:] = [0.0, 0.0, -2.0]
        rid = C.c_uint64()
        assert L.load().rtm_server_submit(srv._h, C.byref(raw), C.byref(rid)) == L.ERR_ARG
        assert "perpendicular unit vectors" in L.last_error()


def test_requests_that_fail_on_the_device_release_their_slot_and_bytes():
    """Admission, the workers and the release of a request's bytes on its failure path: without a GPU
    every admitted request fails at its first device call, and the queue must still drain through the
    slots and the budget (which admits two of these requests at a time) with every request reported."""
    import torch

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    if torch.cuda.is_available():
        pytest.skip("on a GPU these requests run; this test follows the failure path")
    with R.Server(budgetBytes=1.0, maxActive=1) as probe:
        one = probe.poll(probe.submit(_request()))["bytes"]
    with R.Server(budgetBytes=2.5 * one, maxActive=3) as srv:
        ids = [srv.submit(_request()) for _ in range(7)]
        results = [srv.poll(rid, wait=60.0) for rid in ids]
        assert [r["state"] for r in results] == ["failed"] * 7
        assert all(r["status"] == L.ERR_CUDA for r in results)
        assert all(r["finished"] >= r["started"] >= r["submitted"] for r in results)
        # the released bytes admit a later request too
        assert srv.poll(srv.submit(_request()), wait=60.0)["state"] == "failed"


def test_cancelled_admitted_requests_release_their_bytes_under_concurrent_polls():
    """A request cancelled after admission, before a worker starts it, gives its slot and bytes back in the
    same step that marks it cancelled, so a poll that releases the finished record in the meantime cannot
    race the ledger. Many requests are submitted and cancelled at once while a second thread polls each
    with release in a loop; afterwards the whole budget must be free again: a request that needs nearly all
    of it is admitted and reaches a finished state."""
    import threading

    import torch

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    if torch.cuda.is_available():
        pytest.skip("on a GPU these requests run; this test follows the host path of cancelled requests")
    with R.Server(budgetBytes=1.0, maxActive=1) as probe:
        one = probe.poll(probe.submit(_request()))["bytes"]
    with R.Server(budgetBytes=4.5 * one, maxActive=4) as srv:
        for _ in range(5):
            ids = [srv.submit(_request()) for _ in range(24)]
            seen = {}

            def poller():
                pending = list(ids)
                while pending:
                    rest = []
                    for rid in pending:
                        res = srv.poll(rid, release=True)
                        if res["state"] in ("done", "failed", "cancelled"):
                            seen[rid] = res["state"]
                        else:
                            rest.append(rid)
                    pending = rest

            t = threading.Thread(target=poller)
            t.start()
            for rid in ids:
                try:
                    srv.cancel(rid)
                except L.RtmError as e:  # the poller already released this finished request
                    assert "unknown request" in str(e)
            t.join(timeout=120)
            assert not t.is_alive()
            assert sorted(seen) == sorted(ids)
            assert set(seen.values()) <= {"failed", "cancelled"}
        # every released byte is back: four requests' worth fits again
        big = [srv.submit(_request()) for _ in range(4)]
        assert all(srv.poll(rid, wait=60.0)["state"] in ("failed", "cancelled") for rid in big)


def test_an_unknown_transform_size_policy_is_rejected():
    import ctypes as C

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    with pytest.raises(L.RtmError):
        R.Server(transformSizes="primes")
    cfg = L.ServerConfig(1e9, 1, 0, 0, 5)
    h = C.c_void_p()
    with pytest.raises(L.RtmError):
        L.call("rtm_server_create", C.byref(cfg), C.byref(h))


def test_batching_configuration_is_checked():
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    for bad in (-1, 257):
        with pytest.raises(L.RtmError):
            R.Server(maxBatch=bad)


def test_batched_requests_that_fail_on_the_device_are_each_reported():
    """The batching workers' grouping and their fallback: without a GPU a batch's set-up fails, its requests
    then run one by one and fail at their first device call, each reported with its own status, and the
    slots and bytes drain for the requests that wait behind them."""
    import torch

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    if torch.cuda.is_available():
        pytest.skip("on a GPU these requests run; this test follows the failure path")
    # 40 x 32 and 50 x 60 faces share the 64 x 64 power-of-two grid; a strip never joins a batch
    reqs = [_request((40, 32)), _request((50, 60)), _request((64, 33)), _request((33, 64)),
            R.Request.deltaGap(41, 1, 0.05, 0.05, 2 * math.pi, portDirection="x"), _request((40, 32))]
    with R.Server(budgetBytes=1e12, maxActive=4, maxBatch=4, transformSizes="powerOfTwo") as srv:
        ids = [srv.submit(q) for q in reqs]
        results = [srv.poll(rid, wait=60.0) for rid in ids]
    assert [r["state"] for r in results] == ["failed"] * len(reqs)
    assert all(r["status"] == L.ERR_CUDA for r in results)
    assert all(r["finished"] >= r["started"] >= r["submitted"] for r in results)
