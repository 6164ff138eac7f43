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
