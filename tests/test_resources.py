"""Resources.check (src/+rooftopMoM/Resources.m:73-141) on the device byte models: the report of a planned
run and the insufficientMemory error when its peak exceeds the ceiling. Needs no GPU (only the ledger)."""
from __future__ import annotations

import math

import pytest


def test_check_reports_the_stages_and_their_peak():
    import rooftop_mom_b200 as R

    R.Resources.configure()
    rep = R.Resources.check(R.Mesh(64, 48, 0.05, 0.05), method="gmres", restart=30)
    for key in ("generators", "chunk", "product", "productWorking", "preconditioner", "preconditionerWorking",
                "solver", "peak"):
        assert rep[key] >= 0
    solve = rep["generators"] + rep["product"] + rep["preconditioner"] + max(rep["productWorking"],
                                                                             rep["preconditionerWorking"]) + rep["solver"]
    assert rep["peak"] == max(rep["generators"] + rep["chunk"], solve)
    bare = R.Resources.check(R.Mesh(64, 48, 0.05, 0.05), preconditioner=False, method="gmres", restart=30)
    assert bare["preconditioner"] == 0 and bare["peak"] < rep["peak"]


def test_check_raises_when_the_peak_exceeds_the_ceiling():
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    try:
        R.Resources.configure(1e6)
        with pytest.raises(L.RtmError) as e:
            R.Resources.check(R.Mesh(128, 128, 0.05, 0.05))
        assert e.value.identifier == "rooftopMoM:resources:insufficientMemory"
    finally:
        R.Resources.configure(math.inf)
