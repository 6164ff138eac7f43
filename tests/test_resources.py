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


def test_bytes_are_formatted_as_the_reference_formats_them():
    # tests/+unit/+resources/+utils/FormatBytesTest.m:5-11
    from rooftop_mom_b200.api import format_bytes

    assert [format_bytes(v) for v in (512, 1536, 3 * 2 ** 30, math.inf, math.nan)] == \
        ["512 B", "1.5 kB", "3.0 GB", "unlimited", "unknown"]


def test_a_problem_above_the_ceiling_raises_when_it_is_made():
    """tests/+unit/ResourcesTest.m:16-28 (Problem.m:77, :210-219): the message names what the assembly needs,
    and the device assembly's own check (rtm_generators_assemble, before any device work) says the same."""
    import ctypes as C

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    try:
        R.Resources.configure(2 ** 16)
        with pytest.raises(L.RtmError) as e:
            R.Problem(R.Mesh(64, 64, 0.05, 0.05), 2 * math.pi)
        assert e.value.identifier == "rooftopMoM:resources:insufficientMemory"
        assert "The assembly of 8064 rooftops (generators" in str(e.value)
        h = C.c_void_p()
        assert L.load().rtm_generators_assemble(64, 64, 0.05, 0.05, 2 * math.pi, 16, 8, None, C.byref(h)) == \
            L.ERR_OOM_BUDGET
        assert str(e.value).endswith(L.last_error())
    finally:
        R.Resources.configure(math.inf)
