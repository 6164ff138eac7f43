"""The C-ABI library loads and exports every entry point include/rtm.h declares (no GPU needed)."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

from conftest import ROOT


def _declared():
    text = open(os.path.join(ROOT, "include", "rtm.h")).read()
    return sorted(set(re.findall(r"RTM_API int (rtm_\w+)\(", text)))


@pytest.fixture(scope="module")
def library():
    from rooftop_mom_b200 import build

    return build.build()


def test_library_exports_every_declared_symbol(library):
    out = subprocess.run(["nm", "-D", "--defined-only", library], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (rtm_\w+)", out))
    declared = _declared()
    assert declared, "no declarations found"
    assert set(declared) <= exported
    # nothing else leaks out of the library
    assert exported == set(declared)


def test_library_loads_and_binds_every_symbol(library):
    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name)
    assert set(_lib.exported_symbols()) == set(_declared())


def test_version_and_errors_without_a_gpu(library):
    import ctypes as C

    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    assert lib.rtm_version(C.byref(a), C.byref(b), C.byref(c)) == 0
    assert (a.value, b.value, c.value) == (3, 5, 0)
    # argument errors are reported without touching a device
    assert lib.rtm_generators_destroy(None) == 0
    v = C.c_int()
    assert lib.rtm_generators_info(None, C.byref(v), C.byref(v), C.byref(v)) == _lib.ERR_ARG
    out = (C.c_double * 6)()
    assert lib.rtm_estimate_bytes(0, 4, 1, 0, 0, 50, 1000, out) == _lib.ERR_ARG
    assert "invalid grid" in _lib.last_error()


def test_batched_calls_bound_the_vector_count(library):
    """A batched call takes 1 to 65535 vectors; the count is checked before any device work."""
    import ctypes as C

    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    dummy = (C.c_double * 3)(0.0, 0.0, -1.0)
    sink = (C.c_double * 2)()
    args = (8, 8, 0.05, 0.05, 8, 6.283185307179586, dummy, dummy, dummy)
    assert lib.rtm_plane_wave(*args, 65536, sink, _lib.HOST, None) == _lib.ERR_SIZE
    assert "65535" in _lib.last_error()
    assert lib.rtm_plane_wave(*args, 0, sink, _lib.HOST, None) == _lib.ERR_ARG
    assert "positive" in _lib.last_error()


def test_plate_batches_and_transform_sizes_check_their_arguments_first(library):
    """rtm_plate_batch_* and rtm_tune_set reject null handles, entry counts outside 1..65535 and transform
    grids smaller than the face grid before any device work."""
    import ctypes as C

    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    out = C.c_void_p()
    ops = (C.c_void_p * 2)(None, None)
    assert lib.rtm_plate_batch_create(None, None, 1, C.byref(out)) == _lib.ERR_ARG
    assert lib.rtm_plate_batch_create(ops, None, 0, C.byref(out)) == _lib.ERR_ARG
    assert lib.rtm_plate_batch_create(ops, None, 65536, C.byref(out)) == _lib.ERR_SIZE
    assert lib.rtm_plate_batch_create(ops, None, 2, C.byref(out)) == _lib.ERR_ARG
    assert "null operator" in _lib.last_error()
    v64, v = C.c_int64(), C.c_int()
    assert lib.rtm_plate_batch_info(None, C.byref(v64), C.byref(v), C.byref(v), C.byref(v)) == _lib.ERR_ARG
    assert lib.rtm_plate_batch_apply(None, 0, None, None, _lib.HOST, None) == _lib.ERR_ARG
    assert lib.rtm_plate_batch_solve(None, None, None, None, None, _lib.HOST, None, None, None) == _lib.ERR_ARG
    assert lib.rtm_plate_batch_destroy(None) == 0
    assert lib.rtm_tune_set(100, 80, 0, 64, 128) == _lib.ERR_ARG
    assert "smaller than the face grid" in _lib.last_error()
    assert lib.rtm_tune_set(100, 80, 7, 128, 128) == _lib.ERR_ARG
    assert lib.rtm_tune_set(1, 80, 0, 128, 128) == _lib.ERR_ARG


def test_plane_waves_take_perpendicular_unit_vectors(library):
    """generatePlaneWave.m takes a unit direction and a unit polarization perpendicular to it; the ABI checks
    both before any device work."""
    import ctypes as C

    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    one = (C.c_double * 1)(1.0)
    sink = (C.c_double * 2)()
    for d, p in (((0, 0, -2), (1, 0, 0)), ((0, 0, -1), (1, 0, 0.1)), ((1, 0, 0), (1, 0, 0))):
        dv, pv = (C.c_double * 3)(*d), (C.c_double * 3)(*p)
        assert lib.rtm_plane_wave(8, 8, 0.05, 0.05, 8, 6.283185307179586, dv, pv, one, 1, sink, _lib.HOST,
                                  None) == _lib.ERR_ARG
        assert "perpendicular unit vectors" in _lib.last_error()


def test_byte_models_match_the_oracle(library):
    import ctypes as C

    from rooftop_mom_b200 import _lib
    from oracle import excitation as EX, geometry as G

    lib = _lib.load()
    for (cx, cy) in [(5, 4), (256, 256), (9, 1), (1, 6), (1024, 1024), (37, 11)]:
        rt = G.Rooftops(cx, cy, 0.1, 0.1)
        for pname, pid in _lib.PRODUCTS.items():
            for method, mid in (("cg", 0), ("gmres", 1)):
                out = (C.c_double * 6)()
                assert lib.rtm_estimate_bytes(cx, cy, pid, mid, 1, 50, 1000, out) == 0
                stored, working = EX.estimate_product(rt, pname)
                assert out[0] == EX.estimate_generators(rt)
                assert out[1] == stored and out[2] == working
                ps, pw = EX.estimate_preconditioner(rt)
                assert out[3] == ps and out[4] == pw
                assert out[5] == EX.estimate_solver(rt.count, method, True, 50, 1000)


def test_input_impedance_rejects_ports_outside_the_rooftops(library):
    """The port's currents are gathered on the device, so every index must name a rooftop: the ABI checks
    them before any device work."""
    import ctypes as C

    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    n = 3 * 3 + 4 * 2  # a 4 x 3 plate
    current = (C.c_double * (2 * n))()
    out = (C.c_double * 2)()
    for bad in (n, -1):
        port = (C.c_int64 * 2)(1, bad)
        assert lib.rtm_input_impedance(4, 3, 0.1, 0.2, current, port, 2, 1.0, _lib.HOST, out) == _lib.ERR_ARG
        assert "rooftop indices below 17" in _lib.last_error()


def test_memory_messages_format_bytes_as_the_reference():
    """The ceiling message of Budget.require (Budget.m:93-97) with byte counts written as formatBytes.m and
    its tests (tests/+unit/+resources/+utils/FormatBytesTest.m:5-11) write them: whole bytes, then one
    decimal in kB, MB, GB, TB. The ceiling check comes before any device query; nothing is held here."""
    from rooftop_mom_b200 import _lib

    lib = _lib.load()
    cases = [(512.0, 1536.0, "1.5 kB", "512 B"), (3 * 2 ** 30, 4 * 2 ** 30, "4.0 GB", "3.0 GB"),
             (2 ** 20, 1.5 * 2 ** 20, "1.5 MB", "1.0 MB")]
    try:
        for ceiling, need, need_text, ceiling_text in cases:
            assert lib.rtm_budget_configure(ceiling) == 0
            assert lib.rtm_budget_require(need) == _lib.ERR_OOM_BUDGET
            assert _lib.last_error() == (f"The request needs {need_text}, but only {ceiling_text} of the memory "
                                         f"ceiling of {ceiling_text} are left.")
    finally:
        lib.rtm_budget_configure(0.0)
