"""include/rtm.h compiles as strict C99 (gcc -std=c99 -pedantic -Wall -Werror), as a MEX gateway includes
it, and a C program linked against librtm.so calls the entry points that need no GPU: the version, the byte
models (against the oracle), the size of the fixed scratch array, a delta gap built in host memory (against
the oracle), the status and message of two rejected calls, and the serving loop's create / submit / poll /
destroy with a request that fails at submission. The MEX gateway mex/rtm_mex.c compiles against the
header."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def consumer(tmp_path_factory):
    from rooftop_mom_b200 import build

    lib = build.build()
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path_factory.mktemp("c") / "abi_consumer")
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_consumer.c"), "-o", exe, "-L", libdir, "-l:librtm.so",
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=120).stdout
    return {line.split()[0]: line.split()[1:] for line in out.splitlines()}


def test_version(consumer):
    assert consumer["version"] == ["0", "3.5.0"]


def test_byte_models(consumer):
    from oracle import excitation as EX
    from oracle.geometry import Rooftops

    rt = Rooftops(256, 256, 0.1, 0.1)
    stored, working = EX.estimate_product(rt, "splitFFT")
    pc_stored, pc_working = EX.estimate_preconditioner(rt)
    want = [EX.estimate_generators(rt), stored, working, pc_stored, pc_working,
            EX.estimate_solver(rt.count, "gmres", True, 50, 1000)]
    assert consumer["estimate"][0] == "0"
    assert [float(v) for v in consumer["estimate"][1:]] == want


def test_fixed_scratch_size(consumer):
    assert consumer["scratch"] == ["0", str(32 << 20)]


def test_delta_gap_in_host_memory(consumer):
    from oracle import excitation as EX
    from oracle.geometry import Rooftops

    assert consumer["gap"][0] == "0"
    want = EX.delta_gap(Rooftops(4, 3, 0.1, 0.2), [1, 4, 10], 3.0)
    assert [float(v) for v in consumer["gap"][1:]] == list(want)


def test_the_serving_loop_from_c(consumer):
    """rtm_server_* from C: create, a submission that fails at once on the budget, poll, destroy."""
    from rooftop_mom_b200 import _lib as L

    assert consumer["server_create"] == ["0"]
    assert consumer["server_submit"] == ["0", "1"]
    status, state, failure, nbytes = consumer["server_poll"]
    assert (status, L.STATES[int(state)], int(failure)) == ("0", "failed", L.ERR_OOM_BUDGET)
    assert float(nbytes) > 1e6
    assert consumer["server_destroy"] == ["0"]


def test_rejected_calls_report_status_and_message(consumer):
    from rooftop_mom_b200 import _lib as L

    assert consumer["null"][0] == str(L.ERR_ARG)
    assert " ".join(consumer["null"][1:]) == "null output"
    assert consumer["rhs"][0] == str(L.ERR_SIZE)
    assert "65535" in " ".join(consumer["rhs"][1:])


def test_the_mex_gateway_compiles_against_the_header():
    """The C gateway mex/rtm_mex.c, compiled for syntax and types against include/rtm.h and a stand-in for
    MATLAB's mex.h: a signature that drifts from the header fails here."""
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    path = os.path.join(ROOT, "mex", "rtm_mex.c")
    assert "mexFunction" in open(path).read()
    subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "tests", "c", "mex_stub"), "-I", os.path.join(ROOT, "include"), path],
                   check=True, capture_output=True, text=True)


def test_ctypes_structures_match_the_header_layout(tmp_path):
    """Every ABI structure the Python binding mirrors has the header's size and field offsets (a field added
    to one side only would shift the others)."""
    import ctypes as C

    from rooftop_mom_b200 import _lib as L

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    mirrors = {"rtm_solve_config": L.SolveConfig, "rtm_solve_stats": L.SolveStats, "rtm_tune_result": L.TuneResult,
               "rtm_server_config": L.ServerConfig, "rtm_request": L.Request, "rtm_request_result": L.RequestResult}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "rtm.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=60).stdout
    got = {(a, b): int(c) for a, b, c in (line.split() for line in out.splitlines())}
    for cname, cls in mirrors.items():
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
