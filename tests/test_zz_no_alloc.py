"""rtm_operator_apply_fixed_scratch (the product with its working grid in the library's fixed device
array, allocating nothing) against rtm_operator_apply on the same operator and vectors, through the C
ABI. The file is named to be collected last, so it also runs after every other test has used the
library on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-13  # relative; the two paths launch the same kernels on the same grid


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _operator(count, product, precision, max_rhs=1):
    import rooftop_mom_b200 as R

    mesh = R.Mesh(count[0], count[1], 0.05, 0.045)
    prob = R.Problem(mesh, 2 * np.pi)
    return R.Operator(prob, product=product, precision=precision, maxRhs=max_rhs)


def _vectors(n, nrhs, precision, seed):
    import torch

    g = np.random.default_rng(seed)
    x = g.standard_normal((nrhs, n)) + 1j * g.standard_normal((nrhs, n))
    dt = torch.complex128 if precision == "double" else torch.complex64
    return torch.from_numpy(x).to(dtype=dt, device="cuda")


def _held():
    from rooftop_mom_b200 import _lib as L

    ceiling, held = C.c_double(), C.c_double()
    L.call("rtm_budget_query", C.byref(ceiling), C.byref(held))
    return held.value


def _rel(a, b):
    a = a.cpu().numpy().astype(np.complex128)
    b = b.cpu().numpy().astype(np.complex128)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize(
    "count,product,precision,nrhs",
    [
        ((40, 36), "splitFFT", "double", 1),
        ((40, 36), "leanSplitFFT", "double", 2),
        ((33, 28), "fft", "double", 1),
        ((64, 48), "splitFFT", "single", 3),
        ((64, 64), "splitFFT", "double", 2),  # power-of-two grids: the register-resident fast path
        ((64, 32), "splitFFT", "single", 3),
    ],
)
def test_fixed_scratch_matches_the_allocating_product(count, product, precision, nrhs):
    import torch
    from rooftop_mom_b200 import _lib as L

    op = _operator(count, product, precision, max_rhs=nrhs)
    n = op.problem().rooftopCount()
    x = _vectors(n, nrhs, precision, seed=7)
    want = torch.empty_like(x)
    L.call("rtm_operator_apply", op._handle, _ptr(x), _ptr(want), n, nrhs, L.DEVICE, None)
    held = _held()
    for _ in range(2):  # two calls in a row share the array
        got = torch.zeros_like(x)
        L.call("rtm_operator_apply_fixed_scratch", op._handle, _ptr(x), _ptr(got), n, nrhs, None)
        tol = TOLERANCE if precision == "double" else 1e-6
        assert _rel(got, want) < tol
    assert _held() == held  # nothing was allocated through the library's ledger


def test_fixed_scratch_rejects_working_grids_beyond_its_size():
    from rooftop_mom_b200 import _lib as L

    op = _operator((64, 64), "splitFFT", "double")
    n = op.problem().rooftopCount()
    size = C.c_double()
    L.call("rtm_fixed_scratch_bytes", C.byref(size))
    per_rhs = op.info()["working_bytes"]
    nrhs = int(size.value // per_rhs) + 1
    x = _vectors(n, nrhs, "double", seed=3)
    y = x.clone()
    with pytest.raises(L.RtmError) as e:
        L.call("rtm_operator_apply_fixed_scratch", op._handle, _ptr(x), _ptr(y), n, nrhs, None)
    assert e.value.status == L.ERR_SIZE
    assert "fixed scratch" in str(e.value)
