"""Plate batches (rtm_plate_batch_*): plates of uneven size, one right-hand side each, in one launch of each
product kernel, against the same plates' own products and solves (which the other GPU tests pin to the
oracle and the reference's golden data)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel, random_vector

pytestmark = pytest.mark.gpu

# (countX, countY): uneven plates that all take the 256 x 256 power-of-two transform grid
PLATES = [(200, 180), (256, 256), (130, 150), (256, 97)]


def _plates(precision="double", fft=(256, 256), plates=PLATES):
    import rooftop_mom_b200 as R

    out = []
    for cx, cy in plates:
        mesh = R.Mesh(cx, cy, 1 / 20, 1 / 20)
        R.setTransformSize(mesh, fft, precision=precision)
        prob = R.Problem(mesh, 2 * np.pi)
        out.append((prob, R.Operator(prob, precision=precision)))
    return out


@pytest.mark.parametrize("precision", ["double", "single"])
def test_a_fused_batch_product_equals_each_plates_own_product(precision):
    import rooftop_mom_b200 as R

    plates = _plates(precision)
    # the second plate twice: two right-hand sides of one plate are two entries sharing its operator
    ops = [op for _, op in plates] + [plates[1][1]]
    batch = R.PlateBatch(ops)
    assert batch.fused() and batch.count() == 5
    assert batch.stride() == max(op.rooftopCount() for op in ops)
    xs = [random_vector(op.rooftopCount(), seed=40 + k) for k, op in enumerate(ops)]
    ys = batch.apply(xs)
    for op, x, y in zip(ops, xs, ys):
        # the same kernels on the same numbers: equal to the last bit
        assert np.array_equal(np.asarray(y), np.asarray(op.apply(x)))


def test_a_batch_of_products_on_different_transform_grids_runs_entry_by_entry():
    import rooftop_mom_b200 as R

    a = _plates(plates=[(60, 50)], fft=(64, 64))[0][1]
    b = _plates(plates=[(70, 45)], fft=(72, 48))[0][1]  # a 7-smooth grid: the generic engine
    batch = R.PlateBatch([a, b])
    assert not batch.fused()
    xs = [random_vector(op.rooftopCount(), seed=50 + k) for k, op in enumerate((a, b))]
    for op, x, y in zip((a, b), xs, batch.apply(xs)):
        assert np.array_equal(np.asarray(y), np.asarray(op.apply(x)))


def test_a_batch_product_on_the_device_keeps_the_tails_zero():
    import torch

    import rooftop_mom_b200 as R

    plates = _plates()
    ops = [op for _, op in plates]
    batch = R.PlateBatch(ops)
    xs = [torch.as_tensor(random_vector(op.rooftopCount(), seed=60 + k), device="cuda") for k, op in enumerate(ops)]
    packed = batch._pack(xs, True)
    # garbage in the tails of the input is ignored
    for k, op in enumerate(ops):
        packed[k * batch.stride() + op.rooftopCount():(k + 1) * batch.stride()] = 1e30
    y = torch.empty_like(packed)
    import ctypes as C

    from rooftop_mom_b200 import _lib as L

    L.call("rtm_plate_batch_apply", batch._handle, 0, C.c_void_p(packed.data_ptr()), C.c_void_p(y.data_ptr()),
           L.DEVICE, None)
    torch.cuda.synchronize()
    for k, op in enumerate(ops):
        n = op.rooftopCount()
        assert torch.count_nonzero(y[k * batch.stride() + n:(k + 1) * batch.stride()]) == 0
        # the fused kernels read only each plate's own rooftops
        assert rel(y[k * batch.stride():k * batch.stride() + n].cpu().numpy(), op.apply(xs[k].cpu().numpy())) < 1e-15


@pytest.mark.parametrize("method,pc", [("cg", "rChan"), ("gmres", "blockJacobi")])
def test_a_batch_solve_matches_each_plates_own_solve(method, pc):
    """Each entry stops on its own tolerance; its current agrees with the plate's own solve to the accuracy
    both reach (against a solve to 1e-10) and its iteration count with the plate's own within a few."""
    import rooftop_mom_b200 as R

    plates = _plates(plates=PLATES[:3])
    ops = [op for _, op in plates]
    if pc == "rChan":
        pcs = [R.Preconditioner(prob, kernel="rChan") for prob, _ in plates]
    else:
        pcs = [R.Preconditioner.blockJacobi(prob, (2, 2)) for prob, _ in plates]
    dirs = [(0, 0, -1), (0.5, 0, -np.sqrt(0.75)), (0, 0.6, -0.8)]
    pols = [(1, 0, 0), (0, 1, 0), (1, 0, 0)]
    rhs = [R.Excitation.planeWave(prob, direction=d, polarization=p) for (prob, _), d, p in zip(plates, dirs, pols)]
    solver = R.Solver(method=method, tolerance=1e-6, restart=50, maxIterationCount=10000, side="right")
    batch = R.PlateBatch(ops, pcs)
    assert batch.fused() and batch.fusedPreconditioner() == (pc == "blockJacobi")
    res = solver.solveBatch(batch, rhs)
    for k, (r, op, p, e) in enumerate(zip(res, ops, pcs, rhs)):
        own = solver.solve(op, e, preconditioner=p)
        tight = R.Solver(method=method, tolerance=1e-10, restart=50, maxIterationCount=20000,
                         side="right").solve(op, e, preconditioner=p)
        assert r.converged() and r.residualNorm() <= 1e-6, (k, r.iterationCount(), r.residualNorm())
        # the batch's sums run over the padded stride: rounding may move the stopping test by a few iterations
        assert abs(r.iterationCount() - own.iterationCount()) <= max(5, own.iterationCount() // 20)
        assert rel(r.solution(), tight.solution()) < 20 * rel(own.solution(), tight.solution()) + 1e-12
        # the RCS of the entry's plane wave, through the entry's own excitation
        assert abs(r.radarCrossSection() - own.radarCrossSection()) <= 1e-4 * abs(own.radarCrossSection())


@pytest.mark.parametrize("kind", ["blockJacobi", "rChan"])
def test_a_batch_preconditioner_equals_each_plates_own(kind):
    """Block-Jacobi preconditioners of a batch run as one launch, circulant ones entry by entry: either way
    each entry's output is its plate's own preconditioner's, to the last bit."""
    import rooftop_mom_b200 as R

    plates = _plates(plates=[(40, 33), (64, 64), (50, 61)], fft=(64, 64))
    ops = [op for _, op in plates]
    if kind == "blockJacobi":
        pcs = [R.Preconditioner.blockJacobi(prob, (2, 2)) for prob, _ in plates]
    else:
        pcs = [R.Preconditioner(prob, kernel="rChan") for prob, _ in plates]
    batch = R.PlateBatch(ops, pcs)
    assert batch.fused() and batch.fusedPreconditioner() == (kind == "blockJacobi")
    xs = [random_vector(op.rooftopCount(), seed=70 + k) for k, op in enumerate(ops)]
    for p, x, y in zip(pcs, xs, batch.precondition(xs)):
        assert np.array_equal(np.asarray(y), np.asarray(p.apply(x)))
