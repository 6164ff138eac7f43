"""Parity at the benchmarked configurations: the device block-Jacobi preconditioner against its oracle,
the generators at the default quadrature orders [16, 8] (Problem.m:49) on the 32 x 32 and 256 x 256 plates,
and whole solves of those plates against the oracle's.

  C1: 32 x 32 faces of lambda/20, normal incidence, x polarised, unpreconditioned COCG to 1e-8
      (the reference's own plate-scattering set-up, examples/plateScattering.m:31-32);
  C2: 256 x 256 faces of lambda/20, theta = 30 deg, phi = 0, TE, block-Jacobi (2 x 2 faces) GMRES(50).

Tolerances are the path's parity bars: generators 1e-12 relative, currents and RCS 1e-10 with both solves driven
to a relative residual of 1e-12. On the C2 plate the oracle's current at a residual of 1e-12 is within
1.3e-12 of its current at 1e-14, so 1e-10 is well above what conditioning allows at that residual."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import random_vector, rel

pytestmark = pytest.mark.gpu

K = 2 * math.pi


def _c2_wave():
    t = math.radians(30.0)
    return [math.sin(t), 0.0, -math.cos(t)], [0.0, 1.0, 0.0]


def _oracle_problem(R, prob):
    """The oracle's rooftops, generators (the device's own, so that only the stage under test differs) and
    split product of a problem."""
    from oracle import assembly as A, geometry as G, spectra as S

    cx, cy = prob.mesh().count()
    a, b = prob.mesh().faceSize()
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, int(prob.quadratureOrder()[1]))
    gen = A.Generators(xx, yy, e, rt.content)
    sub = S.subband_spectra(gen, a, b)
    return rt, gen, (lambda v: S.split_apply(rt, sub, rt.content, v))


# ------------------------------------------------------------------------------------------------
# Block-Jacobi: the inverses of the diagonal blocks of the Green's matrix (tests/+unit/Base.m:83-113)

BJ_CASES = {
    "c2_256x256_2x2": (256, 256, 1 / 20, 1 / 20, 2, 2),
    "prime_13x17_2x2": (13, 17, 0.07, 0.05, 2, 2),
    "uneven_11x7_3x2": (11, 7, 0.1, 0.1, 3, 2),
    "uneven_13x17_4x2": (13, 17, 0.07, 0.05, 4, 2),
    "stripX_9x1_2x2": (9, 1, 0.1, 0.02, 2, 2),
    "stripY_1x6_2x2": (1, 6, 0.03, 0.1, 2, 2),
    "stripX_10x1_4x1": (10, 1, 0.1, 0.02, 4, 1),
}


@pytest.mark.parametrize("name", sorted(BJ_CASES))
@pytest.mark.parametrize("precision", ["double", "single"])
def test_block_jacobi_apply_matches_the_oracle(name, precision):
    """The device's packed block inverses applied to a vector, against the oracle's dense blocks inverted by
    LAPACK, on the same generators. FP64 within 1e-13; FP32 (the precision form's inner preconditioner)
    within 5e-6, a few float roundings amplified by the blocks' condition."""
    import rooftop_mom_b200 as R
    from oracle import blockjacobi as BJ

    cx, cy, a, b, bx, by = BJ_CASES[name]
    order = (16, 8) if name.startswith("c2") else (3, 3)
    prob = R.Problem(R.Mesh(cx, cy, a, b), K, quadratureOrder=order)
    rt, gen, _ = _oracle_problem(R, prob)
    pc = R.Preconditioner.blockJacobi(prob, (bx, by), precision=precision)
    want_op = BJ.BlockJacobi(gen, rt, bx, by)
    for seed in (1, 2):
        v = random_vector(rt.count, seed=seed)
        assert rel(pc.apply(v), want_op.apply(v)) < (1e-13 if precision == "double" else 5e-6)


def test_block_jacobi_blocks_above_eight_faces_are_rejected():
    """Blocks hold at most 8 faces (16 unknowns) in this build; a 3 x 3 blocking is refused before any device
    work with RTM_ERR_UNSUPPORTED."""
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    prob = R.Problem(R.Mesh(13, 17, 0.07, 0.05), K, quadratureOrder=(3, 3))
    with pytest.raises(L.RtmError) as e:
        R.Preconditioner.blockJacobi(prob, (3, 3))
    assert e.value.status == L.ERR_UNSUPPORTED


def test_batched_block_jacobi_equals_single_applies():
    import torch

    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(40, 24, 0.05, 0.05), K, quadratureOrder=(3, 3))
    pc = R.Preconditioner.blockJacobi(prob, (2, 2))
    n = prob.rooftopCount()
    vs = [random_vector(n, seed=s) for s in range(3)]
    x = torch.from_numpy(np.concatenate(vs)).cuda()
    got = pc.apply(x, nrhs=3).cpu().numpy()
    for k in range(3):
        np.testing.assert_array_equal(got[k * n:(k + 1) * n], pc.apply(vs[k]))


# ------------------------------------------------------------------------------------------------
# Generators at the default orders

@pytest.mark.parametrize("count", [32, 256])
def test_generators_at_default_orders_match_the_oracle(count):
    """MomentAssembler.generate (generate.m:10-59) at the default [16, 8] orders on the C1 and C2 plates."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A

    h = 1 / 20
    prob = R.Problem(R.Mesh(count, count, h, h), K)
    assert tuple(prob.quadratureOrder()) == (16, 8)
    xx, yy, e = prob.generators().arrays()
    ref = A.generate(count, count, h, h, K)
    for got, want in ((xx, ref.magnetic_xx), (yy, ref.magnetic_yy), (e, ref.electric)):
        assert got.shape == want.shape
        assert rel(got, want) < 1e-12
        # entry by entry as well: the far offsets are orders of magnitude below the self terms
        assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) < 1e-10


# ------------------------------------------------------------------------------------------------
# C1: 32 x 32 plate, unpreconditioned COCG to 1e-8
#
# COCG's short recurrence amplifies the differences of rounding between any two implementations once the
# first few tens of iterations are past: the residual histories agree to 1e-6 over the first 30 iterations,
# but the iteration counts drift apart (the oracle alone needs 1206 iterations to 1e-12 on the C2 plate on one
# host and 1230 on another; with rChan the device reaches 1e-6 on that plate in 589 iterations and the oracle
# in 694). So the iteration counts of the C1 plate are held to 5 % of the oracle's, and every solve is judged
# by its current, with both driven to 1e-12 where the 1e-10 parity bar applies.

def _first_below(history, tol):
    """Iterations a solve with this residual history takes to reach tol (the index of the first entry below
    it; IterativeMethod.m stops there)."""
    h = np.asarray(history)
    idx = np.flatnonzero(h < tol)
    return int(idx[0]) if idx.size else None


def test_c1_cocg_solve_matches_the_oracle():
    import rooftop_mom_b200 as R
    from oracle import excitation as EX, solvers as OS

    h = 1 / 20
    prob = R.Problem(R.Mesh(32, 32, h, h), K)
    exc = R.Excitation.planeWave(prob, direction=[0, 0, -1], polarization=[1, 0, 0])
    rt, gen, apply = _oracle_problem(R, prob)
    b = exc.vector()
    np.testing.assert_allclose(b, EX.plane_wave(rt, K, [0, 0, -1], [1, 0, 0], 1.0), rtol=0, atol=1e-13 * np.abs(b).max())
    op = R.Operator(prob)
    res = R.Solver(method="cg", tolerance=1e-8, maxIterationCount=5000).solve(op, exc)
    ref = OS.solve("cg", apply, b, tol=1e-8, maxit=5000)
    assert res.converged() and ref.converged
    assert res.residualNorm() < 1e-8
    np.testing.assert_allclose(res.residualNorms()[:30], ref.residual_norms[:30], rtol=1e-6)
    got6, want6 = _first_below(res.residualNorms(), 1e-6), _first_below(ref.residual_norms, 1e-6)
    assert abs(got6 - want6) <= max(2, 0.05 * want6)
    assert abs(res.iterationCount() - ref.iteration_count) <= max(2, 0.05 * ref.iteration_count)
    assert rel(res.solution(), ref.solution) < 1e-6
    # the 1e-10 parity bar with both driven to 1e-12
    res = R.Solver(method="cg", tolerance=1e-12, maxIterationCount=5000).solve(op, exc)
    ref = OS.solve("cg", apply, b, tol=1e-12, maxit=5000)
    assert res.converged() and ref.converged
    assert rel(res.solution(), ref.solution) < 1e-10
    rcs = EX.radar_cross_section(K, b, ref.solution)
    assert abs(res.radarCrossSection() - rcs) / rcs < 1e-10


# ------------------------------------------------------------------------------------------------
# C2: 256 x 256 plate

@pytest.fixture(scope="module")
def c2():
    """The C2 plate, its device operator and excitation, and the oracle's solution driven to 1e-12 by
    rChan-preconditioned COCG (the reference's default preconditioner; about 1200 iterations, tens of
    seconds on the host cores)."""
    import rooftop_mom_b200 as R
    from oracle import excitation as EX, preconditioner as PC, solvers as OS, spectra as S

    h = 1 / 20
    prob = R.Problem(R.Mesh(256, 256, h, h), K)
    d, p = _c2_wave()
    exc = R.Excitation.planeWave(prob, direction=d, polarization=p)
    rt, gen, apply = _oracle_problem(R, prob)
    b = exc.vector()
    assert rel(b, EX.plane_wave(rt, K, d, p, 1.0)) < 1e-13
    inv = PC.circulant(gen, h, h, "rChan", "partwise")
    ref = OS.solve("cg", apply, b, tol=1e-12, maxit=20000, precond=lambda v: S.fft_apply(rt, inv, rt.content, v))
    assert ref.converged
    return {"prob": prob, "op": R.Operator(prob), "exc": exc, "b": b, "ref": ref, "apply": apply}


def test_c2_block_jacobi_gmres_current_matches_the_oracle(c2):
    """The benchmarked method (block-Jacobi GMRES(50), right preconditioned, FP64) driven to 1e-12: its
    current and monostatic RCS against the oracle's within 1e-10, and its residual checked with the
    oracle's own product."""
    import rooftop_mom_b200 as R
    from oracle import excitation as EX

    pc = R.Preconditioner.blockJacobi(c2["prob"], (2, 2))
    res = R.Solver(method="gmres", tolerance=1e-12, restart=50, maxIterationCount=20000, side="right").solve(
        c2["op"], c2["exc"], preconditioner=pc)
    assert res.converged() and res.residualNorm() < 1e-12
    x = res.solution()
    b = c2["b"]
    assert np.linalg.norm(b - c2["apply"](x)) / np.linalg.norm(b) < 2e-12
    assert rel(x, c2["ref"].solution) < 1e-10
    rcs = EX.radar_cross_section(K, b, c2["ref"].solution)
    assert abs(res.radarCrossSection() - rcs) / rcs < 1e-10


def test_c2_block_jacobi_gmres_to_1e6_meets_the_tolerance_on_the_oracle_product(c2):
    """The benchmark's own solve (to 1e-6): the device's reported true residual agrees with the residual the
    oracle's product gives for the same current."""
    import rooftop_mom_b200 as R

    pc = R.Preconditioner.blockJacobi(c2["prob"], (2, 2))
    res = R.Solver(method="gmres", tolerance=1e-6, restart=50, maxIterationCount=20000, side="right").solve(
        c2["op"], c2["exc"], preconditioner=pc)
    assert res.converged()
    b = c2["b"]
    r = np.linalg.norm(b - c2["apply"](res.solution())) / np.linalg.norm(b)
    assert r < 1e-6
    assert abs(r - res.residualNorm()) < 1e-12


def test_c2_rchan_cocg_matches_the_oracle(c2):
    """The same method as the oracle's (rChan COCG) on the device: the residual histories over the first 30
    iterations, and the current driven to 1e-12 within 1e-10 of the oracle's."""
    import rooftop_mom_b200 as R

    pc = R.Preconditioner(c2["prob"], kernel="rChan")
    res = R.Solver(method="cg", tolerance=1e-12, maxIterationCount=20000).solve(c2["op"], c2["exc"],
                                                                               preconditioner=pc)
    ref = c2["ref"]
    assert res.converged()
    np.testing.assert_allclose(res.residualNorms()[:30], ref.residual_norms[:30], rtol=1e-6)
    assert rel(res.solution(), ref.solution) < 1e-10
