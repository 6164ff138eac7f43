"""The oracle's solvers show the behaviours the reference's solver tests hold
(tests/+unit/+solver/IterativeMethodTest.m:17-92, ConjugateGradientTest.m:5-72,
GeneralizedMinimumResidualTest.m:5-65), on seeded dense systems built like the fixtures of
tests/+unit/+solver/Base.m:11-29. These behaviours are what the device solvers are held to."""
from __future__ import annotations

import warnings

import numpy as np
import pytest

from oracle import solvers


def _symmetric(count, seed=1):
    """4 I plus a complex symmetric random part of norm about 2 (singular values about 2 to 6)."""
    g = np.random.default_rng(seed)
    random = (g.standard_normal((count, count)) + 1j * g.standard_normal((count, count))) / np.sqrt(count)
    return 4 * np.eye(count) + (random + random.T) / 2, g.standard_normal(count) + 1j * g.standard_normal(count)


def _nonsymmetric(count, seed=2):
    """4 I plus a random part with its eigenvalues within about 1.4 of zero."""
    g = np.random.default_rng(seed)
    matrix = 4 * np.eye(count) + (g.standard_normal((count, count)) + 1j * g.standard_normal((count, count))) / np.sqrt(count)
    return matrix, g.standard_normal(count) + 1j * g.standard_normal(count)


METHODS = {
    "cg": lambda A, b, x0, tol, maxit: solvers.solve("cg", A, b, x0, tol, maxit),
    "pcg": lambda A, b, x0, tol, maxit: solvers.solve("cg", A, b, x0, tol, maxit, precond=lambda r: r),
    # no restarts, so every limit counts single iterations
    "gmres": lambda A, b, x0, tol, maxit: solvers.solve("gmres", A, b, x0, tol, maxit, restart=10**9),
}


@pytest.mark.parametrize("method", sorted(METHODS))
def test_solves_the_system(method):
    A, b = _symmetric(30)
    out = METHODS[method](A, b, None, 1e-10, 100)
    want = np.linalg.solve(A, b)
    assert out.converged
    assert np.linalg.norm(out.solution - want) / np.linalg.norm(want) < 1e-9
    assert out.residual_norms.size == out.iteration_count + 1


@pytest.mark.parametrize("method", sorted(METHODS))
def test_output_holds_the_true_residual(method):
    A, b = _symmetric(30)
    out = METHODS[method](A, b, None, 1e-6, 100)
    true = np.linalg.norm(b - A @ out.solution) / np.linalg.norm(b)
    assert out.residual_norm == pytest.approx(true, rel=1e-12)
    assert true < 1e-6


@pytest.mark.parametrize("method", sorted(METHODS))
def test_zero_right_hand_side_gives_the_zero_solution(method):
    out = METHODS[method](np.eye(3), np.zeros(3), np.ones(3, dtype=np.complex128), 1e-10, 100)
    assert np.array_equal(out.solution, np.zeros(3))
    assert out.converged
    assert (out.iteration_count, out.residual_norm) == (0, 0.0)


@pytest.mark.parametrize("method", sorted(METHODS))
def test_exact_initial_guess_needs_no_iteration(method):
    A, b = _symmetric(30)
    out = METHODS[method](A, b, np.linalg.solve(A, b), 1e-10, 100)
    assert out.converged
    assert out.iteration_count == 0


@pytest.mark.parametrize("method", sorted(METHODS))
def test_every_operator_form_gives_the_same_solution(method):
    A, b = _symmetric(30)
    want = METHODS[method](A, b, None, 1e-10, 100).solution

    class Wrapped:
        def apply(self, v):
            return A @ v

    assert np.array_equal(METHODS[method](lambda v: A @ v, b, None, 1e-10, 100).solution, want)
    assert np.array_equal(METHODS[method](Wrapped(), b, None, 1e-10, 100).solution, want)


@pytest.mark.parametrize("method", sorted(METHODS))
def test_non_convergence_is_a_result(method):
    A, b = _symmetric(30)
    out = METHODS[method](A, b, None, 1e-14, 2)
    assert not out.converged
    assert out.iteration_count == 2


def test_cocg_stops_on_the_residual_norm():
    A, b = _symmetric(40)
    out = solvers.solve("cg", A, b, None, 1e-8, 100)
    true = np.linalg.norm(b - A @ out.solution) / np.linalg.norm(b)
    assert out.residual_norms[0] == 1
    assert out.residual_norms[-1] == pytest.approx(true, rel=1e-4)
    assert true < 1e-8


def test_cocg_records_every_iteration():
    A, b = _symmetric(40)
    out = solvers.solve("cg", A, b, None, 1e-8, 100)
    shorter = solvers.solve("cg", A, b, None, 1e-8, out.iteration_count - 1)
    assert out.residual_norms[-1] < 1e-8
    assert np.all(out.residual_norms[:-1] >= 1e-8)
    assert not shorter.converged


def test_diagonal_preconditioner_cuts_the_cocg_iterations():
    A, b = _symmetric(100)
    scaling = np.logspace(0, 2, 100)
    A = scaling[:, None] * A * scaling[None, :]  # still complex symmetric
    diagonal = np.diag(A).copy()
    plain = solvers.solve("cg", A, b, None, 1e-8, 1000)
    pre = solvers.solve("cg", A, b, None, 1e-8, 1000, precond=lambda r: r / diagonal)
    assert pre.converged
    assert pre.residual_norm < 1e-8
    assert pre.iteration_count < plain.iteration_count / 2


def test_cocg_stops_on_a_breakdown():
    # the first direction b has b^T A b = 0: the step length is infinite
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = solvers.solve("cg", np.diag([1.0, -1.0]), np.ones(2), None, 1e-8, 100)
    assert not out.converged
    assert out.iteration_count == 1


def test_gmres_solves_a_nonsymmetric_system_across_restarts():
    A, b = _nonsymmetric(40)
    out = solvers.solve("gmres", A, b, None, 1e-10, 100, restart=10)
    want = np.linalg.solve(A, b)
    assert out.converged
    assert out.iteration_count > 10
    assert np.linalg.norm(out.solution - want) / np.linalg.norm(want) < 1e-9


def test_gmres_stops_at_the_iteration_limit_inside_a_cycle():
    A, b = _nonsymmetric(60)
    out = solvers.solve("gmres", A, b, None, 1e-14, 7, restart=5)
    assert not out.converged
    assert out.iteration_count == 7


def test_gmres_restart_beyond_the_system_size_is_capped():
    A, b = _nonsymmetric(20)
    equal = solvers.solve("gmres", A, b, None, 1e-10, 100, restart=20)
    longer = solvers.solve("gmres", A, b, None, 1e-10, 100, restart=50)
    assert equal.converged
    assert np.array_equal(equal.solution, longer.solution)


def test_gmres_residual_is_that_of_the_preconditioned_system():
    A, b = _nonsymmetric(60)
    A = np.logspace(0, 3, 60)[:, None] * A
    diagonal = np.diag(A).copy()

    def precondition(r):
        return r / diagonal

    plain = solvers.solve("gmres", A, b, None, 1e-10, 200, restart=20)
    out = solvers.solve("gmres", A, b, None, 1e-10, 200, restart=20, precond=precondition)
    want = np.linalg.norm(precondition(b - A @ out.solution)) / np.linalg.norm(precondition(b))
    assert out.converged
    assert abs(out.residual_norms[0] - 1) <= 1e-14
    assert abs(out.residual_norms[-1] - want) <= 1e-12
    assert out.iteration_count < plain.iteration_count
