"""COCG, preconditioned COCG and restarted left-preconditioned GMRES (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+solver/IterativeMethod.m:27-70
  src/+rooftopMoM/+solver/ConjugateGradient.m:12-69
  src/+rooftopMoM/+solver/PreconditionedConjugateGradient.m:18-23
  src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/iterate_.m:1-85
  src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/private/orthogonalize_.m:15-23
  src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/private/generateRotation_.m:11-18
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np


@dataclass
class Output:
    """Output.m:14-21."""

    solution: np.ndarray
    converged: bool
    iteration_count: int
    residual_norms: np.ndarray
    residual_norm: float
    time: float


def _handle(op):
    if op is None:
        return None
    if callable(op):
        return op
    if isinstance(op, np.ndarray):
        return lambda v: op @ v
    return op.apply


def cocg_iterate(apply, b, x0, tol, maxit, precond=None):
    """ConjugateGradient.iterate_ (ConjugateGradient.m:12-62)."""
    bn = np.linalg.norm(b)
    if x0 is None:
        x = np.zeros_like(b)
        r = b.copy()
    else:
        x = x0.copy()
        r = b - apply(x)
    norms = [np.linalg.norm(r) / bn]
    converged = norms[0] < tol
    it = 0
    d = None
    rho = None
    while not converged and it < maxit:
        it += 1
        z = r if precond is None else precond(r)
        rho_next = r @ z
        d = z.copy() if it == 1 else z + (rho_next / rho) * d
        rho = rho_next
        q = apply(d)
        alpha = rho / (d @ q)
        x = x + alpha * d
        r = r - alpha * q
        norms.append(np.linalg.norm(r) / bn)
        converged = norms[-1] < tol
        if not np.isfinite(norms[-1]):
            break
    return x, converged, np.array(norms)


def _rotation(a, b):
    """generateRotation_.m:11-18."""
    radius = np.sqrt(abs(a) ** 2 + abs(b) ** 2)
    if radius > 0:
        return a / radius, b / radius
    return 1.0 + 0j, 0j


def gmres_iterate(apply, b, x0, tol, maxit, restart, precond=None):
    """GeneralizedMinimumResidual.iterate_ (iterate_.m:1-85)."""
    P = (lambda v: v) if precond is None else precond
    n = b.size
    m = int(min(restart, n, maxit))
    ref = np.linalg.norm(P(b))
    if x0 is None:
        x = np.zeros(n, dtype=np.complex128)
        r = P(b)
    else:
        x = x0.astype(np.complex128)
        r = P(b - apply(x))
    rn = np.linalg.norm(r)
    norms = [rn / ref]
    converged = norms[0] < tol
    it = 0
    # column-major as MATLAB's V, so that V(:, 1:step) is one contiguous block for BLAS
    V = np.zeros((n, m + 1), dtype=np.complex128, order="F")
    H = np.zeros((m + 1, m), dtype=np.complex128)
    cs = np.zeros(m, dtype=np.complex128)
    sn = np.zeros(m, dtype=np.complex128)
    while not converged and it < maxit:
        V[:, 0] = r / rn
        g = np.zeros(m + 1, dtype=np.complex128)
        g[0] = rn
        step = 0
        while not converged and step < m and it < maxit:
            step += 1
            it += 1
            w = P(apply(V[:, step - 1]))
            # orthogonalize_.m:15-23: classical Gram-Schmidt twice against the first `step` columns
            # V' * w as conj(V.' * conj(w)): the same products without a conjugated copy of the basis
            Vs = V[:, :step]
            h = (Vs.T @ w.conj()).conj()
            w = w - Vs @ h
            c = (Vs.T @ w.conj()).conj()
            w = w - Vs @ c
            h = h + c
            H[:step, step - 1] = h
            H[step, step - 1] = np.linalg.norm(w)
            for k in range(step - 1):
                a0, a1 = H[k, step - 1], H[k + 1, step - 1]
                H[k, step - 1] = np.conj(cs[k]) * a0 + np.conj(sn[k]) * a1
                H[k + 1, step - 1] = -sn[k] * a0 + cs[k] * a1
            cs[step - 1], sn[step - 1] = _rotation(H[step - 1, step - 1], H[step, step - 1])
            sub = H[step, step - 1]
            H[step - 1, step - 1] = np.conj(cs[step - 1]) * H[step - 1, step - 1] + np.conj(sn[step - 1]) * sub
            H[step, step - 1] = 0
            g[step] = -sn[step - 1] * g[step - 1]
            g[step - 1] = np.conj(cs[step - 1]) * g[step - 1]
            norms.append(abs(g[step]) / ref)
            converged = norms[-1] < tol
            if not converged and sub != 0:
                V[:, step] = w / sub
        y = np.linalg.solve(np.triu(H[:step, :step]), g[:step]) if step > 0 else np.zeros(0)
        x = x + V[:, :step] @ y
        if not converged and it < maxit:
            r = P(b - apply(x))
            rn = np.linalg.norm(r)
    return x, converged, np.array(norms)


def solve(method, apply, b, x0=None, tol=1e-6, maxit=1000, restart=50, precond=None):
    """IterativeMethod.solve (IterativeMethod.m:27-70) for 'cg' (COCG / PCOCG) or 'gmres'."""
    t0 = time.perf_counter()
    A = _handle(apply)
    M = _handle(precond)
    b = np.asarray(b, dtype=np.complex128)
    if np.any(b):
        if method == "cg":
            x, conv, norms = cocg_iterate(A, b, x0, tol, maxit, M)
        else:
            x, conv, norms = gmres_iterate(A, b, x0, tol, maxit, restart, M)
        res = np.linalg.norm(b - A(x)) / np.linalg.norm(b)
    else:
        x = np.zeros_like(b)
        conv, norms, res = True, np.zeros(1), 0.0
    return Output(x, bool(conv), len(norms) - 1, norms, float(res), time.perf_counter() - t0)
