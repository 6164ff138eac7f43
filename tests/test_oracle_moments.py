"""The oracle's moment integrals against their definitions, restating the reference's unit tests
tests/+unit/+assembler/+greensMatrix/+utils/IntegrateMomentsTest.m:5-54 and
tests/+unit/+assembler/+singularIntegrals/GeneratePowerMomentsTest.m:48-66."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import assembly as A
from oracle import singular as SI
from oracle.geometry import gauss_legendre

SIZES, K = (0.1, 0.15), 2 * np.pi


def test_separated_cells_match_the_four_dimensional_rule():
    """On cells three or more apart the Green's function is smooth: a tensor Gauss-Legendre rule over
    both cells integrates the definition of the seven moments as accurately as the reduced rule."""
    offsets = np.array([[4, 0, 3], [1, 5, 4]])
    got = A.integrate_moments(A.reduced_rule(8, (1, 1)), offsets, SIZES, K)
    p, w = gauss_legendre(10, 0.0, 1.0)
    xi, xo, eta, eo = np.meshgrid(p, p, p, p, indexing="ij")
    pair = w[:, None, None, None] * w[None, :, None, None] * w[None, None, :, None] * w[None, None, None, :]
    for n in range(offsets.shape[1]):
        r = np.hypot(SIZES[0] * (xi - xo - offsets[0, n]), SIZES[1] * (eta - eo - offsets[1, n]))
        v = pair * np.exp(-1j * K * r) / r
        want = np.array([v.sum(), (xi * v).sum(), (xo * v).sum(), (xi * xo * v).sum(), (eta * v).sum(),
                         (eo * v).sum(), (eta * eo * v).sum()])
        np.testing.assert_allclose(got[:, n], want, rtol=1e-13)


@pytest.mark.parametrize("offset", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_touching_pairs_integrate_the_remainder(offset):
    nx, ny, w = rule = A.reduced_rule(6, (2, 1))
    nu, eta = np.meshgrid(nx, ny, indexing="ij")
    r = np.hypot(SIZES[0] * (nu.ravel(order="F") - offset[0]), SIZES[1] * (eta.ravel(order="F") - offset[1]))
    want = w @ SI.remainder(r, K)
    got = A.integrate_moments(rule, np.array(offset).reshape(2, 1), SIZES, K)[:, 0]
    np.testing.assert_allclose(got, want, rtol=1e-14)


def test_offsets_are_integrated_independently():
    rule = A.reduced_rule(4, (1, 1))
    offsets = np.array([[0, 1, 2, 7], [0, 1, 0, 3]])
    together = A.integrate_moments(rule, offsets, (0.1, 0.1), K)
    for n in range(offsets.shape[1]):
        alone = A.integrate_moments(rule, offsets[:, n:n + 1], (0.1, 0.1), K)[:, 0]
        np.testing.assert_allclose(together[:, n], alone, rtol=1e-15)


@pytest.mark.parametrize("power", [-1, 1, 3])
def test_transposed_cells_exchange_the_directions(power):
    m = SI.power_moments(0.1, 0.25, power)
    t = SI.power_moments(0.25, 0.1, power)
    swap = [0, 2, 1, 3]  # offsets (0,0), (1,0), (0,1), (1,1) with x and y exchanged
    np.testing.assert_allclose(m[4:7], t[1:4][:, swap], rtol=1e-14)
    np.testing.assert_allclose(m[0], t[0][swap], rtol=1e-14)


@pytest.mark.parametrize("power", [-1, 1, 3])
def test_moments_scale_with_the_power(power):
    m = SI.power_moments(0.1, 0.25, power)
    s = SI.power_moments(0.3, 0.75, power)
    np.testing.assert_allclose(s, 3.0**power * m, rtol=3e-14)
