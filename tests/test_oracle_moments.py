"""The oracle's moment integrals, remainder and moment accumulation against their definitions,
restating the reference's unit tests
tests/+unit/+assembler/+greensMatrix/+utils/IntegrateMomentsTest.m:5-54,
tests/+unit/+assembler/+singularIntegrals/GeneratePowerMomentsTest.m:48-66,
tests/+unit/+assembler/+singularIntegrals/EvaluateRemainderTest.m:5-21,
tests/+unit/+assembler/+greensMatrix/+utils/AccumulateMomentsTest.m:5-59,
tests/+unit/+assembler/+singularIntegrals/+utils/IntegrateMonomialTest.m:9-52 and
tests/+unit/+assembler/+singularIntegrals/GenerateExtractedMomentsTest.m:5-18."""
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


def test_remainder_is_the_greens_function_without_the_extracted_part():
    # tests/+unit/+assembler/+singularIntegrals/EvaluateRemainderTest.m:5-11
    r = np.array([0.05, 0.3, 1.0, 2.5])
    want = np.exp(-1j * K * r) / r - (1 / r - K**2 * r / 2 + K**4 * r**3 / 24)
    np.testing.assert_allclose(SI.remainder(r, K), want, rtol=1e-13)


def test_remainder_keeps_its_accuracy_at_small_distances():
    # EvaluateRemainderTest.m:13-21: the leading terms of the series, which a direct difference loses
    r = np.array([1e-8, 1e-5, 1e-3])
    series = -1j * K + 1j * K**3 * r**2 / 6 - 1j * K**5 * r**4 / 120 - K**6 * r**5 / 720
    np.testing.assert_allclose(SI.remainder(r, K), series, rtol=1e-14)


def _random_moments(counts, seed):
    g = np.random.default_rng(seed)
    c = counts[0] * counts[1]
    moments = g.standard_normal((7, c)) + 1j * g.standard_normal((7, c))
    index = np.arange(c)
    return moments, np.stack([index % counts[0], index // counts[0]])  # offsets in column-major order


def _zero_parts(counts):
    xx = np.zeros((counts[0] - 1, counts[1]), np.complex128) if counts[0] > 1 else None
    yy = np.zeros((counts[0], counts[1] - 1), np.complex128) if counts[1] > 1 else None
    return A.Generators(xx, yy, np.zeros(counts, np.complex128), 3)


def _combine_along_rows(m00, m10, m01, m11):
    """Generator of the rooftops along the first axis from the moments of every offset d:
    (M00 - M10 - M01 + 2 M11)(d) + (M10 - M11)(d + 1) + (M01 - M11)(d - 1), where the pair at d - 1 = -1 is
    the reflection of the pair at +1, so (M01 - M11)(-1) stands for (M10 - M11)(1)."""
    rows = m00.shape[0] - 1
    g = m00[:rows] - m10[:rows] - m01[:rows] + 2 * m11[:rows] + (m10 - m11)[1:rows + 1]
    behind = np.concatenate([(m10 - m11)[1:2], (m01 - m11)[:rows - 1]])
    return g + behind


def _check_generators(parts, moments, counts, scales):
    grid = [moments[row].reshape(counts, order="F") for row in range(7)]
    np.testing.assert_allclose(parts.electric, scales[0] * grid[0], rtol=1e-15)
    if counts[0] > 1:
        np.testing.assert_allclose(parts.magnetic_xx, scales[1] * _combine_along_rows(*grid[:4]), rtol=1e-14)
    if counts[1] > 1:
        t = [grid[0].T, grid[4].T, grid[5].T, grid[6].T]
        np.testing.assert_allclose(parts.magnetic_yy, scales[1] * _combine_along_rows(*t).T, rtol=1e-14)


def test_moments_in_shuffled_chunks_build_the_generators():
    # tests/+unit/+assembler/+greensMatrix/+utils/AccumulateMomentsTest.m:5-22
    counts = (5, 4)
    moments, offsets = _random_moments(counts, 1)
    order = np.random.default_rng(11).permutation(offsets.shape[1])
    parts = _zero_parts(counts)
    for chunk in (order[:7], order[7:]):
        A.accumulate_moments(parts, moments[:, chunk], offsets[:, chunk], (2, 3))
    _check_generators(parts, moments, counts, (2, 3))


def test_chunks_may_end_inside_a_column():
    # AccumulateMomentsTest.m:24-37
    counts = (5, 4)
    moments, offsets = _random_moments(counts, 2)
    parts = _zero_parts(counts)
    for chunk in (slice(0, 7), slice(7, 13), slice(13, 20)):
        A.accumulate_moments(parts, moments[:, chunk], offsets[:, chunk], (2, 3))
    _check_generators(parts, moments, counts, (2, 3))


def test_a_one_cell_wide_grid_builds_only_its_y_generator():
    # AccumulateMomentsTest.m:39-48
    counts = (1, 6)
    moments, offsets = _random_moments(counts, 3)
    parts = A.accumulate_moments(_zero_parts(counts), moments, offsets, (2, 3))
    assert parts.magnetic_xx is None
    _check_generators(parts, moments, counts, (2, 3))


def test_a_missing_direction_is_skipped():
    # AccumulateMomentsTest.m:50-59
    counts = (6, 1)
    parts = A.accumulate_moments(_zero_parts(counts), np.ones((7, 6)), np.stack([np.arange(6), np.zeros(6, int)]),
                                 (1, 1))
    assert parts.magnetic_yy is None
    np.testing.assert_array_equal(parts.electric, np.ones((6, 1)))


# tests/+unit/+assembler/+singularIntegrals/+utils/IntegrateMonomialTest.m:9-52: G(a, b), the integral of
# u^m v^n R^p over [0, a] x [0, b], of which the moments are corner differences.
@pytest.mark.parametrize("power", [-1, 1, 3])
def test_monomial_integrals_vanish_on_the_axes(power):
    for m in range(4):
        for n in range(2):
            np.testing.assert_array_equal(SI.integrate_monomial(power, m, n, [0, 0.7, 0], [0.4, 0, 0]), [0, 0, 0])


@pytest.mark.parametrize("power", [-1, 1, 3])
def test_corner_differences_of_monomial_integrals_are_the_integrals(power):
    from scipy import integrate

    for a0, a1, b0, b1 in ((0.0, 0.6, 0.0, 0.25), (0.3, 0.8, 0.1, 0.9)):  # a corner at the singular point, and not
        for m in range(4):
            for n in range(2):
                def G(a, b):
                    return float(SI.integrate_monomial(power, m, n, a, b))

                want = integrate.dblquad(lambda v, u: u**m * v**n * (u * u + v * v) ** (power / 2), a0, a1, b0, b1,
                                         epsabs=0, epsrel=1e-13)[0]
                got = G(a1, b1) - G(a0, b1) - G(a1, b0) + G(a0, b0)
                assert got == pytest.approx(want, rel=1e-11)


@pytest.mark.parametrize("power", [-1, 1, 3])
def test_monomial_integrals_are_homogeneous(power):
    for m in range(4):
        for n in range(2):
            G = lambda a, b: float(SI.integrate_monomial(power, m, n, a, b))  # noqa: E731
            assert G(0.9, 2.4) == pytest.approx(3.0 ** (m + n + power + 2) * G(0.3, 0.8), rel=1e-14)


@pytest.mark.parametrize("power", [-1, 1, 3])
def test_monomial_integrals_exchange_their_arguments(power):
    G = lambda m, n, a, b: float(SI.integrate_monomial(power, m, n, a, b))  # noqa: E731
    assert G(0, 1, 0.3, 0.7) == pytest.approx(G(1, 0, 0.7, 0.3), rel=1e-14)
    assert G(1, 1, 0.3, 0.7) == pytest.approx(G(1, 1, 0.7, 0.3), rel=1e-14)


def test_extracted_moments_combine_the_power_moments():
    # tests/+unit/+assembler/+singularIntegrals/GenerateExtractedMomentsTest.m:5-18
    a, b = 0.1, 0.15
    want = SI.power_moments(a, b, -1) - K**2 / 2 * SI.power_moments(a, b, 1) + K**4 / 24 * SI.power_moments(a, b, 3)
    np.testing.assert_allclose(SI.extracted_moments(a, b, K), want, rtol=1e-15)
    np.testing.assert_array_equal(SI.extracted_moments(a, b, 0.0), SI.power_moments(a, b, -1))
