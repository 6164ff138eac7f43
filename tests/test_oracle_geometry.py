"""The oracle's rooftops, quadrature rules and constants, restating the reference's unit tests
tests/+unit/+basisFunctions/UniformRooftopsTest.m:5-58, +utils/GenerateGaussLegendre1DTest.m:5-34,
GaussLegendre2RectQuadratureTest.m:5-30 and tests/+unit/+assembler/ConstantsTest.m:5-20."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import geometry as G


def test_counts():
    rt = G.Rooftops(4, 3, 0.1, 0.1, 3)
    assert (rt.count_dir("x"), rt.count_dir("y"), rt.count) == (9, 8, 17)


@pytest.mark.parametrize("grid,content", [((4, 3), G.BOTH), ((4, 1), G.XONLY), ((1, 3), G.YONLY), ((1, 1), G.NONE)])
def test_content(grid, content):
    assert G.Rooftops(*grid, 0.1, 0.1, 3).content == content


def test_reference_rooftops():
    rt = G.Rooftops(4, 3, 0.1, 0.2, 3)
    _, _, w = G.quadrature_2d(rt.order)
    x = rt.reference_rooftop("x")
    assert tuple(x["second_face_offset"]) == (1, 0)
    assert (x["length"], x["height"]) == (0.1, 0.2)
    # a rooftop of unit height covers half of each of its two faces
    np.testing.assert_allclose(w @ x["amplitudes"], [0.5, 0.5], rtol=1e-14)
    y = rt.reference_rooftop("y")
    assert tuple(y["second_face_offset"]) == (0, 1)
    assert (y["length"], y["height"]) == (0.2, 0.1)


def test_amplitudes_rise_and_fall_along_the_direction():
    rt = G.Rooftops(4, 3, 0.1, 0.1, 3)
    pu, pv, _ = G.quadrature_2d(rt.order)
    np.testing.assert_array_equal(rt.reference_rooftop("x")["amplitudes"], np.stack([pu, 1 - pu], axis=1))
    np.testing.assert_array_equal(rt.reference_rooftop("y")["amplitudes"], np.stack([pv, 1 - pv], axis=1))


def test_edge_lengths():
    # rooftops 0 to 8 are x-directed (edges along y), 9 to 16 y-directed
    rt = G.Rooftops(4, 3, 0.1, 0.2, 3)
    np.testing.assert_array_equal(rt.edge_lengths([0, 8, 9, 16]), [0.2, 0.2, 0.1, 0.1])


@pytest.mark.parametrize("order", [1, 2, 5, 12])
def test_gauss_legendre_integrates_polynomials_exactly(order):
    p, w = G.gauss_legendre(order, 0.0, 1.0)
    for degree in range(2 * order):
        assert w @ p**degree == pytest.approx(1 / (degree + 1), rel=1e-14)


@pytest.mark.parametrize("order", [1, 2, 5, 12])
def test_gauss_legendre_points_ascend_inside_the_interval(order):
    p, _ = G.gauss_legendre(order, -2.0, 3.0)
    assert p.shape == (order,)
    assert np.all(np.diff(p) > 0)
    assert np.all((p > -2) & (p < 3))


def test_the_two_point_rule():
    p, w = G.gauss_legendre(2, -1.0, 1.0)
    np.testing.assert_allclose(p, [-1 / math.sqrt(3), 1 / math.sqrt(3)], atol=1e-15)
    np.testing.assert_allclose(w, [1.0, 1.0], atol=1e-15)


def test_the_face_rule_integrates_polynomials_exactly():
    order = 3
    pu, pv, w = G.quadrature_2d(order)
    for du in range(2 * order):
        for dv in range(2 * order):
            assert (pu**du * pv**dv) @ w == pytest.approx(1 / ((du + 1) * (dv + 1)), rel=1e-14)


def test_the_u_coordinate_runs_fastest():
    pu, pv, _ = G.quadrature_2d(2)
    np.testing.assert_array_equal(pu[:2], pu[2:4])
    assert pv[0] == pv[1]
    assert pu[0] < pu[1]


def test_constants_are_those_of_the_reference():
    # src/+rooftopMoM/+assembler/Constants.m:8-17 and tests/+unit/+assembler/ConstantsTest.m:5-20: c exact,
    # Z0 given, mu0 and epsilon0 derived from them and within CODATA 2018's uncertainty
    import rooftop_mom_b200.api as api

    assert G.SPEED_OF_LIGHT == api.SPEED_OF_LIGHT == 299792458.0
    assert G.Z0 == api.Z0 == 376.730313668
    assert G.SPEED_OF_LIGHT**2 * G.MU0 * G.EPSILON0 == pytest.approx(1.0, rel=4 * np.finfo(float).eps)
    assert math.sqrt(G.MU0 / G.EPSILON0) == pytest.approx(G.Z0, rel=4 * np.finfo(float).eps)
    assert G.MU0 == pytest.approx(1.25663706212e-6, rel=1.5e-10)
    assert G.EPSILON0 == pytest.approx(8.8541878128e-12, rel=1.5e-10)
