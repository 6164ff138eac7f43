"""The oracle's excitations and outputs, restating the reference's unit tests
tests/+unit/+operator/GeneratePlaneWaveTest.m:5-49, GenerateDeltaGapTest.m:5-14,
+utils/GenerateMiddlePortTest.m:5-20, ComputeRadarCrossSectionTest.m:5-23 and
ComputeInputImpedanceTest.m:5-35."""
from __future__ import annotations

import math

import numpy as np
import pytest
from scipy import integrate

from oracle import assembly as A
from oracle import excitation as EX
from oracle.geometry import Z0, Rooftops

K = 2 * math.pi


def test_normal_incidence_gives_the_face_area():
    # a rooftop of unit height covers half of each of its two faces: one face area in total
    rt = Rooftops(4, 3, 0.1, 0.2, 3)
    got = EX.plane_wave(rt, K, [0, 0, -1], [0.6, 0.8, 0], 2)
    want = np.r_[np.full(9, 2 * 0.6 * 0.02), np.full(8, 2 * 0.8 * 0.02)]
    np.testing.assert_allclose(got, want, rtol=1e-14)


def test_a_strip_has_only_its_direction():
    rt = Rooftops(6, 1, 0.1, 0.02, 3)
    np.testing.assert_allclose(EX.plane_wave(rt, K, [0, 0, -1], [1, 0, 0], 1), np.full(5, 0.1 * 0.02), rtol=1e-14)


def test_phase_follows_the_direction_of_propagation():
    rt = Rooftops(4, 3, 0.1, 0.2, 3)
    d = np.array([1, 2, -2]) / 3
    e = EX.plane_wave(rt, K, d, np.array([2, -1, 0]) / math.sqrt(5), 1)
    part_x = e[:9].reshape(3, 3, order="F")
    part_y = e[9:].reshape(4, 2, order="F")
    np.testing.assert_allclose(part_x[1:] / part_x[:-1], np.full((2, 3), np.exp(-1j * K * d[0] * 0.1)), rtol=1e-13)
    np.testing.assert_allclose(part_y[:, 1] / part_y[:, 0], np.full(4, np.exp(-1j * K * d[1] * 0.2)), rtol=1e-13)


def test_plane_wave_matches_adaptive_integration():
    # one x-directed rooftop, rising over [0, 0.1] x [0, 0.2] and falling over the next face
    rt = Rooftops(2, 1, 0.1, 0.2, 8)
    d = np.array([1, 2, -2]) / 3
    p = np.array([2, -1, 0]) / math.sqrt(5)
    got = EX.plane_wave(rt, K, d, p, 1)

    def wave(x, y):
        return p[0] * np.exp(-1j * K * (d[0] * x + d[1] * y))

    def part(shape, x0, x1):
        re = integrate.dblquad(lambda y, x: (shape(x) * wave(x, y)).real, x0, x1, 0, 0.2, epsabs=1e-16, epsrel=1e-13)
        im = integrate.dblquad(lambda y, x: (shape(x) * wave(x, y)).imag, x0, x1, 0, 0.2, epsabs=1e-16, epsrel=1e-13)
        return re[0] + 1j * im[0]

    want = part(lambda x: x / 0.1, 0.0, 0.1) + part(lambda x: (0.2 - x) / 0.1, 0.1, 0.2)
    np.testing.assert_allclose(got, [want], rtol=1e-12)


def test_delta_gap_is_the_voltage_times_the_edge_length():
    # rooftops 1 and 4 are x-directed (edges 0.2), rooftop 10 is y-directed (edge 0.1); 0-based indices
    rt = Rooftops(4, 3, 0.1, 0.2, 3)
    want = np.zeros(17)
    want[[1, 4]] = 3 * 0.2
    want[10] = 3 * 0.1
    np.testing.assert_array_equal(EX.delta_gap(rt, [1, 4, 10], 3), want)


@pytest.mark.parametrize("counts,direction,want", [
    ((6, 1), "x", [2]),  # the edge between the third and fourth of six faces
    ((5, 1), "x", [1]),  # five faces: the edge just before the middle
    ((1, 6), "y", [2]),
    ((4, 3), "x", [1, 4, 7]),  # second row of the 3 x 3 x-directed rooftops
    ((4, 3), "y", [9, 10, 11, 12]),  # first column of the 4 x 2 y-directed ones, after the 9 x-directed
])
def test_middle_port(counts, direction, want):
    np.testing.assert_array_equal(EX.middle_port(Rooftops(*counts, 0.1, 0.1, 3), direction), want)


def test_radar_cross_section_value():
    # excitation^T current = 2i
    got = EX.radar_cross_section(2, np.array([1, 1j]), np.array([1j, 1]), 1)
    assert got == pytest.approx((2 * Z0) ** 2 * 4 / (4 * math.pi), rel=1e-15)


def test_radar_cross_section_does_not_depend_on_the_intensity():
    g = np.random.default_rng(3)
    e = g.standard_normal(5) + 1j * g.standard_normal(5)
    j = g.standard_normal(5) + 1j * g.standard_normal(5)
    assert EX.radar_cross_section(K, 3 * e, 3 * j, 3) == pytest.approx(EX.radar_cross_section(K, e, j, 1), rel=1e-14)


def test_input_impedance_is_the_voltage_over_the_port_current():
    rt = Rooftops(4, 3, 0.1, 0.2, 3)
    current = np.zeros(17, dtype=np.complex128)
    current[[1, 4]] = [1 + 2j, 3]
    got = EX.input_impedance(rt, current, [1, 4], 5)
    assert got == pytest.approx(5 / ((4 + 2j) * 0.2), rel=1e-15)


def test_input_impedance_does_not_depend_on_the_scale():
    """A half-wave strip dipole scaled together with the wavelength keeps its input impedance."""

    def dipole(scale):
        rt = Rooftops(20, 1, scale * 0.025, scale * 0.004, 4)
        gen = A.generate(20, 1, rt.size_x, rt.size_y, K / scale, (4, 4))
        port = EX.middle_port(rt, "x")
        current = np.linalg.solve(EX.dense_matrix(gen, rt), EX.delta_gap(rt, port, 1))
        return EX.input_impedance(rt, current, port, 1)

    assert dipole(10) == pytest.approx(dipole(1), rel=1e-10)
