"""The oracle's generator assembly against its definition, restating the reference's unit tests
tests/+unit/+assembler/+greensMatrix/MomentAssemblerTest.m:5-19 (generator sizes and content),
:45-56 (tiling of the far pass does not change the result) and :95-119 (touching entries against an
adaptive integration of the Green's function itself, with no singularity extracted)."""
from __future__ import annotations

import math

import numpy as np
from scipy import integrate

from oracle import assembly as A
from oracle.geometry import BOTH, XONLY, Z0

K = 2 * math.pi

# Rooftop weights of the moments over nu in [-1, 1] (one per kind alpha + 2 beta): W00, W10, W01, W11.
_WEIGHTS = (
    lambda v: 1 - abs(v),
    lambda v: (1 + v) ** 2 / 2 if v < 0 else (1 - v * v) / 2,
    lambda v: (1 - v * v) / 2 if v < 0 else (1 - v) ** 2 / 2,
    lambda v: (1 - abs(v)) ** 2 * (2 + abs(v)) / 6,
)


def _adaptive_moment(sizes, offset, kinds):
    """M_{alpha beta} of exp(-ikR)/R at a touching offset, integrated adaptively over the quadrants of
    [-1, 1]^2, each of which has the singular point at a corner."""
    weight = _WEIGHTS[kinds[0] + 2 * kinds[1]]

    def integrand(eta, nu, part):
        r = math.hypot(sizes[0] * (nu - offset[0]), sizes[1] * (eta - offset[1]))
        v = weight(nu) * (1 - abs(eta)) * complex(math.cos(K * r), -math.sin(K * r)) / r
        return v.real if part == 0 else v.imag

    total = 0j
    for a0, a1 in ((-1, 0), (0, 1)):
        for b0, b1 in ((-1, 0), (0, 1)):
            re = integrate.dblquad(integrand, a0, a1, b0, b1, args=(0,), epsabs=0, epsrel=1e-12)[0]
            im = integrate.dblquad(integrand, a0, a1, b0, b1, args=(1,), epsabs=0, epsrel=1e-12)[0]
            total += re + 1j * im
    return total


def test_generator_sizes_and_content():
    g = A.generate(5, 4, 0.1, 0.1, K, (3, 3))
    assert g.magnetic_xx.shape == (4, 4)
    assert g.magnetic_yy.shape == (5, 3)
    assert g.electric.shape == (5, 4)
    assert g.content == BOTH


def test_a_strip_has_one_direction():
    g = A.generate(6, 1, 0.1, 0.1, K, (3, 3))
    assert g.magnetic_xx.shape == (5, 1)
    assert g.magnetic_yy is None
    assert g.content == XONLY


def test_tiling_of_the_far_pass_does_not_change_the_result():
    counts, sizes, order = (5, 4), (0.1, 0.15), 3
    rule = A.reduced_rule(order, (1, 1))
    scales = A.scales_of(sizes[0], sizes[1], K)
    out = []
    for tile in (None, 1):
        e, xx, yy = A.allocate_parts(counts, (4 * 4, 5 * 3))
        parts = A.Generators(xx, yy, e, BOTH)
        A.integrate_lattice(parts, counts, sizes, K, rule, order, (2, 2), scales, column_tile=tile)
        out.append(parts)
    for name in ("electric", "magnetic_xx", "magnetic_yy"):
        np.testing.assert_allclose(getattr(out[1], name), getattr(out[0], name), rtol=1e-14)


def test_touching_entries_match_adaptive_integration():
    sizes = (0.1, 0.15)
    g = A.generate(3, 3, *sizes, K, (16, 8))
    scale = 1j * Z0 / (4 * math.pi) * (sizes[0] * sizes[1]) ** 2
    for offset in ((0, 0), (1, 0), (0, 1), (1, 1)):
        want = scale / K * _adaptive_moment(sizes, offset, (0, 0))
        assert abs(g.electric[offset] - want) <= 1e-10 * abs(want)
    # the rooftop at the origin: its wedge pairs meet in the cell pairs at the offsets (0, 0) and (1, 0)
    c = [_adaptive_moment(sizes, (0, 0), kinds) for kinds in ((0, 0), (1, 0), (0, 1), (1, 1))]
    neighbour = _adaptive_moment(sizes, (1, 0), (1, 0)) - _adaptive_moment(sizes, (1, 0), (1, 1))
    want = scale * K * (c[0] - c[1] - c[2] + 2 * c[3] + 2 * neighbour)
    assert abs(g.magnetic_xx[0, 0] - want) <= 1e-10 * abs(want)
