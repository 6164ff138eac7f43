"""Physical and algebraic invariants the reference's tests hold (ResultTest.m:27-37,
ComputeInputImpedanceTest.m:16-22, PreconditionerTest.m:33-55), on the GPU path: results scale exactly with
the wavelength, every circulant preconditioner is complex symmetric, and a circulant cuts COCG's iterations."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _plate_rcs(wavelength):
    import rooftop_mom_b200 as R

    h = wavelength / 10
    prob = R.Problem(R.Mesh(12, 10, h, h), 2 * math.pi / wavelength)
    exc = R.Excitation.planeWave(prob, direction=(0, 0, -1), polarization=(1, 0, 0))
    res = R.Solver(method="cg", tolerance=1e-10, maxIterationCount=3000).solve(R.Operator(prob), exc)
    assert res.converged()
    return res


def test_normalized_rcs_does_not_depend_on_the_scale():
    small, large = _plate_rcs(1.0), _plate_rcs(2.0)
    assert large.radarCrossSection() == pytest.approx(4 * small.radarCrossSection(), rel=1e-8)
    assert large.normalizedRadarCrossSection() == pytest.approx(small.normalizedRadarCrossSection(), rel=1e-8)


def _dipole_impedance(scale):
    import rooftop_mom_b200 as R

    # a strip half a wavelength long (20 faces of 0.025) and 0.004 wide at the wavelength `scale`
    prob = R.Problem(R.Mesh(20, 1, 0.025 * scale, 0.004 * scale), 2 * math.pi / scale)
    gap = R.Excitation.deltaGap(prob, direction="x", voltage=1.0)
    res = R.Solver(method="cg", tolerance=1e-12, maxIterationCount=3000).solve(R.Operator(prob), gap)
    assert res.converged()
    return res.inputImpedance()


def test_input_impedance_does_not_depend_on_the_scale():
    z1, z10 = _dipole_impedance(1.0), _dipole_impedance(10.0)
    assert abs(z10 - z1) <= 1e-10 * abs(z1)


@pytest.mark.parametrize("builder", ["partwise", "blockwise", "hybrid"])
@pytest.mark.parametrize("kernel", ["strang", "tChan", "rChan", "huckle", "superoptimal"])
def test_every_circulant_preconditioner_is_complex_symmetric(kernel, builder):
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(5, 4, 0.1, 0.15), 2 * math.pi, quadratureOrder=3)
    bw = (2, 2) if kernel == "huckle" else None
    pc = R.Preconditioner(prob, kernel=kernel, builder=builder, bandwidth=bw)
    g = np.random.default_rng(1)
    n = prob.rooftopCount()
    x = g.standard_normal(n) + 1j * g.standard_normal(n)
    y = g.standard_normal(n) + 1j * g.standard_normal(n)
    a, b = x @ pc.apply(y), y @ pc.apply(x)
    # the superoptimal spectra come out of ~40 transforms and a division: 1e-10
    assert abs(a - b) <= (1e-10 if kernel == "superoptimal" else 1e-12) * abs(a)


def test_a_blockwise_circulant_cuts_the_iterations():
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(16, 16, 0.05, 0.05), 2 * math.pi, quadratureOrder=3)
    op = R.Operator(prob)
    exc = R.Excitation.planeWave(prob)
    solver = R.Solver(method="cg", tolerance=1e-8, maxIterationCount=3000)
    plain = solver.solve(op, exc)
    pre = solver.solve(op, exc, preconditioner=R.Preconditioner(prob, kernel="rChan", builder="blockwise"))
    assert pre.converged() and pre.iterationCount() < plain.iterationCount()
    if plain.converged():
        assert rel(pre.solution(), plain.solution()) < 1e-6
