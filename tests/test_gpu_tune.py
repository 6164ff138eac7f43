"""The autotuner of the split product (rtm_tune_product): what it measures, that the products built after it
take its choice, and that those products still match the oracle (a transform grid larger than the
reference's gives the same product up to rounding)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import random_vector, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _forget_tuning():
    import rooftop_mom_b200 as R

    R.clearTuning()
    yield
    R.clearTuning()


@pytest.mark.parametrize("count,precision", [((200, 120), "double"), ((300, 64), "single"), ((64, 64), "double")])
def test_tuned_products_match_the_oracle(count, precision):
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, spectra as S

    cx, cy = count
    h = 0.05
    mesh = R.Mesh(cx, cy, h, h)
    choice = R.tuneProduct(mesh, precision=precision)
    assert choice["candidates"] >= 1 and choice["seconds"] > 0
    assert choice["seconds"] <= choice["referenceSeconds"] * 1.0001
    assert choice["fftSize"][0] >= cx and choice["fftSize"][1] >= cy
    prob = R.Problem(mesh, 2 * math.pi, quadratureOrder=3)
    op = R.Operator(prob, precision=precision)
    assert (op.info()["fft_x"], op.info()["fft_y"]) == choice["fftSize"]
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, h, h, 3)
    want_sub = S.subband_spectra(A.Generators(xx, yy, e, rt.content), h, h)
    v = random_vector(rt.count, seed=11)
    want = S.split_apply(rt, want_sub, rt.content, v)
    assert rel(op.apply(v), want) < (1e-13 if precision == "double" else 2e-5)


def test_the_reference_sizes_stay_when_asked():
    import rooftop_mom_b200 as R

    mesh = R.Mesh(200, 120, 0.05, 0.05)
    choice = R.tuneProduct(mesh, referenceSizes=True)
    assert choice["fftSize"] == (R.fast_fft_size(200), R.fast_fft_size(120))


def test_every_schedule_of_a_power_of_two_grid_is_measured():
    """FP64 256 x 256: y passes with 1, 2 or 3 CTAs an SM times the x-mix forms (3 direct, pipelined)."""
    import rooftop_mom_b200 as R

    choice = R.tuneProduct(R.Mesh(256, 256, 0.05, 0.05))
    assert choice["candidates"] == 12
    assert choice["fftSize"] == (256, 256)
    assert 1 <= choice["yBlocks"] <= 3 and 0 <= choice["mixKind"] <= 3


def test_solves_on_tuned_products_converge_like_untuned_ones():
    import rooftop_mom_b200 as R

    mesh = R.Mesh(100, 72, 1 / 20, 1 / 20)
    prob = R.Problem(mesh, 2 * math.pi)
    exc = R.Excitation.planeWave(prob)
    plain = R.Solver(method="gmres", tolerance=1e-8, restart=50, maxIterationCount=5000).solve(R.Operator(prob), exc)
    R.tuneProduct(mesh)
    tuned = R.Solver(method="gmres", tolerance=1e-8, restart=50, maxIterationCount=5000).solve(R.Operator(prob), exc)
    assert plain.converged() and tuned.converged()
    assert abs(plain.iterationCount() - tuned.iterationCount()) <= 3
    assert rel(tuned.solution(), plain.solution()) < 1e-7


def test_invalid_tuning_requests_are_rejected():
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    with pytest.raises(L.RtmError):
        R.tuneProduct(R.Mesh(1, 50, 0.05, 0.05))
    with pytest.raises(L.RtmError):
        R.tuneProduct(R.Mesh(50, 50, 0.05, 0.05), nrhs=0)
