"""The byte models against the objects they describe once the oracle has built them, on the grids of the
reference's tests/+unit/+resources/EstimateMemoryTest.m:5-44 (plates, strips, the smallest plate and sizes
that need a larger fast FFT): the generators, the stored spectra of the three products and the stored
spectra of a partwise circulant preconditioner. The same models are the admission contract of the C ABI
(rtm_estimate_bytes, checked against them in test_abi.py)."""
from __future__ import annotations

import math

import pytest

from oracle import assembly as A
from oracle import excitation as EX
from oracle import preconditioner as PC
from oracle import spectra as S
from oracle.geometry import Rooftops

GRIDS = [(4, 3), (7, 1), (1, 6), (2, 2), (9, 5), (13, 11)]


def _bytes(*arrays):
    return sum(a.size * 16 for a in arrays if a is not None)  # complex doubles


def _spectra_bytes(s):
    return _bytes(s.xx, s.xy, s.yx, s.yy)


def _built(grid):
    rt = Rooftops(grid[0], grid[1], 0.1, 0.15, 2)
    return rt, A.generate(grid[0], grid[1], 0.1, 0.15, 2 * math.pi, (2, 2))


@pytest.mark.parametrize("grid", GRIDS)
def test_generators(grid):
    rt, gen = _built(grid)
    assert EX.estimate_generators(rt) == _bytes(gen.magnetic_xx, gen.magnetic_yy, gen.electric)


@pytest.mark.parametrize("product", ["fft", "splitFFT", "leanSplitFFT"])
@pytest.mark.parametrize("grid", GRIDS)
def test_stored_product(grid, product):
    rt, gen = _built(grid)
    if product == "fft":
        stored = _spectra_bytes(S.embedding_spectra(gen, rt.size_x, rt.size_y))
    else:
        stored = sum(_spectra_bytes(s) for s in S.subband_spectra(gen, rt.size_x, rt.size_y))
    assert EX.estimate_product(rt, product)[0] == stored


@pytest.mark.parametrize("grid", GRIDS)
def test_stored_preconditioner(grid):
    rt, gen = _built(grid)
    spectra = PC.circulant_spectra(gen, rt.size_x, rt.size_y, kernel="tChan", builder="partwise")
    assert EX.estimate_preconditioner(rt)[0] == _spectra_bytes(spectra)
