"""The oracle's three products against the dense Green's matrix on the grids of the reference's
tests/+unit/+assembler/+greensMatrix/ApplicatorTest.m:5-34 (plates, an odd plate, a plate two faces
wide and strips along both directions), and the per-frequency inverse of the block spectra
(tests/+unit/+assembler/+greensMatrix/SpectraTest.m:5-29)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import assembly as A
from oracle import excitation as EX
from oracle import spectra as S
from oracle.geometry import BOTH, XONLY, Rooftops

GRIDS = {
    "plate": (5, 4, 0.1, 0.15),
    "oddPlate": (11, 7, 0.1, 0.1),
    "twoFacesWide": (2, 5, 0.1, 0.1),
    "stripX": (9, 1, 0.1, 0.02),
    "stripY": (1, 6, 0.03, 0.1),
}


def _product(kind, rt, gen):
    if kind == "fft":
        spec = S.embedding_spectra(gen, rt.size_x, rt.size_y)
        return lambda x: S.fft_apply(rt, spec, rt.content, x)
    sub = S.subband_spectra(gen, rt.size_x, rt.size_y)
    apply = S.split_apply if kind == "splitFFT" else S.lean_apply
    return lambda x: apply(rt, sub, rt.content, x)


@pytest.mark.parametrize("grid", sorted(GRIDS))
@pytest.mark.parametrize("kind", ["fft", "splitFFT", "leanSplitFFT"])
def test_products_match_the_dense_matrix(kind, grid):
    cx, cy, a, b = GRIDS[grid]
    rt = Rooftops(cx, cy, a, b, 3)
    gen = A.generate(cx, cy, a, b, 2 * math.pi, (3, 3))
    g = np.random.default_rng(1)
    x = g.standard_normal(rt.count) + 1j * g.standard_normal(rt.count)
    want = EX.dense_matrix(gen, rt) @ x
    got = _product(kind, rt, gen)(x)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-12


def test_inverse_times_the_spectra_is_the_identity():
    g = np.random.default_rng(1)

    def block():
        return g.standard_normal((4, 3)) + 1j * g.standard_normal((4, 3))

    s = S.Spectra(block(), block(), block(), block())
    inv = s.invert(BOTH)
    one, zero = np.ones((4, 3)), np.zeros((4, 3))
    np.testing.assert_allclose(s.xx * inv.xx + s.xy * inv.yx, one, atol=1e-12)
    np.testing.assert_allclose(s.xx * inv.xy + s.xy * inv.yy, zero, atol=1e-12)
    np.testing.assert_allclose(s.yx * inv.xx + s.yy * inv.yx, zero, atol=1e-12)
    np.testing.assert_allclose(s.yx * inv.xy + s.yy * inv.yy, one, atol=1e-12)


def test_inverse_of_a_strip_is_the_reciprocal():
    inv = S.Spectra(np.array([2.0, 4.0]), None, None, None).invert(XONLY)
    np.testing.assert_array_equal(inv.xx, [0.5, 0.25])
    assert inv.yy is None


def test_grid_size_of_the_spectra():
    assert S.Spectra(None, None, None, np.zeros((3, 5), np.complex128)).grid_size() == (3, 5)
