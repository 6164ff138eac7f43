"""Pins of the oracle's circulant kernels and spatial blocks against the reference's own known answers
(tests/+unit/+assembler/+preconditioner/+kernels/KernelsTest.m and
tests/+unit/+assembler/+preconditioner/+utils/GenerateSpatialBlocksTest.m): the superoptimal kernel
against its definition through dense two-level Toeplitz and Fourier matrices, its symmetry for even
generators, reversal of the generator transposing every circulant, and the spatial blocks reproducing the
dense Green's matrix."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import assembly as A
from oracle import excitation as EX
from oracle import geometry as G
from oracle import preconditioner as PC


def _toeplitz(g):
    """Dense two-level Toeplitz matrix of a two-sided generator, x index fastest (KernelsTest Base.m)."""
    gx, gy = (g.shape[0] + 1) // 2, (g.shape[1] + 1) // 2
    m, n = np.meshgrid(np.arange(gx), np.arange(gy), indexing="ij")
    m, n = m.ravel(order="F"), n.ravel(order="F")
    return g[m[:, None] - m[None, :] + gx - 1, n[:, None] - n[None, :] + gy - 1]


def _fourier(gx, gy):
    return np.kron(np.fft.fft(np.eye(gy)), np.fft.fft(np.eye(gx))) / np.sqrt(gx * gy)


def test_superoptimal_matches_its_definition():
    rng = np.random.default_rng(1)
    g = rng.standard_normal((7, 5)) + 1j * rng.standard_normal((7, 5))
    T = _toeplitz(g)
    F = _fourier(4, 3)
    expected = np.diag(F @ (T @ T.conj().T) @ F.conj().T) / np.conj(np.diag(F @ T @ F.conj().T))
    actual = np.fft.fft2(PC.superoptimal(g)).ravel(order="F")
    assert np.max(np.abs(actual - expected)) <= 1e-12 * np.max(np.abs(expected))


def test_superoptimal_of_an_even_generator_is_symmetric():
    rng = np.random.default_rng(1)
    c = PC.superoptimal(PC.extend_evenly(rng.standard_normal((5, 4)) + 1j * rng.standard_normal((5, 4))))
    ix, iy = np.r_[0, np.arange(4, 0, -1)], np.r_[0, np.arange(3, 0, -1)]
    assert np.max(np.abs(c - c[np.ix_(ix, iy)])) <= 1e-13 * np.max(np.abs(c))


@pytest.mark.parametrize("kernel", ["strang", "tChan", "rChan", "huckle", "superoptimal"])
def test_reversed_generator_gives_the_transposed_circulant(kernel):
    rng = np.random.default_rng(1)
    g = rng.standard_normal((11, 9))
    fn, _ = PC._kernel_fn(kernel, (3, 2))
    c = fn(g)
    ix, iy = np.r_[0, np.arange(5, 0, -1)], np.r_[0, np.arange(4, 0, -1)]
    assert np.max(np.abs(fn(np.rot90(g, 2)) - c[np.ix_(ix, iy)])) <= 1e-12 * max(1.0, np.max(np.abs(c)))


def test_strang_and_tchan_keep_a_circulant():
    rng = np.random.default_rng(1)
    circ = rng.standard_normal((6, 5))
    g = circ[np.ix_(np.mod(np.arange(-5, 6), 6), np.mod(np.arange(-4, 5), 5))]
    assert np.max(np.abs(PC.strang(g) - circ)) <= 1e-14
    assert np.max(np.abs(PC.t_chan(g) - circ)) <= 1e-14


@pytest.mark.parametrize("grid", [(4, 3), (2, 3), (5, 1), (1, 4)])
def test_spatial_blocks_reproduce_the_greens_matrix(grid):
    cx, cy = grid
    a, b = 0.1, 0.15
    gen = A.generate(cx, cy, a, b, 2 * np.pi, orders=(3, 3))
    rt = G.Rooftops(cx, cy, a, b, 3)
    M = EX.dense_matrix(gen, rt)
    blocks = PC.spatial_blocks(gen, a, b)
    table = [[blocks[0], blocks[1]], [blocks[2], blocks[3]]]
    counts = [rt.grid_size("x")[0] * rt.grid_size("x")[1], rt.grid_size("y")[0] * rt.grid_size("y")[1]]
    first = [0, counts[0]]

    def faces(d):
        rows, _ = rt.grid_size(d)
        ii = np.arange(counts["xy".index(d)])
        return ii % rows, ii // rows

    for m, dm in enumerate("xy"):
        for n, dn in enumerate("xy"):
            if not counts[m] or not counts[n]:
                continue
            (im, jm), (in_, jn) = faces(dm), faces(dn)
            blk = table[m][n][im[:, None] - in_[None, :] + cx - 1, jm[:, None] - jn[None, :] + cy - 1]
            want = M[first[m]:first[m] + counts[m], first[n]:first[n] + counts[n]]
            assert np.max(np.abs(blk - want)) <= 1e-13 * np.max(np.abs(M))
