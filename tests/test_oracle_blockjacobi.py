"""The block-Jacobi oracle against the dense Green's matrix it restates (the reference's dense definition,
tests/+unit/Base.m:83-113, as oracle.excitation.dense_matrix): every entry it forms equals the dense
matrix's, the blocks partition the rooftops, and applying it inverts each diagonal block of the dense
matrix. Block-Jacobi is not in the reference, so this is its only pin on the CPU; the GPU build is
compared with this oracle in the GPU tests."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import assembly as A
from oracle import blockjacobi as BJ
from oracle import excitation as EX
from oracle.geometry import Rooftops

CASES = [((5, 4), (2, 2)), ((7, 5), (2, 2)), ((6, 1), (2, 2)), ((1, 5), (2, 2)), ((5, 4), (3, 1)), ((4, 6), (1, 3))]


def _built(grid):
    rt = Rooftops(grid[0], grid[1], 0.1, 0.15, 3)
    gen = A.generate(grid[0], grid[1], 0.1, 0.15, 2 * math.pi, (3, 3))
    return rt, gen, EX.dense_matrix(gen, rt)


@pytest.mark.parametrize("grid,block", CASES)
def test_blocks_partition_the_rooftops(grid, block):
    rt, _, _ = _built(grid)
    idx = np.concatenate([b[0] for b in BJ.block_indices(rt, *block) if b[0].size])
    assert np.array_equal(np.sort(idx), np.arange(rt.count))


@pytest.mark.parametrize("grid,block", CASES)
def test_entries_are_the_dense_matrix(grid, block):
    rt, gen, dense = _built(grid)
    for idx, dirs, faces in BJ.block_indices(rt, *block):
        for a in range(idx.size):
            for b in range(idx.size):
                got = BJ.entry(gen, rt, dirs[a], tuple(faces[a]), dirs[b], tuple(faces[b]))
                assert got == pytest.approx(dense[idx[a], idx[b]], rel=1e-13, abs=1e-13 * abs(dense).max())


@pytest.mark.parametrize("grid,block", CASES)
def test_apply_inverts_each_diagonal_block(grid, block):
    rt, gen, dense = _built(grid)
    g = np.random.default_rng(4)
    x = g.standard_normal(rt.count) + 1j * g.standard_normal(rt.count)
    y = BJ.BlockJacobi(gen, rt, *block).apply(x)
    for idx, _, _ in BJ.block_indices(rt, *block):
        if idx.size:
            want = np.linalg.solve(dense[np.ix_(idx, idx)], x[idx])
            np.testing.assert_allclose(y[idx], want, rtol=1e-11, atol=1e-11 * np.abs(want).max())
