"""The oracle's circulant building blocks against their definitions, restating the reference's unit tests
tests/+unit/+assembler/+preconditioner/+utils/FoldGeneratorTest.m:5-45, ExtendEvenlyTest.m:5-15,
GeneratePartSpectraTest.m:9-28, GenerateOptimalOfProductTest.m:9-24 and
+kernels/KernelsTest.m:36-104: folding puts the windowed offset p of a count-n direction at p mod n, the
even extension mirrors both offsets, the four part spectra sum to the two-level Toeplitz matrix, the
optimal circulant of a product keeps the diagonal of the product in the Fourier basis, and each kernel
places and weights the offsets as its window says."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import preconditioner as PC


def _toeplitz(g):
    """Dense two-level Toeplitz matrix of a two-sided generator, x index fastest."""
    gx, gy = (g.shape[0] + 1) // 2, (g.shape[1] + 1) // 2
    m, n = np.meshgrid(np.arange(gx), np.arange(gy), indexing="ij")
    m, n = m.ravel(order="F"), n.ravel(order="F")
    return g[m[:, None] - m[None, :] + gx - 1, n[:, None] - n[None, :] + gy - 1]


def _fourier(gx, gy):
    return np.kron(np.fft.fft(np.eye(gy)), np.fft.fft(np.eye(gx))) / np.sqrt(gx * gy)


def _fold_by_definition(g, window):
    """c(d) = sum over the offsets p = d mod n of w_x(p) w_y(q) g(p, q), for a two-sided generator."""
    cx, cy = (g.shape[0] + 1) // 2, (g.shape[1] + 1) // 2
    out = np.zeros((cx, cy), dtype=np.result_type(g, float))
    for i, p in enumerate(range(-(cx - 1), cx)):
        for j, q in enumerate(range(-(cy - 1), cy)):
            wx = window(np.array([p]), cx, 1)[0]
            wy = window(np.array([q]), cy, 2)[0]
            out[p % cx, q % cy] += wx * wy * g[i, j]
    return out


def test_fold_of_a_four_point_toeplitz_with_the_t_chan_window():
    g = (np.arange(-3, 4) + 10.0).reshape(7, 1)

    def window(o, n, d):
        return (n - np.abs(o)) / n

    got = PC.fold_generator(g, window)
    np.testing.assert_allclose(got, _fold_by_definition(g, window), atol=1e-14)
    # t(0) alone at 0; t(1) and t(-3) at 1 with weights 3/4 and 1/4
    assert got[0, 0] == pytest.approx(10.0, abs=1e-14)
    assert got[1, 0] == pytest.approx((3 * 11 + 7) / 4, abs=1e-14)


def test_one_sided_even_fold_is_the_fold_of_the_even_extension():
    g = np.random.default_rng(1)
    gen = g.standard_normal((6, 5)) + 1j * g.standard_normal((6, 5))

    def window(o, n, d):  # deliberately not even
        return (n + o + d) / n

    np.testing.assert_allclose(PC.fold_generator(gen, window, even=True),
                               PC.fold_generator(PC.extend_evenly(gen), window), atol=1e-14)


def test_unit_weights_fold_along_both_directions():
    g = np.arange(1.0, 16.0).reshape(3, 5, order="F")

    def window(o, n, d):
        return np.ones(np.shape(o))

    got = PC.fold_generator(g, window)
    assert got.shape == (2, 3)
    np.testing.assert_array_equal(got, _fold_by_definition(g, window))


def test_extend_evenly_mirrors_both_offsets():
    np.testing.assert_array_equal(PC.extend_evenly(np.array([[1, 2], [3, 4]])),
                                  np.array([[4, 3, 4], [2, 1, 2], [4, 3, 4]]))
    assert PC.extend_evenly(None) is None


@pytest.mark.parametrize("grid", [(4, 3), (6, 1), (1, 5)])
def test_part_spectra_sum_to_the_toeplitz_matrix(grid):
    g = np.random.default_rng(1)
    shape = (2 * grid[0] - 1, 2 * grid[1] - 1)
    gen = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    spectra = PC.part_spectra(gen)
    F = _fourier(*grid)
    mod_x = [np.ones(grid[0]), np.exp(1j * np.pi * np.arange(grid[0]) / grid[0])]
    mod_y = [np.ones(grid[1]), np.exp(1j * np.pi * np.arange(grid[1]) / grid[1])]
    total = np.zeros((grid[0] * grid[1],) * 2, dtype=np.complex128)
    for m in range(2):
        for n in range(2):
            D = np.diag(np.kron(mod_y[n], mod_x[m]))
            total += D.conj().T @ F.conj().T @ np.diag(spectra[m][n].ravel(order="F")) @ F @ D
    np.testing.assert_allclose(total, _toeplitz(gen), atol=1e-13)


@pytest.mark.parametrize("grid", [(4, 3), (5, 4), (6, 1), (1, 5)])
def test_optimal_of_a_product_keeps_the_fourier_diagonal(grid):
    g = np.random.default_rng(1)
    shape = (2 * grid[0] - 1, 2 * grid[1] - 1)
    ga = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    gb = g.standard_normal(shape) + 1j * g.standard_normal(shape)
    got = PC.optimal_of_product(PC.part_spectra(ga), PC.part_spectra(gb))
    F = _fourier(*grid)
    product = _toeplitz(ga) @ _toeplitz(gb).conj().T
    want = np.diag(F @ product @ F.conj().T).reshape(grid, order="F")
    np.testing.assert_allclose(got, want, atol=1e-12 * np.abs(want).max())


# The kernels (tests/+unit/+assembler/+preconditioner/+kernels/KernelsTest.m:36-104), on the even extension
# of one-sided generators with integer entries, so every sum is exact.
def _one_sided(rows, cols):
    return np.arange(1.0, rows * cols + 1).reshape(rows, cols, order="F")


@pytest.mark.parametrize("kernel", [PC.t_chan, PC.r_chan])
@pytest.mark.parametrize("grid", [(5, 4), (1, 6), (7, 1)])
def test_t_chan_and_r_chan_fold_an_even_generator_one_sided(kernel, grid):
    g = np.random.default_rng(1)
    gen = g.standard_normal(grid) + 1j * g.standard_normal(grid)
    np.testing.assert_allclose(kernel(gen, even=True), kernel(PC.extend_evenly(gen)), atol=1e-14)
    assert kernel(None, even=True) is None


def test_strang_copies_the_central_offsets():
    g = _one_sided(5, 4)
    c = PC.strang(PC.extend_evenly(g))
    np.testing.assert_array_equal(c[:3, :3], g[:3, :3])
    np.testing.assert_array_equal(c[3:5, 0], g[[2, 1], 0])  # offsets -2 and -1 wrap to 3 and 4
    assert c[0, 3] == g[0, 1]  # along a count of 4, offset -1 wraps to 3


def test_r_chan_adds_the_reflection_in_every_direction():
    g = _one_sided(4, 3)
    c = PC.r_chan(PC.extend_evenly(g))
    assert c[0, 0] == g[0, 0]
    assert c[1, 0] == g[1, 0] + g[3, 0]
    assert c[0, 1] == g[0, 1] + g[0, 2]
    assert c[1, 1] == g[1, 1] + g[3, 1] + g[1, 2] + g[3, 2]


def test_huckle_with_unit_bandwidths_keeps_the_zero_offset():
    g = _one_sided(5, 4)
    want = np.zeros((5, 4))
    want[0, 0] = g[0, 0]
    np.testing.assert_array_equal(PC.huckle(PC.extend_evenly(g), 1, 1), want)


def test_huckle_damps_and_wraps():
    g = _one_sided(5, 4)
    c = PC.huckle(PC.extend_evenly(g), 2, 1)
    np.testing.assert_array_equal(c[[1, 4], 0], [0.5 * g[1, 0]] * 2)  # offset 1 damped by 1 - 1/2, at 1 and 4
    np.testing.assert_array_equal(c[[2, 3], 0], [0, 0])


def test_empty_generators_give_empty_circulants():
    assert PC.strang(None) is None
    assert PC.t_chan(None) is None
    assert PC.r_chan(None) is None
    assert PC.huckle(None, 2, 2) is None
    assert PC.superoptimal(None) is None
