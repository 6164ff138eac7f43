"""Circulant preconditioners (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+assembler/+preconditioner/generateCirculant.m:16-25
  src/+rooftopMoM/+assembler/+preconditioner/generatePartwiseSpectra.m:16-30
  src/+rooftopMoM/+assembler/+preconditioner/generateBlockwiseSpectra.m:17-33
  src/+rooftopMoM/+assembler/+preconditioner/generateHybridSpectra.m:16-26
  src/+rooftopMoM/+assembler/+preconditioner/+utils/{foldGenerator,extendEvenly,generateSpatialBlocks,
      generatePartSpectra,generateOptimalOfProduct}.m
  src/+rooftopMoM/+assembler/+preconditioner/+kernels/generate{Strang,TChan,RChan,Huckle,Superoptimal}.m
"""
from __future__ import annotations

import numpy as np

from .geometry import XONLY, YONLY
from .spectra import Spectra, block_spectra, fft, fft2, ifft, ifft2, shift_phases, _pad


def extend_evenly(g):
    """extendEvenly.m:12-13."""
    if g is None:
        return None
    cx, cy = g.shape
    ix = np.r_[np.arange(cx - 1, 0, -1), np.arange(cx)]
    iy = np.r_[np.arange(cy - 1, 0, -1), np.arange(cy)]
    return g[np.ix_(ix, iy)]


def _fold_rows(g):
    count = (g.shape[0] + 1) // 2
    out = g[count - 1:, :].copy()
    out[1:, :] += g[: count - 1, :]
    return out


def fold_generator(g, window, even=False):
    """foldGenerator.m:27-61."""
    if even:
        cx, cy = g.shape
    else:
        cx = (g.shape[0] + 1) // 2
        cy = (g.shape[1] + 1) // 2
    wx = np.asarray(window(np.arange(-(cx - 1), cx), cx, 1), dtype=np.float64).reshape(-1, 1)
    wy = np.asarray(window(np.arange(-(cy - 1), cy), cy, 2), dtype=np.float64).reshape(1, -1)
    if even:
        px = np.r_[0.0, wx[: cx - 1, 0]][:, None]
        py = np.r_[0.0, wy[0, : cy - 1]][None, :]
        rx = np.r_[0, np.arange(cx - 1, 0, -1)]
        ry = np.r_[0, np.arange(cy - 1, 0, -1)]
        c = wx[cx - 1:] * g + px * g[rx, :]
        c = c * wy[:, cy - 1:] + c[:, ry] * py
        return c
    w = wx * g * wy
    c = _fold_rows(w)
    return _fold_rows(c.T).T


def strang(g):
    if g is None:
        return None
    return fold_generator(g, lambda o, n, d: (np.abs(o) < n / 2).astype(float) + 0.5 * (np.abs(o) == n / 2))


def t_chan(g, even=False):
    if g is None:
        return None
    return fold_generator(g, lambda o, n, d: (n - np.abs(o)) / n, even)


def r_chan(g, even=False):
    if g is None:
        return None
    return fold_generator(g, lambda o, n, d: np.ones(np.shape(o)), even)


def huckle(g, bw_x, bw_y):
    if g is None:
        return None
    bws = (bw_x, bw_y)
    return fold_generator(g, lambda o, n, d: np.maximum(0.0, 1 - np.abs(o) / bws[d - 1]))


def _split_rows(g):
    count = (g.shape[0] + 1) // 2
    pos = g[count - 1:, :]
    neg = np.vstack([np.zeros((1, g.shape[1]), dtype=g.dtype), g[: count - 1, :]])
    return ((pos + neg) / 2, (pos - neg) / 2)


def part_spectra(g):
    """generatePartSpectra.m:15-49."""
    cx = (g.shape[0] + 1) // 2
    cy = (g.shape[1] + 1) // 2
    mx = np.exp(1j * np.pi * np.arange(cx) / cx)[:, None]
    my = np.exp(1j * np.pi * np.arange(cy) / cy)[None, :]
    parts_x = _split_rows(g)
    out = [[None, None], [None, None]]
    for m in range(2):
        parts_y = _split_rows(parts_x[m].T)
        for n in range(2):
            part = parts_y[n].T
            if m == 1:
                part = mx * part
            if n == 1:
                part = part * my
            out[m][n] = fft2(part)
    return out


def _kernel_spec(count):
    d = np.arange(count, dtype=np.float64)
    return np.fft.fft(1.0 / (count**2 * np.sin(np.pi * (2 * d + 1) / (2 * count)) ** 2))


def _convolve(values, kern, dim):
    if dim == 0:
        return ifft(kern[:, None] * fft(values, 0), 0)
    return ifft(kern[None, :] * fft(values, 1), 1)


def optimal_of_product(pa, pb):
    """generateOptimalOfProduct.m:18-62."""
    cx, cy = pa[0][0].shape
    kerns = (_kernel_spec(cx), _kernel_spec(cy))
    types = ((0, 0), (1, 0), (0, 1), (1, 1))
    eig = np.zeros((cx, cy), dtype=np.complex128)
    for ta in types:
        for tb in types:
            va = pa[ta[0]][ta[1]]
            vb = pb[tb[0]][tb[1]]
            for d in range(2):
                if ta[d] == 1 and tb[d] == 0:
                    va = _convolve(va, kerns[d], d)
            for d in range(2):
                if ta[d] == 0 and tb[d] == 1:
                    vb = _convolve(vb, kerns[d], d)
            prod = va * np.conj(vb)
            for d in range(2):
                if ta[d] == 1 and tb[d] == 1:
                    prod = _convolve(prod, kerns[d], d)
            eig = eig + prod
    return eig


def superoptimal(g):
    """generateSuperoptimal.m:14-25."""
    if g is None:
        return None
    parts = part_spectra(g)
    sq = optimal_of_product(parts, parts)
    opt = fft2(t_chan(g))
    return ifft2(sq / np.conj(opt))


def spatial_blocks(gen, a, b):
    """generateSpatialBlocks.m:19-61."""
    e = gen.electric
    cx, cy = e.shape
    has_x = gen.content != YONLY
    has_y = gen.content != XONLY
    bxx = bxy = byx = byy = None
    bordered = np.zeros((2 * cx + 1, 2 * cy + 1), dtype=e.dtype)
    bordered[1:-1, 1:-1] = extend_evenly(e)

    def sh(da, db):
        return bordered[1 + da: 2 * cx + da, 1 + db: 2 * cy + db]

    p = np.arange(-(cx - 1), cx)[:, None]
    q = np.arange(-(cy - 1), cy)[None, :]
    if has_x:
        bxx = extend_evenly(_pad(gen.magnetic_xx, cx, cy)) - (2 * sh(0, 0) - sh(-1, 0) - sh(1, 0)) / a**2
        bxx[np.abs(p[:, 0]) > cx - 2, :] = 0
    if has_y:
        byy = extend_evenly(_pad(gen.magnetic_yy, cx, cy)) - (2 * sh(0, 0) - sh(0, -1) - sh(0, 1)) / b**2
        byy[:, np.abs(q[0]) > cy - 2] = 0
    if has_x and has_y:
        bxy = -(sh(0, 0) - sh(0, -1) - sh(1, 0) + sh(1, -1)) / (a * b)
        bxy[p[:, 0] > cx - 2, :] = 0
        bxy[:, q[0] < -(cy - 2)] = 0
        byx = np.rot90(bxy, 2)
    return bxx, bxy, byx, byy


KERNELS = ("strang", "tChan", "rChan", "huckle", "superoptimal")
BUILDERS = ("partwise", "blockwise", "hybrid")


def _kernel_fn(kernel, bandwidth):
    if kernel == "strang":
        return strang, False
    if kernel == "tChan":
        return t_chan, True
    if kernel == "rChan":
        return r_chan, True
    if kernel == "huckle":
        return (lambda g: huckle(g, bandwidth[0], bandwidth[1])), False
    if kernel == "superoptimal":
        return superoptimal, False
    raise ValueError(kernel)


def circulant_spectra(gen, a, b, kernel="rChan", builder="partwise", bandwidth=None):
    """Uninverted block spectra of the circulant approximation on the face grid."""
    cx, cy = gen.electric.shape
    if bandwidth is None:
        bandwidth = (cx, cy)
    fn, takes_even = _kernel_fn(kernel, bandwidth)
    if builder == "partwise":
        # generatePartwiseSpectra.m:16-30
        if takes_even:
            approx = lambda g: None if g is None else fft2(fn(_pad(g, cx, cy), True))
        else:
            approx = lambda g: None if g is None else fft2(fn(extend_evenly(_pad(g, cx, cy))))
        sx, sy = shift_phases(cx, cy, 0, 0)
        return block_spectra(approx(gen.magnetic_xx), approx(gen.magnetic_yy), approx(gen.electric),
                             gen.content, a, b, sx, sy)
    bxx, bxy, _, byy = spatial_blocks(gen, a, b)
    f2 = lambda g: None if g is None else fft2(fn(g))
    if builder == "blockwise":
        # generateBlockwiseSpectra.m:17-33
        coupling = f2(bxy)
        transposed = None
        if coupling is not None:
            ix = np.r_[0, np.arange(coupling.shape[0] - 1, 0, -1)]
            iy = np.r_[0, np.arange(coupling.shape[1] - 1, 0, -1)]
            transposed = coupling[np.ix_(ix, iy)]
        return Spectra(f2(bxx), coupling, transposed, f2(byy))
    if builder == "hybrid":
        # generateHybridSpectra.m:16-26
        sx, sy = shift_phases(cx, cy, 0, 0)
        electric = fft2(fn(extend_evenly(gen.electric)))
        coupling = block_spectra(None, None, electric, gen.content, a, b, sx, sy)
        return Spectra(f2(bxx), coupling.xy, coupling.yx, f2(byy))
    raise ValueError(builder)


def circulant(gen, a, b, kernel="rChan", builder="partwise", bandwidth=None):
    """generateCirculant.m:16-25: inverted spectra for an FFTApplicator on the face grid."""
    return circulant_spectra(gen, a, b, kernel, builder, bandwidth).invert(gen.content)
