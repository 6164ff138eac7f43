"""Block spectra and the FFT / split-FFT / lean split-FFT products (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateSubbandSpectra.m:20-77
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateBlockSpectra.m:19-50
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateShiftPhases.m:16-17
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateSubbandModulation.m:12-15
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateEmbeddingSpectra.m:15-40
  src/+rooftopMoM/+assembler/+greensMatrix/FFTApplicator.m:14-88
  src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/applyBothDirections_.m:14-85
  src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/applySingleDirection_.m:14-26
  src/+rooftopMoM/+assembler/+greensMatrix/@LeanSplitFFTApplicator/applyBothDirections_.m:13-91
  src/+rooftopMoM/+assembler/+greensMatrix/@Spectra/{invert,determinant}.m

Grids are numpy arrays [x, y] (MATLAB's column-major rows and columns); rooftop vectors are the
column-major flattening (``order='F'``) of the x-directed grid followed by the y-directed one.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

from .geometry import BOTH, XONLY, YONLY, Rooftops, fast_fft_size

WORKERS = int(os.environ.get("RTM_ORACLE_WORKERS", os.cpu_count() or 1))


def fft(a, axis):
    return sfft.fft(a, axis=axis, workers=WORKERS)


def ifft(a, axis):
    return sfft.ifft(a, axis=axis, workers=WORKERS)


def fft2(a, s=None):
    return sfft.fft2(a, s=s, workers=WORKERS)


def ifft2(a):
    return sfft.ifft2(a, workers=WORKERS)


@dataclass
class Spectra:
    """Spectra.m: 2x2 block spectra; a missing direction's blocks are None."""

    xx: np.ndarray | None
    xy: np.ndarray | None
    yx: np.ndarray | None
    yy: np.ndarray | None

    def grid_size(self):
        for b in (self.xx, self.yy, self.xy, self.yx):
            if b is not None:
                return b.shape
        raise ValueError("empty spectra")

    def determinant(self, content):
        # determinant.m:10-16
        if content == XONLY:
            return self.xx
        if content == YONLY:
            return self.yy
        return self.xx * self.yy - self.xy * self.yx

    def invert(self, content):
        # invert.m:12-20
        with np.errstate(divide="ignore", invalid="ignore"):
            if content == XONLY:
                return Spectra(1.0 / self.xx, None, None, None)
            if content == YONLY:
                return Spectra(None, None, None, 1.0 / self.yy)
            d = self.determinant(content)
            return Spectra(self.yy / d, -self.xy / d, -self.yx / d, self.xx / d)


def shift_phases(size_x, size_y, parity_x, parity_y):
    """generateShiftPhases.m:16-17: exp(i pi (2m + parity)/size), column in x, row in y."""
    sx = np.exp(1j * np.pi * (2 * np.arange(size_x) + parity_x) / size_x)[:, None]
    sy = np.exp(1j * np.pi * (2 * np.arange(size_y) + parity_y) / size_y)[None, :]
    return sx, sy


def modulation(n):
    """generateSubbandModulation.m:15: exp(-i pi d / n), d = 0..n-1."""
    return np.exp(-1j * np.pi * np.arange(n) / n)


def block_spectra(mxx, myy, e, content, a, b, sx, sy):
    """generateBlockSpectra.m:19-50."""
    mxx = 0 if mxx is None else mxx
    myy = 0 if myy is None else myy
    has_x = content != YONLY
    has_y = content != XONLY
    xx = xy = yx = yy = None
    if has_x:
        xx = mxx - (np.abs(1 - sx) / a) ** 2 * e
    if has_y:
        yy = myy - (np.abs(1 - sy) / b) ** 2 * e
    if has_x and has_y:
        xy = ((1 - sx) / (a * b)) * (np.conj(sy) - 1) * e
        yx = ((np.conj(sx) - 1) / (a * b)) * (1 - sy) * e
    return Spectra(xx, xy, yx, yy)


def subband_spectra(gen, a, b):
    """generateSubbandSpectra.m:20-77 -> list of Spectra, index parityX + 2 parityY (or 2 for strips)."""
    cx, cy = gen.electric.shape
    P = fast_fft_size(cx) if cx > 1 else 1
    Q = fast_fft_size(cy) if cy > 1 else 1
    step_x = 2 if P > 1 else 1
    step_y = 2 if Q > 1 else 1
    nsub = step_x * step_y
    pars = [(px, py) for py in range(step_y) for px in range(step_x)]  # ndgrid order: px fastest
    kernels = [gen.magnetic_xx, gen.magnetic_yy, gen.electric]
    sub = [[None] * nsub for _ in range(3)]
    for n, g in enumerate(kernels):
        if g is None:
            continue
        rows, cols = g.shape
        emb = np.zeros((step_x * P, step_y * Q), dtype=np.complex128)
        emb[:rows, :cols] = g / nsub
        if rows > 1:
            emb[emb.shape[0] - rows + 1:, :cols] = emb[rows - 1:0:-1, :cols]
        if cols > 1:
            emb[:, emb.shape[1] - cols + 1:] = emb[:, cols - 1:0:-1]
        emb = fft2(emb)
        if np.isrealobj(g):
            emb = emb.real
        for kk, (px, py) in enumerate(pars):
            sub[n][kk] = emb[px::step_x, py::step_y]
    out = []
    for kk, (px, py) in enumerate(pars):
        sx, sy = shift_phases(P, Q, px, py)
        out.append(block_spectra(sub[0][kk], sub[1][kk], sub[2][kk], gen.content, a, b, sx, sy))
    return out


def _pad(g, cx, cy):
    if g is None:
        return None
    out = np.zeros((cx, cy), dtype=g.dtype)
    r = min(g.shape[0], cx)
    c = min(g.shape[1], cy)
    out[:r, :c] = g[:r, :c]
    return out


def embedding_spectra(gen, a, b):
    """generateEmbeddingSpectra.m:15-31: mirror to period 2n-2, fft2, blocks."""
    cx, cy = gen.electric.shape
    mx = np.r_[np.arange(cx), np.arange(cx - 2, 0, -1)]
    my = np.r_[np.arange(cy), np.arange(cy - 2, 0, -1)]

    def embed(g):
        if g is None:
            return None
        return fft2(_pad(g, cx, cy)[np.ix_(mx, my)])

    sx, sy = shift_phases(len(mx), len(my), 0, 0)
    return block_spectra(embed(gen.magnetic_xx), embed(gen.magnetic_yy), embed(gen.electric), gen.content,
                         a, b, sx, sy)


def _split_input(rt: Rooftops, x):
    rx, cx = rt.grid_size("x")
    ry, cy = rt.grid_size("y")
    nx = rx * cx
    return (x[:nx].reshape(rx, cx, order="F"), x[nx:].reshape(ry, cy, order="F"))


def fft_apply(rt: Rooftops, spec: Spectra, content, x):
    """FFTApplicator.apply (FFTApplicator.m:14-88)."""
    x = np.asarray(x, dtype=np.complex128)
    if content in (XONLY, YONLY):
        d = "x" if content == XONLY else "y"
        blk = spec.xx if content == XONLY else spec.yy
        r, c = rt.grid_size(d)
        out = ifft2(blk * fft2(x.reshape(r, c, order="F"), s=blk.shape))
        return out[:r, :c].ravel(order="F")
    ix, iy = _split_input(rt, x)
    s = spec.grid_size()
    fx = fft2(ix, s=s)
    ox = spec.xx * fx
    oy = spec.yx * fx
    fy = fft2(iy, s=s)
    ox = ox + spec.xy * fy
    oy = oy + spec.yy * fy
    ox = ifft2(ox)[: ix.shape[0], : ix.shape[1]]
    oy = ifft2(oy)[: iy.shape[0], : iy.shape[1]]
    return np.concatenate([ox.ravel(order="F"), oy.ravel(order="F")])


def split_apply(rt: Rooftops, spectra, content, x):
    """SplitFFTApplicator.apply (apply.m:10-20, applyBothDirections_.m:14-85, applySingleDirection_.m)."""
    x = np.asarray(x, dtype=np.complex128)
    P, Q = spectra[0].grid_size()
    if content in (XONLY, YONLY):
        even = spectra[0].xx if content == XONLY else spectra[0].yy
        odd = spectra[1].xx if content == XONLY else spectra[1].yy
        n = even.size
        mod = modulation(n)
        v = np.zeros(n, dtype=np.complex128)
        v[: x.size] = x
        e1 = even.ravel()
        o1 = odd.ravel()
        out = np.fft.ifft(e1 * np.fft.fft(v))
        out = out + np.fft.ifft(o1 * np.fft.fft(v * mod)) * np.conj(mod)
        return out[: x.size]
    ix, iy = _split_input(rt, x)
    gx = np.zeros((P, Q), dtype=np.complex128)
    gy = np.zeros((P, Q), dtype=np.complex128)
    gx[: ix.shape[0], : ix.shape[1]] = ix
    gy[: iy.shape[0], : iy.shape[1]] = iy
    modx = modulation(P)[:, None]
    mody = modulation(Q)[None, :]
    outx = outy = None
    for py in range(2):
        ax = gx * mody if py else gx
        ay = gy * mody if py else gy
        sxp = fft(ax, 1)
        syp = fft(ay, 1)
        acc_x = acc_y = None
        for px in range(2):
            if px:
                sxp = sxp * modx
                syp = syp * modx
            ux = fft(sxp, 0)
            uy = fft(syp, 0)
            blk = spectra[px + 2 * py]
            ox = ifft(blk.xx * ux + blk.xy * uy, 0)
            oy = ifft(blk.yx * ux + blk.yy * uy, 0)
            if px:
                acc_x = acc_x + ox * np.conj(modx)
                acc_y = acc_y + oy * np.conj(modx)
            else:
                acc_x, acc_y = ox, oy
        acc_x = ifft(acc_x, 1)
        acc_y = ifft(acc_y, 1)
        if py:
            outx = outx + acc_x * np.conj(mody)
            outy = outy + acc_y * np.conj(mody)
        else:
            outx, outy = acc_x, acc_y
    ox = outx[: ix.shape[0], : ix.shape[1]]
    oy = outy[: iy.shape[0], : iy.shape[1]]
    return np.concatenate([ox.ravel(order="F"), oy.ravel(order="F")])


def lean_apply(rt: Rooftops, spectra, content, x):
    """LeanSplitFFTApplicator.applyBothDirections_ (applyBothDirections_.m:13-91): one contribution
    (subband, input component, output component) at a time in one grid buffer; strips as split."""
    if content != BOTH:
        return split_apply(rt, spectra, content, x)
    x = np.asarray(x, dtype=np.complex128)
    P, Q = spectra[0].grid_size()
    comps = _split_input(rt, x)
    modx = modulation(P)[:, None]
    mody = modulation(Q)[None, :]
    names = (("xx", "xy"), ("yx", "yy"))
    outs = [np.zeros(c.shape, dtype=np.complex128) for c in comps]
    for k in range(4):
        odd_x = k % 2 == 1
        odd_y = k >= 2
        blk = spectra[k]
        for ic in range(2):
            for oc in range(2):
                buf = np.zeros((P, Q), dtype=np.complex128)
                part = comps[ic]
                if odd_x:
                    part = part * modx[: part.shape[0]]
                if odd_y:
                    part = part * mody[:, : part.shape[1]]
                buf[: part.shape[0], : part.shape[1]] = part
                buf = fft(fft(buf, 1), 0)
                buf = getattr(blk, names[oc][ic]) * buf
                buf = ifft(ifft(buf, 0), 1)
                r, c = outs[oc].shape
                part = buf[:r, :c]
                if odd_x:
                    part = part * np.conj(modx[:r])
                if odd_y:
                    part = part * np.conj(mody[:, :c])
                outs[oc] += part
    return np.concatenate([outs[0].ravel(order="F"), outs[1].ravel(order="F")])
