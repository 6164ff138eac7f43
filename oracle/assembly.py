"""Green's-matrix generator assembly (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/generate.m:10-59
  src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/private/countNearOffsets_.m:1-11
  src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/private/integrateCellPairs_.m:1-44
  src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/private/integrateLattice_.m:1-127
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateReducedRule.m:21-66
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/integrateMoments.m:17-39
  src/+rooftopMoM/+assembler/+greensMatrix/+utils/accumulateMoments.m:27-133

Generators are numpy arrays indexed [dX, dY] (the MATLAB column-major grids).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .geometry import Z0, gauss_legendre
from .singular import extracted_moments, remainder

NEAR_GAP = 3  # MomentAssembler.m:13


@dataclass
class Generators:
    """Generators.m:1-59. A missing rooftop direction has ``None``."""

    magnetic_xx: np.ndarray | None
    magnetic_yy: np.ndarray | None
    electric: np.ndarray
    content: int

    def modify(self, fn):
        f = (lambda g: None if g is None else fn(g))
        return Generators(f(self.magnetic_xx), f(self.magnetic_yy), fn(self.electric), self.content)


def _round_half_away(x):
    return np.floor(np.asarray(x, dtype=np.float64) + 0.5).astype(int)


def _axis(order: int, parts: int):
    """generateReducedRule.m:36-66: nodes on [-1, 1] and the 4 weight columns W00, W10, W01, W11."""
    points, pw = gauss_legendre(order, 0.0, 1.0)
    right = np.concatenate([(points + p) / parts for p in range(parts)])
    nodes = np.concatenate([right - 1.0, right])
    pw = np.tile(pw / parts, 2 * parts)
    left = nodes < 0
    w10 = (1 - nodes**2) / 2
    w10[left] = (1 + nodes[left]) ** 2 / 2
    w01 = (1 - nodes) ** 2 / 2
    w01[left] = (1 - nodes[left] ** 2) / 2
    d = np.abs(nodes)
    weights = pw[:, None] * np.stack([1 - d, w10, w01, (1 - d) ** 2 * (2 + d) / 6], axis=1)
    return nodes, weights


def reduced_rule(order: int, part_counts):
    """generateReducedRule.m:21-34.

    Returns (nodes_x (Px), nodes_y (Py), weights (7 x Px*Py) with nu running fastest).
    """
    nx, wx = _axis(order, int(part_counts[0]))
    ny, wy = _axis(order, int(part_counts[1]))
    # kron(wy[:,0], wx): row iy*Px + ix; columns M00, M10, M01, M11
    m_part = (wy[:, 0][:, None, None] * wx[None, :, :]).reshape(-1, 4)
    # kron(wy[:,1:4], wx[:,0]): columns N10, N01, N11
    n_part = (wy[:, 1:4][:, None, :] * wx[:, 0][None, :, None]).reshape(-1, 3)
    weights = np.concatenate([m_part, n_part], axis=1).T.copy()
    return nx, ny, weights


def count_near_offsets(counts, sizes, gap=NEAR_GAP):
    """countNearOffsets_.m:1-11."""
    out = []
    for n in range(2):
        gaps = np.maximum(np.arange(counts[n]) - 1, 0) * sizes[n]
        out.append(int(np.count_nonzero(gaps < gap * max(sizes))))
    return out


def integrate_moments(rule, offsets, sizes, k):
    """7 x C moments over the cell pairs at the offsets (integrateMoments.m:17-39).

    ``offsets`` is 2 x C. Touching offsets integrate the remainder of the extraction.
    """
    nx, ny, weights = rule
    offsets = np.asarray(offsets)
    dx = sizes[0] * (nx[None, :, None] - offsets[0][None, None, :])  # [1, Px, C]
    dy = sizes[1] * (ny[:, None, None] - offsets[1][None, None, :])  # [Py, 1, C]
    dist = np.hypot(dx, dy)  # [Py, Px, C], nu fastest after reshape
    kern = np.exp(-1j * k * dist) / dist
    touching = np.all(offsets <= 1, axis=0)
    if np.any(touching):
        kern[:, :, touching] = remainder(dist[:, :, touching], k)
    return weights @ kern.reshape(-1, offsets.shape[1])


# accumulateMoments.m:43-49: rows E; XX at e, e-u, e+u; YY at e, e-u, e+u.
_COMBINE = np.array([
    [1, 0, 0, 0, 0, 0, 0],
    [1, -1, -1, 2, 0, 0, 0],
    [0, 1, 0, -1, 0, 0, 0],
    [0, 0, 1, -1, 0, 0, 0],
    [1, 0, 0, 0, -1, -1, 2],
    [0, 0, 0, 0, 1, 0, -1],
    [0, 0, 0, 0, 0, 1, -1],
], dtype=np.float64)


def accumulate_moments(parts: Generators, moments, offsets, scales):
    """Add the moments of distinct cell-pair offsets to the generators (accumulateMoments.m:27-133).

    Each offset e adds scales[0]*M00 to electric[e]; to magneticXX the rising-rising term at e, the
    rising-falling term at e - u_x (doubled at dX = 1, the reflection of the pair at -u_x) and the
    falling-rising term at e + u_x; likewise for magneticYY along y.
    """
    offsets = np.asarray(offsets)
    if offsets.size == 0:
        return parts
    scale = np.array([scales[0]] + [scales[1]] * 6)[:, None]
    terms = (scale * _COMBINE) @ moments
    cx, cy = parts.electric.shape
    dX = offsets[0].astype(int)
    dY = offsets[1].astype(int)
    np.add.at(parts.electric, (dX, dY), terms[0])
    if parts.magnetic_xx is not None:
        xx = parts.magnetic_xx
        m = dX <= cx - 2
        np.add.at(xx, (dX[m], dY[m]), terms[1][m])
        m = dX >= 1
        rising = np.where(dX == 1, 2.0, 1.0) * terms[2]
        np.add.at(xx, (dX[m] - 1, dY[m]), rising[m])
        m = dX <= cx - 3
        np.add.at(xx, (dX[m] + 1, dY[m]), terms[3][m])
    if parts.magnetic_yy is not None:
        yy = parts.magnetic_yy
        m = dY <= cy - 2
        np.add.at(yy, (dX[m], dY[m]), terms[4][m])
        m = dY >= 1
        rising = np.where(dY == 1, 2.0, 1.0) * terms[5]
        np.add.at(yy, (dX[m], dY[m] - 1), rising[m])
        m = dY <= cy - 3
        np.add.at(yy, (dX[m], dY[m] + 1), terms[6][m])
    return parts


def _lattice_quadrants(rule, order):
    """splitQuadrants_ (integrateLattice_.m:92-111): 4 x (7 x order^2 weights, shift)."""
    w = rule[2].reshape(7, 2 * order, 2 * order, order="F")  # w[:, kx, ky]
    quads = []
    for hy in range(2):
        for hx in range(2):
            q = w[:, hx * order:(hx + 1) * order, hy * order:(hy + 1) * order]
            quads.append((q.reshape(7, -1, order="F"), (int(hx == 0), int(hy == 0))))
    return quads


def integrate_lattice(parts, counts, sizes, k, rule, order, excluded, scales, column_tile=None):
    """Far pass on the shared lattice of blocks (integrateLattice_.m:17-90).

    The kernel is evaluated once on the order x order points of every block (m, n), m = 0..countX,
    n = 0..countY, x = a (p - m), y = b (p - n); the moments of the offset (dX, dY) are the sums over
    its four quadrants, each the quadrant weights times the block (dX + sx, dY + sy).
    """
    points = rule[0][order:2 * order]
    quads = _lattice_quadrants(rule, order)
    cx, cy = counts
    if column_tile is None:
        column_tile = max(1, min(cy, (1 << 26) // max(1, 16 * order * order * (cx + 1))))
    bx = np.arange(cx + 1)
    xs = sizes[0] * (points[:, None] - bx[None, :])  # [px, m]
    for c0 in range(0, cy, column_tile):
        c1 = min(cy, c0 + column_tile)
        by = np.arange(c0, c1 + 1)
        ys = sizes[1] * (points[:, None] - by[None, :])  # [py, n]
        dist = np.hypot(xs[None, :, :, None], ys[:, None, None, :])  # [py, px, m, n]
        kern = np.exp(-1j * k * dist) / dist
        del dist
        kf = kern.reshape(order * order, -1)  # row py*order + px (px fastest)
        mom = np.zeros((7, cx, c1 - c0), dtype=np.complex128)
        for wq, (sx, sy) in quads:
            sums = (wq @ kf).reshape(7, cx + 1, c1 - c0 + 1)
            mom += sums[:, sx:sx + cx, sy:sy + (c1 - c0)]
        del kern, kf
        dX, dY = np.meshgrid(np.arange(cx), np.arange(c0, c1), indexing="ij")
        keep = (dX >= excluded[0]) | (dY >= excluded[1])
        offs = np.stack([dX[keep], dY[keep]])
        accumulate_moments(parts, mom[:, keep], offs, scales)
    return parts



def allocate_parts(counts, content_counts):
    """allocateParts_.m:1-16."""
    cx, cy = counts
    e = np.zeros((cx, cy), dtype=np.complex128)
    xx = np.zeros((cx - 1, cy), dtype=np.complex128) if content_counts[0] > 0 else None
    yy = np.zeros((cx, cy - 1), dtype=np.complex128) if content_counts[1] > 0 else None
    return e, xx, yy


def scales_of(size_x, size_y, k):
    """generate.m:20: i Z0/(4 pi) (ab)^2 [1/k, k]."""
    s = 1j * Z0 / (4 * math.pi) * (size_x * size_y) ** 2
    return (s / k, s * k)


def generate(count_x, count_y, size_x, size_y, k, orders=(16, 8)):
    """MomentAssembler.generate (generate.m:10-59): near pass, far lattice, extracted touching moments."""
    counts = (int(count_x), int(count_y))
    sizes = (float(size_x), float(size_y))
    nx_roof = (counts[0] - 1) * counts[1]
    ny_roof = counts[0] * (counts[1] - 1)
    from .geometry import BOTH, XONLY, YONLY, NONE
    content = BOTH if (nx_roof > 0 and ny_roof > 0) else XONLY if nx_roof > 0 else YONLY if ny_roof > 0 else NONE
    e, xx, yy = allocate_parts(counts, (nx_roof, ny_roof))
    parts = Generators(xx, yy, e, content)
    scales = scales_of(sizes[0], sizes[1], k)
    near = count_near_offsets(counts, sizes)
    near_rule = reduced_rule(orders[0], _round_half_away(np.array(sizes) / min(sizes)))
    far_rule = reduced_rule(orders[1], (1, 1))
    # Near pass: every offset 0..near-1 (integrateCellPairs_.m with excluded [0, 0]).
    dX, dY = np.meshgrid(np.arange(near[0]), np.arange(near[1]), indexing="ij")
    offs = np.stack([dX.ravel(order="F"), dY.ravel(order="F")])
    accumulate_moments(parts, integrate_moments(near_rule, offs, sizes, k), offs, scales)
    # Far pass on the lattice (generate.m:42).
    integrate_lattice(parts, counts, sizes, k, far_rule, orders[1], near, scales)
    # Touching pairs: extracted part in closed form (generate.m:45-52).
    touching = np.array([[0, 1, 0, 1], [0, 0, 1, 1]])
    inside = np.all(touching < np.array(counts)[:, None], axis=0)
    ext = extracted_moments(sizes[0], sizes[1], k)
    accumulate_moments(parts, ext[:, inside], touching[:, inside], scales)
    return parts
