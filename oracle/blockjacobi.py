"""Block-Jacobi preconditioner over blocks of bx x by faces (oracle; test infrastructure).

Not in the reference (its Preconditioner offers circulant kernels only). The blocks are the
diagonal blocks of the Green's matrix as the reference's dense oracle defines it
(tests/+unit/Base.m:83-113): for the rooftops p, q whose first faces lie in one block, the magnetic
generator of their direction at the offset of their first faces minus sum_{f, f'} div_p(f) E(f - f')
div_q(f'), with div = +1/h on the first face and -1/h on the second. Parity of the GPU build with
this restatement is the test; there is no reference number to pin it to.
"""
from __future__ import annotations

import numpy as np

from .geometry import Rooftops


def block_indices(rt: Rooftops, bx: int, by: int):
    """List of (indices, dirs, first_faces) per block, in the GPU's order (x blocks fastest)."""
    cx, cy = rt.count_x, rt.count_y
    nx = (cx - 1) * cy
    out = []
    for J in range((cy + by - 1) // by):
        for I in range((cx + bx - 1) // bx):
            idx, dirs, faces = [], [], []
            for d in range(2):
                for j in range(J * by, min((J + 1) * by, cy)):
                    for i in range(I * bx, min((I + 1) * bx, cx)):
                        if d == 0 and i > cx - 2:
                            continue
                        if d == 1 and j > cy - 2:
                            continue
                        idx.append(i + (cx - 1) * j if d == 0 else nx + i + cx * j)
                        dirs.append(d)
                        faces.append((i, j))
            out.append((np.array(idx), np.array(dirs), np.array(faces)))
    return out


def entry(gen, rt: Rooftops, dp, fp, dq, fq):
    """Green's-matrix entry between rooftops of directions dp, dq with first faces fp, fq."""
    z = 0j
    if dp == dq:
        dx, dy = abs(fp[0] - fq[0]), abs(fp[1] - fq[1])
        z = (gen.magnetic_xx if dp == 0 else gen.magnetic_yy)[dx, dy]
    hp = rt.size_x if dp == 0 else rt.size_y
    hq = rt.size_x if dq == 0 else rt.size_y
    for s in range(2):
        f = (fp[0] + (s and dp == 0), fp[1] + (s and dp == 1))
        for t in range(2):
            g = (fq[0] + (t and dq == 0), fq[1] + (t and dq == 1))
            w = (1.0 if s == t else -1.0) / (hp * hq)
            z -= w * gen.electric[abs(f[0] - g[0]), abs(f[1] - g[1])]
    return z


class BlockJacobi:
    """Block-Jacobi preconditioner: the inverses of the diagonal blocks, applied per block."""

    def __init__(self, gen, rt: Rooftops, bx=2, by=2):
        groups = {}
        for idx, dirs, faces in block_indices(rt, bx, by):
            if idx.size:  # a block at the edge of a strip can hold no rooftop
                groups.setdefault(idx.size, []).append((idx, dirs, faces))
        self.groups = {}
        for size, items in groups.items():
            idx = np.array([it[0] for it in items])          # [B, n]
            dirs = np.array([it[1] for it in items])         # [B, n]
            faces = np.array([it[2] for it in items])        # [B, n, 2]
            M = _entries(gen, rt, dirs, faces)               # [B, n, n]
            self.groups[size] = (idx, np.linalg.inv(M))

    def apply(self, x):
        x = np.asarray(x)
        y = np.empty_like(x, dtype=np.complex128)
        for idx, inv in self.groups.values():
            y[idx] = np.einsum("brc,bc->br", inv, x[idx])
        return y


def _entries(gen, rt: Rooftops, dirs, faces):
    """entry() for all pairs of all blocks at once: dirs [B, n], faces [B, n, 2] -> [B, n, n]."""
    dp, dq = dirs[:, :, None], dirs[:, None, :]
    fp, fq = faces[:, :, None, :], faces[:, None, :, :]
    dx = np.abs(fp[..., 0] - fq[..., 0])
    dy = np.abs(fp[..., 1] - fq[..., 1])
    z = np.zeros(dx.shape, dtype=np.complex128)
    if gen.magnetic_xx is not None:
        m = (dp == 0) & (dq == 0)
        z[m] = gen.magnetic_xx[dx[m], dy[m]]
    if gen.magnetic_yy is not None:
        m = (dp == 1) & (dq == 1)
        z[m] = gen.magnetic_yy[dx[m], dy[m]]
    hp = np.where(dp == 0, rt.size_x, rt.size_y)
    hq = np.where(dq == 0, rt.size_x, rt.size_y)
    for s in range(2):
        fi = fp[..., 0] + (s * (dp == 0))
        fj = fp[..., 1] + (s * (dp == 1))
        for t in range(2):
            gi = fq[..., 0] + (t * (dq == 0))
            gj = fq[..., 1] + (t * (dq == 1))
            w = (1.0 if s == t else -1.0) / (hp * hq)
            z -= w * gen.electric[np.abs(fi - gi), np.abs(fj - gj)]
    return z
