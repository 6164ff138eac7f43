"""Excitations, results, byte models and the dense-matrix check (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+operator/generatePlaneWave.m:18-42
  src/+rooftopMoM/+operator/generateDeltaGap.m:13-14
  src/+rooftopMoM/+operator/+utils/generateMiddlePort.m:14-28
  src/+rooftopMoM/+operator/computeRadarCrossSection.m:18-19
  src/+rooftopMoM/+operator/computeInputImpedance.m:17
  src/+rooftopMoM/+resources/estimate{Generators,Product,Preconditioner,Solver}.m
  tests/+unit/Base.m:83-124 (the dense Green's matrix built from the generators)
"""
from __future__ import annotations

import math

import numpy as np

from .geometry import BOTH, Z0, Rooftops, fast_fft_size, quadrature_2d


def plane_wave(rt: Rooftops, k, direction, polarization, intensity=1.0):
    """generatePlaneWave.m:18-42: reference rooftop integral times separable phase."""
    direction = np.asarray(direction, dtype=np.float64)
    polarization = np.asarray(polarization, dtype=np.float64)
    area = rt.size_x * rt.size_y
    pu, pv, w = quadrature_2d(rt.order)
    steps = -1j * k * direction[:2] * np.array([rt.size_x, rt.size_y])
    point_phases = np.exp(steps[0] * pu + steps[1] * pv)
    parts = []
    for n, d in enumerate("xy"):
        roof = rt.reference_rooftop(d)
        rows, cols = rt.grid_size(d)
        sfo = np.array(roof["second_face_offset"], dtype=np.float64)
        second_phase = np.exp(steps @ sfo)
        amps = roof["amplitudes"][:, 0] + second_phase * roof["amplitudes"][:, 1]
        ref = intensity * polarization[n] * area * (point_phases @ (w * amps))
        trans = np.exp(steps[0] * np.arange(rows))[:, None] * np.exp(steps[1] * np.arange(cols))[None, :]
        parts.append(ref * trans.ravel(order="F"))
    return np.concatenate(parts)


def middle_port(rt: Rooftops, direction="x"):
    """generateMiddlePort.m:14-28 (0-based rooftop indices)."""
    rows, cols = rt.grid_size(direction)
    if direction == "x":
        r = np.full(cols, rt.count_x // 2 - 1)
        c = np.arange(cols)
        first = 0
    else:
        r = np.arange(rows)
        c = np.full(rows, rt.count_y // 2 - 1)
        first = rt.count_dir("x")
    return first + r + c * rows


def delta_gap(rt: Rooftops, port, voltage=1.0):
    """generateDeltaGap.m:13-14."""
    e = np.zeros(rt.count, dtype=np.float64)
    port = np.asarray(port)
    e[port] = voltage * rt.edge_lengths(port)
    return e


def radar_cross_section(k, excitation, current, intensity=1.0):
    """computeRadarCrossSection.m:18-19."""
    return (k * Z0) ** 2 * abs(np.asarray(excitation) @ np.asarray(current)) ** 2 / (4 * math.pi * intensity**4)


def input_impedance(rt: Rooftops, current, port, voltage=1.0):
    """computeInputImpedance.m:17."""
    port = np.asarray(port)
    return voltage / (rt.edge_lengths(port) @ np.asarray(current)[port])


# Byte models (resources/estimate*.m), used as the admission contract.
def estimate_generators(rt: Rooftops):
    return 16 * (rt.count + rt.count_x * rt.count_y)


def estimate_product(rt: Rooftops, product="splitFFT"):
    counts = (rt.count_x, rt.count_y)
    blocks = 1 + 3 * (rt.content == BOTH)
    if product == "fft":
        sizes = (max(2 * counts[0] - 2, 1), max(2 * counts[1] - 2, 1))
        subbands = 1
    else:
        sizes = tuple(fast_fft_size(c) if c > 1 else 1 for c in counts)
        subbands = 2 ** sum(c > 1 for c in counts)
    stored = 16 * blocks * subbands * sizes[0] * sizes[1]
    grid = 16 * sizes[0] * sizes[1]
    if product == "fft":
        working = 3 * grid + 16 * rt.count_dir("y") if rt.content == BOTH else 2.5 * grid
    elif product == "splitFFT":
        working = 8 * grid if rt.content == BOTH else 3 * grid
    else:
        if rt.content != BOTH:
            working = 3 * grid
        else:
            rows = (rt.grid_size("x")[0], rt.grid_size("y")[0])
            cols = (rt.grid_size("x")[1], rt.grid_size("y")[1])
            chunk = max(r * math.ceil(c / min(32, c)) for r, c in zip(rows, cols))
            working = 16 * (rt.count + sizes[0] * sizes[1] + 3 * chunk)
    return stored, working


def estimate_preconditioner(rt: Rooftops):
    blocks = 1 + 3 * (rt.content == BOTH)
    stored = 16 * blocks * rt.count_x * rt.count_y
    grid = 16 * rt.count_x * rt.count_y
    working = 3 * grid + 16 * rt.count_dir("y") if rt.content == BOTH else 2.5 * grid
    return stored, working


def estimate_solver(count, method, preconditioned, restart=50, maxit=1000):
    if method == "cg":
        vectors = 5 + int(preconditioned)
    else:
        basis = min(restart, count, maxit) + 1
        vectors = 1.5 * basis + 2 + int(preconditioned)
    return 16 * count * vectors


def dense_matrix(gen, rt: Rooftops):
    """tests/+unit/Base.m:83-124: blkdiag(XX, YY) - D^T E D from the generators by definition."""
    cx, cy = rt.count_x, rt.count_y
    fx, fy = np.meshgrid(np.arange(cx), np.arange(cy), indexing="ij")
    faces = np.stack([fx.ravel(order="F"), fy.ravel(order="F")])

    def toeplitz(g, offs):
        if offs.shape[1] == 0:
            return np.zeros((0, 0), dtype=np.complex128)
        dx = np.abs(offs[0][:, None] - offs[0][None, :])
        dy = np.abs(offs[1][:, None] - offs[1][None, :])
        return g[dx, dy]

    fmat = toeplitz(gen.electric, faces)
    blocks = []
    div = []
    sizes = (rt.size_x, rt.size_y)
    for n, d in enumerate("xy"):
        rows, cols = rt.grid_size(d)
        cnt = rows * cols
        ii = np.arange(cnt)
        first = np.stack([ii % rows, ii // rows]) if cnt else np.zeros((2, 0), dtype=int)
        second = first + np.array([[1], [0]]) if d == "x" else first + np.array([[0], [1]])
        g = gen.magnetic_xx if d == "x" else gen.magnetic_yy
        blocks.append(toeplitz(g, first) if cnt else np.zeros((0, 0)))
        D = np.zeros((cx * cy, cnt))
        if cnt:
            D[first[0] + first[1] * cx, ii] += 1.0 / sizes[n]
            D[second[0] + second[1] * cx, ii] -= 1.0 / sizes[n]
        div.append(D)
    Dm = np.hstack(div)
    n0 = blocks[0].shape[0]
    n1 = blocks[1].shape[0]
    M = np.zeros((n0 + n1, n0 + n1), dtype=np.complex128)
    if n0:
        M[:n0, :n0] = blocks[0]
    if n1:
        M[n0:, n0:] = blocks[1]
    return M - Dm.T @ fmat @ Dm
