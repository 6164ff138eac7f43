"""Closed-form moments of R^-1, R, R^3 over the touching cell pairs (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+assembler/+singularIntegrals/+utils/integrateMonomial.m:18-81
  src/+rooftopMoM/+assembler/+singularIntegrals/generatePowerMoments.m:17-155
  src/+rooftopMoM/+assembler/+singularIntegrals/generateExtractedMoments.m:16-18
  src/+rooftopMoM/+assembler/+singularIntegrals/evaluateRemainder.m:13-14

The mixed antiderivatives G(a, b) of u^m v^n (u^2 + v^2)^(p/2) are closed forms of the calculus;
they are the same formulas as the reference's table because they are the same integrals.
"""
from __future__ import annotations

import numpy as np

from .geometry import gauss_legendre


def integrate_monomial(power: int, m: int, n: int, a, b):
    """Integral of u^m v^n R^power over [0, a] x [0, b] (integrateMonomial.m:18-81)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        R = np.sqrt(a * a + b * b)
        lb = np.arcsinh(b / a)
        la = np.arcsinh(a / b)
        key = (power, m, n)
        if key == (-1, 0, 0):
            v = a * lb + b * la
        elif key == (-1, 0, 1):
            v = (-a**2 + a * R + b**2 * la) / 2
        elif key == (-1, 1, 0):
            v = (-b**2 + b * R + a**2 * lb) / 2
        elif key == (-1, 1, 1):
            v = (-a**3 - b**3 + (a**2 + b**2) * R) / 3
        elif key == (-1, 2, 0):
            v = (a * b * R + 2 * a**3 * lb - b**3 * la) / 6
        elif key == (-1, 2, 1):
            v = (-2 * a**4 + a * (2 * a**2 + b**2) * R - b**4 * la) / 8
        elif key == (-1, 3, 0):
            v = (2 * b**4 + b * (a**2 - 2 * b**2) * R + 3 * a**4 * lb) / 12
        elif key == (-1, 3, 1):
            v = (-3 * a**5 + 2 * b**5 + (3 * a**4 + a**2 * b**2 - 2 * b**4) * R) / 15
        elif key == (1, 0, 0):
            v = (2 * a * b * R + a**3 * lb + b**3 * la) / 6
        elif key == (1, 0, 1):
            v = (-2 * a**4 + a * (2 * a**2 + 5 * b**2) * R + 3 * b**4 * la) / 24
        elif key == (1, 1, 0):
            v = (-2 * b**4 + b * (5 * a**2 + 2 * b**2) * R + 3 * a**4 * lb) / 24
        elif key == (1, 1, 1):
            v = (-a**5 - b**5 + (a**4 + 2 * a**2 * b**2 + b**4) * R) / 15
        elif key == (1, 2, 0):
            v = (a * b * (6 * a**2 + b**2) * R + 4 * a**5 * lb - b**5 * la) / 40
        elif key == (1, 2, 1):
            v = (-8 * a**6 + a * (8 * a**4 + 14 * a**2 * b**2 + 3 * b**4) * R - 3 * b**6 * la) / 144
        elif key == (1, 3, 0):
            v = (4 * b**6 + b * (21 * a**4 + 2 * a**2 * b**2 - 4 * b**4) * R + 15 * a**6 * lb) / 180
        elif key == (1, 3, 1):
            v = (-5 * a**7 + 2 * b**7 + (5 * a**6 + 8 * a**4 * b**2 + a**2 * b**4 - 2 * b**6) * R) / 105
        elif key == (3, 0, 0):
            v = (7 * a * b * (a**2 + b**2) * R + 3 * a**5 * lb + 3 * b**5 * la) / 40
        elif key == (3, 0, 1):
            v = (-8 * a**6 + a * (8 * a**4 + 26 * a**2 * b**2 + 33 * b**4) * R + 15 * b**6 * la) / 240
        elif key == (3, 1, 0):
            v = (-8 * b**6 + b * (33 * a**4 + 26 * a**2 * b**2 + 8 * b**4) * R + 15 * a**6 * lb) / 240
        elif key == (3, 1, 1):
            v = (-a**7 - b**7 + (a**6 + 3 * a**4 * b**2 + 3 * a**2 * b**4 + b**6) * R) / 35
        elif key == (3, 2, 0):
            v = (a * b * (38 * a**4 + 26 * a**2 * b**2 + 3 * b**4) * R + 18 * a**7 * lb
                 - 3 * b**7 * la) / 336
        elif key == (3, 2, 1):
            v = (-48 * a**8 + a * (48 * a**6 + 136 * a**4 * b**2 + 118 * a**2 * b**4 + 15 * b**6) * R
                 - 15 * b**8 * la) / 1920
        elif key == (3, 3, 0):
            v = (16 * b**8 + b * (215 * a**6 + 134 * a**4 * b**2 + 8 * a**2 * b**4 - 16 * b**6) * R
                 + 105 * a**8 * lb) / 2240
        elif key == (3, 3, 1):
            v = (-7 * a**9 + 2 * b**9
                 + (7 * a**8 + 19 * a**6 * b**2 + 15 * a**4 * b**4 + a**2 * b**6 - 2 * b**8) * R) / 315
        else:
            raise ValueError(f"no closed form for power={power}, m={m}, n={n}")
    v = np.where((a == 0) | (b == 0), 0.0, v)
    return v


def _rectangles(power: int, ratio: float):
    """Integrals of u^m v^n R^power over [0,1]|[1,2] x [0,r]|[r,2r] (generatePowerMoments.m:68-119).

    Returns rect[m, n, iu, iv] for m in 0..3, n in 0..1.
    """
    a_s = np.array([0.0, 1.0, 2.0])[:, None] * np.ones((1, 3))
    b_s = np.ones((3, 1)) * (ratio * np.array([0.0, 1.0, 2.0]))[None, :]
    rect = np.zeros((4, 2, 2, 2))
    for m in range(4):
        for n in range(2):
            corners = integrate_monomial(power, m, n, a_s, b_s)
            rect[m, n] = np.diff(np.diff(corners, axis=0), axis=1)
    # Far rectangles: Gauss-Legendre 20 x 20 instead of the cancelling corner sums (:94-118).
    pts, w = gauss_legendre(20, 0.0, 1.0)
    for k in range(2):
        for l in range(2):
            if np.hypot(k, ratio * l) < max(1.0, ratio):
                continue
            u = (k + pts)[:, None]
            v = (ratio * (l + pts))[None, :]
            kern = np.sqrt(u * u + v * v) ** power
            for m in range(4):
                for n in range(2):
                    rect[m, n, k, l] = ratio * (w @ ((u**m) * (v**n) * kern) @ w)
    return rect


# Correlation weights W00, W10, W01, W11 of the rooftop profiles, ascending coefficients in nu on
# the parts [-1, 0] and [0, 1] (generatePowerMoments.m:32-37).
_WEIGHTS = (
    ((1.0, 1.0), (1.0, -1.0)),
    ((0.5, 1.0, 0.5), (0.5, 0.0, -0.5)),
    ((0.5, 0.0, -0.5), (0.5, -1.0, 0.5)),
    ((1 / 3, 0.5, 0.0, -1 / 6), (1 / 3, -0.5, 0.0, 1 / 6)),
)
_TOUCHING = ((0, 0), (1, 0), (0, 1), (1, 1))


def _compose_part(weight, part: int, offset: int, cell: float, count: int):
    """Weight on one part as a polynomial in u = sigma*cell*(nu - offset) (generatePowerMoments.m:121-155)."""
    ends = ((-1.0, 0.0), (0.0, 1.0))[part]
    shifted = (ends[0] - offset, ends[1] - offset)
    sigma = -1.0 if shifted[1] <= 0 else 1.0
    interval = int(min(sigma * shifted[0], sigma * shifted[1]))  # 0 -> [0, cell], 1 -> [cell, 2 cell]
    coeffs = np.zeros(count)
    term = np.array([1.0])
    for k, wk in enumerate(weight):
        coeffs[: k + 1] += wk * term
        term = np.convolve(term, [float(offset), sigma / cell])
    return coeffs, interval


def _along_x(a: float, b: float, power: int):
    """M00, M10, M01, M11 at the 4 touching offsets, 4x4 (generatePowerMoments.m:23-66)."""
    ratio = b / a
    rect = _rectangles(power, ratio)
    mom = np.zeros((4, 4))
    for k in range(4):
        for l, (ox, oy) in enumerate(_TOUCHING):
            for s in range(2):
                ca, ia = _compose_part(_WEIGHTS[k][s], s, ox, 1.0, 4)
                for t in range(2):
                    cb, ib = _compose_part(_WEIGHTS[0][t], t, oy, ratio, 2)
                    mom[k, l] += ca @ rect[:, :, ia, ib] @ cb
    return a**power * mom / ratio


def power_moments(size_x: float, size_y: float, power: int):
    """7x4 moments of R^power divided by (ab)^2 at offsets (0,0),(1,0),(0,1),(1,1).

    Rows M00, M10, M01, M11, N10, N01, N11 (generatePowerMoments.m:17-21).
    """
    ax = _along_x(size_x, size_y, power)
    ay = _along_x(size_y, size_x, power)
    return np.vstack([ax, ay[1:4][:, [0, 2, 1, 3]]])


def extracted_moments(size_x: float, size_y: float, k: float):
    """Moments of S(R) = 1/R - k^2 R/2 + k^4 R^3/24 (generateExtractedMoments.m:16-18)."""
    return (power_moments(size_x, size_y, -1)
            - k**2 / 2 * power_moments(size_x, size_y, 1)
            + k**4 / 24 * power_moments(size_x, size_y, 3))


def remainder(distance, k: float):
    """exp(-ikR)/R - S(R), with exp(-ikR) - 1 = -2 sin^2(kR/2) - i sin(kR) (evaluateRemainder.m:13-14)."""
    d = np.asarray(distance, dtype=np.float64)
    kr = k * d
    s = np.sin(kr / 2)
    em1 = (-2.0 * s * s) - 1j * np.sin(kr)
    return em1 / d + k * k / 2 * d - k**4 / 24 * d**3
