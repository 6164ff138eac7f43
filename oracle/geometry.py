"""Grid, rooftop layout, Gauss-Legendre rules and physical constants (oracle; test infrastructure).

Follows:
  src/+rooftopMoM/+mesh/UniformRectPrimitive.m:1-44
  src/+rooftopMoM/+basisFunctions/UniformRooftops.m:31-132
  src/+rooftopMoM/+basisFunctions/GaussLegendre2RectQuadrature.m:13-22
  src/+rooftopMoM/+basisFunctions/+utils/generateGaussLegendre1D.m:16-25
  src/+rooftopMoM/+assembler/Constants.m:8-17
"""
from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

import numpy as np
from scipy.linalg import eigh_tridiagonal

# Constants.m:8-17 (CODATA 2018): c exact, Z0 given, mu0 and epsilon0 derived.
SPEED_OF_LIGHT = 299792458.0
Z0 = 376.730313668
MU0 = Z0 / SPEED_OF_LIGHT
EPSILON0 = 1.0 / (Z0 * SPEED_OF_LIGHT)

# RooftopContent.m:5-10
NONE, XONLY, YONLY, BOTH = 0, 1, 2, 3


@lru_cache(maxsize=None)
def _gauss_legendre_unit(order: int):
    """Golub-Welsch on [-1, 1]: eigenvalues of the Jacobi matrix, weights 2 v_0^2.

    generateGaussLegendre1D.m:16-22.
    """
    if order == 1:
        return np.zeros(1), np.full(1, 2.0)
    n = np.arange(1, order, dtype=np.float64)
    off = n / np.sqrt(4.0 * n * n - 1.0)
    values, vectors = eigh_tridiagonal(np.zeros(order), off)
    perm = np.argsort(values)
    values = values[perm]
    weights = 2.0 * vectors[0, perm] ** 2
    return values, weights


def gauss_legendre(order: int, a: float = 0.0, b: float = 1.0):
    """Points (ascending) and weights of the order-point Gauss-Legendre rule on [a, b].

    generateGaussLegendre1D.m:24-25.
    """
    values, weights = _gauss_legendre_unit(int(order))
    points = (a + b) / 2.0 + (b - a) / 2.0 * values
    return points, (b - a) / 2.0 * weights


def quadrature_2d(order: int):
    """Tensor rule on the unit square, u running fastest.

    GaussLegendre2RectQuadrature.m:13-22: returns (pointsU, pointsV, weights2D), each of length order^2.
    """
    p, w = gauss_legendre(order, 0.0, 1.0)
    pu = np.tile(p, order)
    pv = np.repeat(p, order)
    w2 = np.tile(w, order) * np.repeat(w, order)
    return pu, pv, w2


@dataclass(frozen=True)
class Rooftops:
    """Rooftops of unit height on a countX x countY grid of sizeX x sizeY faces.

    UniformRooftops.m:1-8: x-directed rooftops first, then y-directed; within a direction the x
    index runs fastest (column-major grids of (countX-1) x countY and countX x (countY-1)).
    ``order`` is the far quadrature order, used by the excitation only (Problem.m:62-64).
    """

    count_x: int
    count_y: int
    size_x: float
    size_y: float
    order: int = 8

    def grid_size(self, direction: str):
        # UniformRooftops.m:44-55
        if direction == "x":
            return self.count_x - 1, self.count_y
        return self.count_x, self.count_y - 1

    def count_dir(self, direction: str) -> int:
        r, c = self.grid_size(direction)
        return r * c

    @property
    def count(self) -> int:
        return self.count_dir("x") + self.count_dir("y")

    @property
    def content(self) -> int:
        # UniformRooftops.m:57-72
        hx = self.count_dir("x") > 0
        hy = self.count_dir("y") > 0
        if hx and hy:
            return BOTH
        if hx:
            return XONLY
        if hy:
            return YONLY
        return NONE

    def edge_lengths(self, indices):
        """Edge length of rooftops (0-based indices): sizeY for x-directed, sizeX for y-directed.

        UniformRooftops.m:89-101.
        """
        indices = np.asarray(indices)
        out = np.full(indices.shape, self.size_x, dtype=np.float64)
        out[indices < self.count_dir("x")] = self.size_y
        return out

    def reference_rooftop(self, direction: str):
        """UniformRooftops.m:103-132: amplitudes (B x 2) on the rising and falling faces."""
        pu, pv, _ = quadrature_2d(self.order)
        if direction == "x":
            coord = pu
            second = (1, 0)
            length, height = self.size_x, self.size_y
        else:
            coord = pv
            second = (0, 1)
            length, height = self.size_y, self.size_x
        amps = np.stack([coord, 1.0 - coord], axis=1)
        return {"second_face_offset": second, "length": length, "height": height, "amplitudes": amps}


def fast_fft_size(count: int) -> int:
    """Smallest size >= count whose prime factors are at most 7 (generateFastFFTSize.m:11-15)."""
    n = int(count)
    while True:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1
