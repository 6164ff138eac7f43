"""Regenerate the golden fixtures of this directory from the reference's own test data.

Reads (only when run by hand, in a container that has the reference checkout):
  <reference>/tests/data/reference.mat     -> reference_cases.npz
  <reference>/tests/data/exactMoments.csv  -> exact_moments.csv (copied verbatim)

reference.mat holds three grids (5x4 a=0.1 b=0.15, 6x1, 1x5; order 3/4/3; k = 2 pi), each with the
v2 generators, a seeded input vector, the FFT / split / lean products of it, the partwise Strang and
T. Chan preconditioned vectors, a plane wave, and for the first grid the dense impedance matrix
(tests/data/generateReferenceData.m:20-37 of the reference). exactMoments.csv holds the moments of
R^-1, R, R^3 over five cells at the four touching offsets to 30 digits
(tests/data/generateExactMoments.py of the reference).

Usage: python tests/golden/make_golden.py <reference_root>
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np
import scipy.io

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root: str) -> None:
    data = scipy.io.loadmat(os.path.join(root, "tests", "data", "reference.mat"))["reference"]
    out = {}
    for c in range(data.shape[1]):
        case = data[0, c]
        for name in case.dtype.names:
            v = case[name]
            if name == "preconditioned":
                for kk, item in enumerate(v.ravel()):
                    out[f"c{c}_preconditioned{kk}"] = np.asarray(item).astype(np.complex128).ravel()
                continue
            v = np.asarray(v)
            if v.size == 0:
                out[f"c{c}_{name}"] = np.zeros((0, 0))
                continue
            if name in ("countX", "countY", "order"):
                out[f"c{c}_{name}"] = np.array(int(v.ravel()[0]))
            elif name in ("sizeX", "sizeY", "wavenumber", "intensity"):
                out[f"c{c}_{name}"] = np.array(float(v.ravel()[0]))
            elif name in ("vector", "productFFT", "productSplit", "productLean", "planeWave", "direction",
                          "polarization"):
                out[f"c{c}_{name}"] = v.astype(np.complex128 if np.iscomplexobj(v) else np.float64).ravel()
            else:
                out[f"c{c}_{name}"] = v
    out["case_count"] = np.array(data.shape[1])
    np.savez_compressed(os.path.join(HERE, "reference_cases.npz"), **out)
    shutil.copyfile(os.path.join(root, "tests", "data", "exactMoments.csv"), os.path.join(HERE, "exact_moments.csv"))
    print("wrote", sorted(out)[:8], "...", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference_root>")
    main(sys.argv[1])
