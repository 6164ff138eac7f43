"""Shared fixtures: the `gpu` marker, the golden fixtures and seeded inputs."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and librtm.so")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this container")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(GOLDEN, "reference_cases.npz"))


def reference_case(golden, c):
    """Grid, generators and stored vectors of reference case c (tests/data/reference.mat)."""
    g = lambda n: golden[f"c{c}_{n}"]
    xx, yy = g("magneticXX"), g("magneticYY")
    return {
        "countX": int(g("countX")), "countY": int(g("countY")),
        "sizeX": float(g("sizeX")), "sizeY": float(g("sizeY")),
        "order": int(g("order")), "wavenumber": float(g("wavenumber")),
        "magneticXX": xx if xx.size else None, "magneticYY": yy if yy.size else None,
        "electric": g("electric"), "vector": g("vector"),
        "productFFT": g("productFFT"), "productSplit": g("productSplit"), "productLean": g("productLean"),
        "preconditioned": [g("preconditioned0"), g("preconditioned1")],
        "direction": g("direction"), "polarization": g("polarization"), "intensity": float(g("intensity")),
        "planeWave": g("planeWave"), "impedanceMatrix": g("impedanceMatrix"),
    }


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def random_vector(n, seed=1):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)
