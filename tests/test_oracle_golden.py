"""The oracle against the reference's golden data and the invariants of its unit tests (CPU only).

Golden data: tests/data/reference.mat and tests/data/exactMoments.csv of the reference, copied into
tests/golden/ by tests/golden/make_golden.py. Tolerances are those of the reference's tests.
"""
from __future__ import annotations

import csv
import os

import numpy as np
import pytest

from conftest import GOLDEN, reference_case, rel
from oracle import assembly as A
from oracle import excitation as EX
from oracle import geometry as G
from oracle import preconditioner as PC
from oracle import singular as SI
from oracle import solvers as OS
from oracle import spectra as S


def _rt_gen(d):
    rt = G.Rooftops(d["countX"], d["countY"], d["sizeX"], d["sizeY"], d["order"])
    return rt, A.Generators(d["magneticXX"], d["magneticYY"], d["electric"], rt.content)


@pytest.mark.parametrize("case", [0, 1, 2])
def test_products_match_reference_mat(golden, case):
    # +reference/+assembler/+greensMatrix/ApplicatorTest.m:5-21 (1e-13)
    d = reference_case(golden, case)
    rt, gen = _rt_gen(d)
    sub = S.subband_spectra(gen, d["sizeX"], d["sizeY"])
    emb = S.embedding_spectra(gen, d["sizeX"], d["sizeY"])
    assert rel(S.split_apply(rt, sub, rt.content, d["vector"]), d["productSplit"]) < 1e-13
    assert rel(S.lean_apply(rt, sub, rt.content, d["vector"]), d["productLean"]) < 1e-13
    assert rel(S.fft_apply(rt, emb, rt.content, d["vector"]), d["productFFT"]) < 1e-13


def test_dense_matrix_matches_reference_mat(golden):
    # +reference/+assembler/+greensMatrix/ApplicatorTest.m:23-34 (1e-10) and the dense oracle of tests/+unit/Base.m
    d = reference_case(golden, 0)
    rt, gen = _rt_gen(d)
    emb = S.embedding_spectra(gen, d["sizeX"], d["sizeY"])
    assert rel(S.fft_apply(rt, emb, rt.content, d["vector"]), d["impedanceMatrix"] @ d["vector"]) < 1e-10
    assert rel(EX.dense_matrix(gen, rt) @ d["vector"], d["productFFT"]) < 1e-13


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("k", [0, 1])
def test_preconditioners_match_reference_mat(golden, case, k):
    # +reference/+assembler/+preconditioner/GenerateCirculantTest.m:5-25 (1e-12)
    d = reference_case(golden, case)
    rt, gen = _rt_gen(d)
    inv = PC.circulant(gen, d["sizeX"], d["sizeY"], ["strang", "tChan"][k], "partwise")
    assert rel(S.fft_apply(rt, inv, rt.content, d["vector"]), d["preconditioned"][k]) < 1e-12


@pytest.mark.parametrize("case", [0, 1, 2])
def test_plane_wave_matches_reference_mat(golden, case):
    # +reference/+operator/GeneratePlaneWaveTest.m:5-13 (1e-13)
    d = reference_case(golden, case)
    rt, _ = _rt_gen(d)
    pw = EX.plane_wave(rt, d["wavenumber"], d["direction"], d["polarization"], d["intensity"])
    assert rel(pw, d["planeWave"]) < 1e-13


def test_power_moments_match_exact_moments():
    # +unit/+assembler/+singularIntegrals/GeneratePowerMomentsTest.m:9-30 (1e-13, 1e-12 beyond aspect 4)
    rows = list(csv.reader(open(os.path.join(GOLDEN, "exact_moments.csv"))))[1:]
    assert len(rows) == 60
    col = {(0, 0): 0, (1, 0): 1, (0, 1): 2, (1, 1): 3}
    for r in rows:
        a, b, p, dx, dy = float(r[0]), float(r[1]), int(r[2]), int(r[3]), int(r[4])
        exact = np.array([float(v) for v in r[5:12]])
        got = SI.power_moments(a, b, p)[:, col[(dx, dy)]]
        tol = 1e-12 if max(a, b) / min(a, b) > 4 else 1e-13
        np.testing.assert_allclose(got, exact, rtol=tol)


def test_lattice_equals_per_offset_integration():
    # +unit/+assembler/+greensMatrix/MomentAssemblerTest.m:55-77 (1e-14)
    counts, h, order, k = (9, 7), 0.1, 6, 2 * np.pi
    gen = A.generate(9, 7, h, h, k, (order, order))
    rule = A.reduced_rule(order, (1, 1))
    dX, dY = np.meshgrid(np.arange(9), np.arange(7), indexing="ij")
    offs = np.stack([dX.ravel(order="F"), dY.ravel(order="F")])
    e, xx, yy = A.allocate_parts(counts, (1, 1))
    parts = A.Generators(xx, yy, e, G.BOTH)
    sc = A.scales_of(h, h, k)
    A.accumulate_moments(parts, A.integrate_moments(rule, offs, (h, h), k), offs, sc)
    A.accumulate_moments(parts, SI.extracted_moments(h, h, k), np.array([[0, 1, 0, 1], [0, 0, 1, 1]]), sc)
    for name in ("electric", "magnetic_xx", "magnetic_yy"):
        np.testing.assert_allclose(getattr(gen, name), getattr(parts, name), rtol=1e-14)


@pytest.mark.parametrize("case", [(12, 12, 0.1, 0.1), (6, 40, 0.1, 0.01), (30, 1, 0.025, 0.004)])
def test_default_orders_reach_the_rounding_level(case):
    # MomentAssemblerTest.m:79-91 (3e-14)
    d = A.generate(*case, 2 * np.pi, (16, 8))
    p = A.generate(*case, 2 * np.pi, (32, 24))
    for name in ("electric", "magnetic_xx", "magnetic_yy"):
        x, y = getattr(d, name), getattr(p, name)
        if x is not None:
            np.testing.assert_allclose(x, y, rtol=3e-14)


def test_generators_do_not_depend_on_the_grid_size():
    # MomentAssemblerTest.m:24-33 (1e-13)
    narrow = A.generate(2, 3, 0.1, 0.1, 2 * np.pi, (3, 3))
    wide = A.generate(5, 3, 0.1, 0.1, 2 * np.pi, (3, 3))
    np.testing.assert_allclose(narrow.magnetic_xx, wide.magnetic_xx[:1, :], rtol=1e-13)
    np.testing.assert_allclose(narrow.magnetic_yy, wide.magnetic_yy[:2, :], rtol=1e-13)
    np.testing.assert_allclose(narrow.electric, wide.electric[:2, :], rtol=1e-13)


def test_transposed_grid_transposes_the_generators():
    # MomentAssemblerTest.m:35-43 (1e-13)
    g = A.generate(5, 4, 0.1, 0.15, 2 * np.pi, (4, 4))
    t = A.generate(4, 5, 0.15, 0.1, 2 * np.pi, (4, 4))
    np.testing.assert_allclose(t.magnetic_yy, g.magnetic_xx.T, rtol=1e-13)
    np.testing.assert_allclose(t.electric, g.electric.T, rtol=1e-13)


def test_reduced_rule_is_exact_on_polynomials():
    # +unit/+assembler/+greensMatrix/+utils/GenerateReducedRuleTest.m: W00 integrates to 1 on [-1, 1]
    nx, ny, w = A.reduced_rule(5, (2, 3))
    # the M00 row integrates 1 to (int W00)^2 = 1
    assert abs(w[0].sum() - 1.0) < 1e-14
    # M10 row integrates the constant to int W10 = 1/2 (times int W00 = 1)
    assert abs(w[1].sum() - 0.5) < 1e-14
    # M11: int W11 = int (1 - |nu|)^2 (2 + |nu|) / 6 = 1/4
    assert abs(w[3].sum() - 0.25) < 1e-14


@pytest.mark.parametrize("method", ["cg", "gmres"])
def test_oracle_solvers_converge_on_dense_systems(method):
    rng = np.random.default_rng(1)
    n = 40
    r = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    Am = 4 * np.eye(n) + (r + r.T) / 2
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    out = OS.solve(method, Am, b, tol=1e-10, restart=10)
    assert out.converged and out.residual_norm < 1e-10
    assert len(out.residual_norms) == out.iteration_count + 1


def test_gauss_legendre_is_exact():
    p, w = G.gauss_legendre(8, 0.0, 1.0)
    for deg in range(16):
        assert abs(w @ p**deg - 1.0 / (deg + 1)) < 1e-15


def test_fast_fft_sizes():
    assert [G.fast_fft_size(n) for n in (1, 11, 13, 97, 1031, 1024)] == [1, 12, 14, 98, 1050, 1024]
