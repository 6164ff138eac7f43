"""GPU products, spectra, preconditioners and excitations against the reference's golden data and
the oracle (the reference's tests: +reference/+assembler/+greensMatrix/ApplicatorTest.m,
+reference/+assembler/+preconditioner/GenerateCirculantTest.m, +reference/+operator/GeneratePlaneWaveTest.m,
+unit/+assembler/+greensMatrix/ApplicatorTest.m)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import reference_case, rel, random_vector

pytestmark = pytest.mark.gpu

PRODUCTS = ("fft", "splitFFT", "leanSplitFFT")
FIELDS = {"fft": "productFFT", "splitFFT": "productSplit", "leanSplitFFT": "productLean"}


def _problem_from_reference(d):
    import rooftop_mom_b200 as R

    mesh = R.Mesh(d["countX"], d["countY"], d["sizeX"], d["sizeY"])
    prob = R.Problem(mesh, d["wavenumber"], quadratureOrder=d["order"])
    prob.setGenerators(R.Generators.fromArrays(mesh, d["magneticXX"], d["magneticYY"], d["electric"]))
    return prob


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("product", PRODUCTS)
def test_products_match_the_reference(golden, case, product):
    import rooftop_mom_b200 as R

    d = reference_case(golden, case)
    op = R.Operator(_problem_from_reference(d), product=product)
    assert rel(op.apply(d["vector"]), d[FIELDS[product]]) < 1e-13


def test_product_matches_the_reference_dense_matrix(golden):
    import rooftop_mom_b200 as R

    d = reference_case(golden, 0)
    op = R.Operator(_problem_from_reference(d), product="fft")
    assert rel(op.apply(d["vector"]), d["impedanceMatrix"] @ d["vector"]) < 1e-10


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("k", [0, 1])
def test_partwise_preconditioners_match_the_reference(golden, case, k):
    import rooftop_mom_b200 as R

    d = reference_case(golden, case)
    pc = R.Preconditioner(_problem_from_reference(d), kernel=["strang", "tChan"][k], builder="partwise")
    assert rel(pc.apply(d["vector"]), d["preconditioned"][k]) < 1e-12


@pytest.mark.parametrize("case", [0, 1, 2])
def test_plane_wave_matches_the_reference(golden, case):
    import rooftop_mom_b200 as R

    d = reference_case(golden, case)
    prob = _problem_from_reference(d)
    exc = R.Excitation.planeWave(prob, direction=d["direction"], polarization=d["polarization"],
                                 intensity=d["intensity"])
    assert rel(exc.vector(), d["planeWave"]) < 1e-13


GRIDS = {
    "plate": (5, 4, 0.1, 0.15),
    "oddPlate": (11, 7, 0.1, 0.1),
    "twoFacesWide": (2, 5, 0.1, 0.1),
    "stripX": (9, 1, 0.1, 0.02),
    "stripY": (1, 6, 0.03, 0.1),
    "square32": (32, 32, 0.05, 0.05),
    "prime": (13, 17, 0.07, 0.05),
}


@pytest.mark.parametrize("name", sorted(GRIDS))
@pytest.mark.parametrize("product", PRODUCTS)
def test_products_match_the_dense_matrix(name, product):
    """+unit/+assembler/+greensMatrix/ApplicatorTest.m: product of the assembled generators vs the
    dense matrix of the same generators (oracle), rel 1e-12; the GPU generators vs the oracle's."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, excitation as EX, geometry as G

    cx, cy, a, b = GRIDS[name]
    mesh = R.Mesh(cx, cy, a, b)
    prob = R.Problem(mesh, 2 * np.pi, quadratureOrder=3)
    gen_gpu = prob.generators()
    xx, yy, e = gen_gpu.arrays()
    ref = A.generate(cx, cy, a, b, 2 * np.pi, (3, 3))
    assert rel(e, ref.electric) < 1e-12
    if ref.magnetic_xx is not None:
        assert rel(xx, ref.magnetic_xx) < 1e-12
    if ref.magnetic_yy is not None:
        assert rel(yy, ref.magnetic_yy) < 1e-12
    rt = G.Rooftops(cx, cy, a, b, 3)
    dense = EX.dense_matrix(A.Generators(xx, yy, e, rt.content), rt)
    v = random_vector(rt.count, seed=1)
    assert rel(R.Operator(prob, product=product).apply(v), dense @ v) < 1e-12


@pytest.mark.parametrize("name,content", [("plate", 3), ("stripX", 1), ("stripY", 2)])
def test_generators_info_reports_the_grid_and_content(name, content):
    """rtm_generators_info: the face counts and the rooftop content (RTM_BOTH, RTM_XONLY, RTM_YONLY) of
    assembled generators (Generators.content, Generators.m)."""
    import ctypes as C

    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    cx, cy, a, b = GRIDS[name]
    gen = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3).generators()
    got = [C.c_int(), C.c_int(), C.c_int()]
    L.call("rtm_generators_info", gen.handle, *[C.byref(v) for v in got])
    assert [v.value for v in got] == [cx, cy, content]


@pytest.mark.parametrize("name", ["plate", "stripX", "stripY"])
@pytest.mark.parametrize("modifier", ["real", "imag"])
@pytest.mark.parametrize("product", PRODUCTS)
def test_the_modifier_selects_a_part_of_the_matrix(product, modifier, name):
    """+unit/OperatorTest.m:18-25: the operator of the real or imaginary part of the generators
    (Generators.modify, rtm_generators_modify) is that part of the dense matrix, rel 1e-12."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, excitation as EX, geometry as G

    cx, cy, a, b = GRIDS[name]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 3)
    part = np.real if modifier == "real" else np.imag
    dense = part(EX.dense_matrix(A.Generators(xx, yy, e, rt.content), rt))
    v = random_vector(rt.count, seed=2)
    assert rel(R.Operator(prob, product=product, modifier=modifier).apply(v), dense @ v) < 1e-12


@pytest.mark.parametrize("name", ["plate", "oddPlate", "stripX", "stripY", "square32"])
def test_spectra_match_the_oracle(name):
    import rooftop_mom_b200 as R
    from oracle import assembly as A, spectra as S

    cx, cy, a, b = GRIDS[name]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    op = R.Operator(prob, product="splitFFT")
    xx, yy, e = prob.generators().arrays()
    content = 3 if (cx > 1 and cy > 1) else (1 if cy == 1 else 2)
    sub = S.subband_spectra(A.Generators(xx, yy, e, content), a, b)
    got = op.spectra()
    if content == 3:
        for s in range(4):
            # E, MXX, MYY per subband: rebuild the reference blocks from the raw spectra
            blk = sub[s]
            P, Q = got.shape[1:]
            sx, sy = S.shift_phases(P, Q, s % 2, s // 2)
            mine = S.block_spectra(got[3 * s + 1], got[3 * s + 2], got[3 * s], content, a, b, sx, sy)
            for f in ("xx", "xy", "yx", "yy"):
                assert rel(getattr(mine, f), getattr(blk, f)) < 1e-13
    else:
        for s in range(2):
            want = sub[s].xx if content == 1 else sub[s].yy
            assert rel(got[s].ravel(), want.ravel()) < 1e-13


@pytest.mark.parametrize("kernel", ["strang", "tChan", "rChan", "huckle"])
@pytest.mark.parametrize("name", ["plate", "oddPlate", "stripX", "stripY", "prime"])
def test_circulant_preconditioners_match_the_oracle(kernel, name):
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, preconditioner as PC, spectra as S

    cx, cy, a, b = GRIDS[name]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    bw = (max(1, cx // 2), max(1, cy // 2)) if kernel == "huckle" else None
    pc = R.Preconditioner(prob, kernel=kernel, bandwidth=bw)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 3)
    inv = PC.circulant(A.Generators(xx, yy, e, rt.content), a, b, kernel, "partwise", bw)
    v = random_vector(rt.count, seed=3)
    assert rel(pc.apply(v), S.fft_apply(rt, inv, rt.content, v)) < 1e-12


@pytest.mark.parametrize("builder", ["partwise", "blockwise", "hybrid"])
@pytest.mark.parametrize("kernel", ["strang", "tChan", "rChan", "huckle", "superoptimal"])
@pytest.mark.parametrize("name", ["plate", "oddPlate", "twoFacesWide", "stripX", "stripY", "prime"])
def test_every_kernel_and_builder_matches_the_oracle(kernel, builder, name):
    """generateCirculant.m:16-25 for the kernels x builders of Preconditioner.m:26-29; the oracle's
    superoptimal kernel and spatial blocks are pinned to the reference's known answers on the CPU."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, preconditioner as PC, spectra as S

    cx, cy, a, b = GRIDS[name]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    bw = (max(1, cx // 2), max(1, cy // 2)) if kernel == "huckle" else None
    pc = R.Preconditioner(prob, kernel=kernel, builder=builder, bandwidth=bw)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 3)
    inv = PC.circulant(A.Generators(xx, yy, e, rt.content), a, b, kernel, builder, bw)
    v = random_vector(rt.count, seed=5)
    # the superoptimal kernel chains ~40 transforms and a spectral division: 1e-10; the folds: 1e-11
    assert rel(pc.apply(v), S.fft_apply(rt, inv, rt.content, v)) < (1e-10 if kernel == "superoptimal" else 1e-11)


def test_single_precision_product_is_within_fp32_rounding():
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(64, 48, 0.05, 0.05), 2 * np.pi)
    v = random_vector(prob.rooftopCount(), seed=4)
    y64 = R.Operator(prob, precision="double").apply(v)
    y32 = R.Operator(prob, precision="single").apply(v)
    assert rel(y32, y64) < 2e-5


def test_size_mismatch_raises_the_reference_error():
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(5, 4, 0.1, 0.15), 2 * np.pi)
    op = R.Operator(prob)
    with pytest.raises(R.RtmError) as e:
        op.apply(np.zeros(prob.rooftopCount() + 1, complex))
    assert e.value.identifier == "rooftopMoM:product:sizeMismatch"


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("count", [(32, 32), (64, 64), (64, 128), (128, 64), (256, 256), (512, 512), (1024, 1024)])
def test_power_of_two_products_match_the_oracle(count, precision):
    """The power-of-two fast path (transform sizes 32..1024; FP64 up to 512, the generic engine above)
    against the oracle's split product (applyBothDirections_.m:14-85) of the same generators. Every line
    length runs in both directions: 64 x 128 and 128 x 64 exchange the x-mix and the y transforms."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, spectra as S

    cx, cy = count
    a = b = 0.05
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 8)
    sub = S.subband_spectra(A.Generators(xx, yy, e, rt.content), a, b)
    v = random_vector(rt.count, seed=6)
    want = S.split_apply(rt, sub, rt.content, v)
    got = R.Operator(prob, precision=precision).apply(v)
    assert rel(got, want) < (1e-13 if precision == "double" else 2e-5)


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batched_power_of_two_product_equals_single_products(precision):
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(64, 32, 0.05, 0.05), 2 * np.pi)
    n = prob.rooftopCount()
    op = R.Operator(prob, precision=precision, maxRhs=3)
    vs = [random_vector(n, seed=20 + k) for k in range(3)]
    ys = op.apply(np.concatenate(vs), nrhs=3)
    for k in range(3):
        assert rel(ys[k * n:(k + 1) * n], op.apply(vs[k])) < 1e-14


def test_batched_product_equals_single_products():
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(40, 24, 0.05, 0.05), 2 * np.pi)
    n = prob.rooftopCount()
    op = R.Operator(prob, maxRhs=4)
    vs = [random_vector(n, seed=10 + k) for k in range(4)]
    ys = op.apply(np.concatenate(vs), nrhs=4)
    for k in range(4):
        assert rel(ys[k * n:(k + 1) * n], op.apply(vs[k])) < 1e-15 + 1e-14


@pytest.mark.parametrize("kernel", ["rChan", "tChan"])
def test_a_singular_circulant_raises(kernel):
    """+unit/PreconditionerTest.m:57-60: generators that vanish make every block spectrum zero, so the
    circulant cannot be inverted (rooftopMoM:preconditioner:singular)."""
    import rooftop_mom_b200 as R
    from rooftop_mom_b200 import _lib as L

    mesh = R.Mesh(5, 4, 0.1, 0.15)
    prob = R.Problem(mesh, 2 * np.pi, quadratureOrder=3)
    prob.setGenerators(R.Generators.fromArrays(mesh, np.zeros((4, 4), complex), np.zeros((5, 3), complex),
                                               np.zeros((5, 4), complex)))
    with pytest.raises(L.RtmError) as e:
        R.Preconditioner(prob, kernel=kernel)
    assert e.value.identifier == "rooftopMoM:preconditioner:singular"


# Face grids whose counts have a prime factor above the largest direct radix (61): their transforms run as
# Bluestein (chirp-z) convolutions of a power-of-two length (FFTApplicator.m:57,70 takes any face count).
BLUESTEIN_GRIDS = {
    "prime67": (67, 67, 0.05, 0.05),
    "prime127x131": (127, 131, 0.05, 0.04),
    "strip1x127": (1, 127, 0.01, 0.05),
    "strip127x1": (127, 1, 0.05, 0.01),
    "mixed134x71": (134, 71, 0.05, 0.05),
}


@pytest.mark.parametrize("name", sorted(BLUESTEIN_GRIDS))
@pytest.mark.parametrize("kernel", ["rChan", "strang", "tChan"])
def test_circulants_on_large_prime_face_grids_match_the_oracle(name, kernel):
    """The reference's default rChan / partwise preconditioner (Preconditioner.m:26-29) and the Strang and
    T. Chan ones on face grids of 67, 127, 131 faces: built and applied through Bluestein transforms,
    against the oracle's circulant (1e-11, as the folds on the other grids)."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, preconditioner as PC, spectra as S

    cx, cy, a, b = BLUESTEIN_GRIDS[name]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    pc = R.Preconditioner(prob, kernel=kernel)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 3)
    inv = PC.circulant(A.Generators(xx, yy, e, rt.content), a, b, kernel, "partwise")
    v = random_vector(rt.count, seed=7)
    assert rel(pc.apply(v), S.fft_apply(rt, inv, rt.content, v)) < 1e-11


@pytest.mark.parametrize("builder", ["blockwise", "hybrid"])
def test_other_builders_on_a_large_prime_face_grid_match_the_oracle(builder):
    import rooftop_mom_b200 as R
    from oracle import assembly as A, geometry as G, preconditioner as PC, spectra as S

    cx, cy, a, b = BLUESTEIN_GRIDS["prime67"]
    prob = R.Problem(R.Mesh(cx, cy, a, b), 2 * np.pi, quadratureOrder=3)
    pc = R.Preconditioner(prob, kernel="rChan", builder=builder)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, a, b, 3)
    inv = PC.circulant(A.Generators(xx, yy, e, rt.content), a, b, "rChan", builder)
    v = random_vector(rt.count, seed=8)
    assert rel(pc.apply(v), S.fft_apply(rt, inv, rt.content, v)) < 1e-11


@pytest.mark.parametrize("precision", ["double", "single"])
def test_large_prime_circulant_in_both_precisions_against_fp64(precision):
    """The FP32 Bluestein tables (the precision form's inner preconditioner) against the FP64 apply."""
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(127, 131, 0.05, 0.04), 2 * np.pi, quadratureOrder=3)
    v = random_vector(prob.rooftopCount(), seed=9)
    ref = R.Preconditioner(prob, kernel="rChan").apply(v)
    got = R.Preconditioner(prob, kernel="rChan", precision=precision).apply(v)
    assert rel(got, ref) < (1e-14 if precision == "double" else 2e-5)


@pytest.mark.parametrize("count", [(68, 40), (40, 68), (68, 1)])
def test_fft_product_with_a_large_prime_embedding_matches_the_dense_matrix(count):
    """The 'fft' product embeds on 2n - 2 faces (generateEmbeddingSpectra.m); 2 * 68 - 2 = 2 * 67 runs as a
    Bluestein transform."""
    import rooftop_mom_b200 as R
    from oracle import assembly as A, excitation as EX, geometry as G

    cx, cy = count
    prob = R.Problem(R.Mesh(cx, cy, 0.05, 0.05), 2 * np.pi, quadratureOrder=3)
    xx, yy, e = prob.generators().arrays()
    rt = G.Rooftops(cx, cy, 0.05, 0.05, 3)
    dense = EX.dense_matrix(A.Generators(xx, yy, e, rt.content), rt)
    v = random_vector(rt.count, seed=10)
    assert rel(R.Operator(prob, product="fft").apply(v), dense @ v) < 1e-12


def test_a_rchan_cocg_solve_on_a_large_prime_plate_converges():
    """COCG with the reference's default preconditioner on a 67 x 67 plate (before the Bluestein stage
    this preconditioner could not be built on it)."""
    import rooftop_mom_b200 as R

    prob = R.Problem(R.Mesh(67, 67, 1 / 20, 1 / 20), 2 * np.pi)
    op = R.Operator(prob)
    exc = R.Excitation.planeWave(prob)
    plain = R.Solver(method="cg", tolerance=1e-8, maxIterationCount=5000).solve(op, exc)
    pre = R.Solver(method="cg", tolerance=1e-8, maxIterationCount=5000).solve(op, exc,
                                                                              preconditioner=R.Preconditioner(prob))
    assert plain.converged() and pre.converged()
    assert pre.iterationCount() < plain.iterationCount()
    assert rel(pre.solution(), plain.solution()) < 1e-6
