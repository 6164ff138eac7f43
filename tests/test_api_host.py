"""The host side of the Python mirror of the MATLAB API, which needs no GPU until generators are assembled:
Mesh and Problem as the reference's tests/+unit/MeshTest.m:5-29 and ProblemTest.m:5-16, :18-29 and
:64-140 hold them, and the argument checks of Excitation and Solver. MATLAB's argument validators
(MATLAB:validators:*) have no Python counterpart; the mirror raises RtmError with a rooftopMoM:*
identifier for the same inputs."""
from __future__ import annotations

import math

import numpy as np
import pytest

from rooftop_mom_b200 import Mesh, Problem, RtmError


def test_mesh_getters():
    mesh = Mesh(4, 3, 0.1, 0.2)
    assert (*mesh.count(), *mesh.faceSize()) == (4, 3, 0.1, 0.2)


def test_mesh_radius_is_half_the_diagonal():
    assert Mesh(4, 3, 0.1, 0.2).radius() == pytest.approx(math.hypot(0.4, 0.6) / 2, rel=1e-15)


@pytest.mark.parametrize("args", [(0, 3, 0.1, 0.1), (2.5, 3, 0.1, 0.1), (4, 3, -0.1, 0.1), (4, 3, 0.1, math.inf)])
def test_invalid_meshes_raise(args):
    with pytest.raises(RtmError):
        Mesh(*args)


def test_a_single_face_has_no_rooftop():
    with pytest.raises(RtmError) as e:
        Mesh(1, 1, 0.1, 0.1)
    assert e.value.identifier == "rooftopMoM:mesh:noRooftops"


def test_problem_getters():
    mesh = Mesh(4, 3, 0.1, 0.1)
    problem = Problem(mesh, 2 * math.pi, quadratureOrder=3)
    assert problem.mesh() is mesh
    assert problem.wavenumber() == 2 * math.pi
    assert problem.rooftopCount() == 17
    assert problem.quadratureOrder() == (3, 3)


def test_quadrature_orders_of_the_near_and_the_far_pairs():
    mesh = Mesh(4, 3, 0.1, 0.1)
    assert Problem(mesh, 2 * math.pi).quadratureOrder() == (16, 8)
    assert Problem(mesh, 2 * math.pi, quadratureOrder=(12, 6)).quadratureOrder() == (12, 6)


def test_electrical_size_sets_the_wavenumber():
    mesh = Mesh(4, 3, 0.1, 0.2)
    problem = Problem(mesh, electricalSize=0.5, quadratureOrder=3)
    assert problem.wavenumber() == pytest.approx(0.5 / mesh.radius(), rel=1e-15)
    assert problem.electricalSize() == pytest.approx(0.5, rel=1e-15)


def test_density_counts_the_longer_face_side():
    # faces of 0.08 m along y: 12.5 per wavelength of 1 m
    assert Problem(Mesh(4, 3, 0.05, 0.08), 2 * math.pi, quadratureOrder=3).density() == pytest.approx(12.5, rel=1e-15)


def test_from_electrical_size_meshes_the_plate():
    # ka = 4 at 1 m: the diagonal is 4 / pi, the sides 1.139 and 0.569 m, 13.7 and 6.8 faces at 12 a wavelength
    problem = Problem.fromElectricalSize(4, density=12, aspect=2, quadratureOrder=3)
    (cx, cy), (sx, sy) = problem.mesh().count(), problem.mesh().faceSize()
    assert (cx, cy) == (14, 7)
    assert cx * sx / (cy * sy) == pytest.approx(2, rel=1e-14)
    assert problem.wavenumber() == 2 * math.pi
    assert problem.electricalSize() == pytest.approx(4, rel=1e-14)
    assert problem.density() >= 12


def test_from_electrical_size_rounds_the_counts_to_fast_fft_sizes():
    # ka = 4.6 needs 10.35 faces a side at 10 a wavelength; the 11 that reach it round up to 12
    problem = Problem.fromElectricalSize(4.6, density=10, quadratureOrder=3)
    assert problem.mesh().count() == (12, 12)
    assert problem.density() >= 10


def test_from_electrical_size_meshes_a_strip_one_face_across():
    problem = Problem.fromElectricalSize(math.pi / 2, density=20, aspect=250, quadratureOrder=3)
    assert problem.mesh().count() == (10, 1)


def test_from_electrical_size_refuses_a_single_face():
    with pytest.raises(RtmError) as e:
        Problem.fromElectricalSize(0.1)
    assert e.value.identifier == "rooftopMoM:problem:singleFace"


def test_invalid_problems_raise():
    mesh = Mesh(4, 3, 0.1, 0.1)
    with pytest.raises(RtmError):
        Problem(mesh, 0)
    with pytest.raises(RtmError) as e:
        Problem(mesh, 2 * math.pi, quadratureOrder=2.5)
    assert e.value.identifier == "rooftopMoM:problem:invalidQuadratureOrder"
    with pytest.raises(RtmError) as e:
        Problem(mesh, 2 * math.pi, quadratureOrder=(16, 8, 4))
    assert e.value.identifier == "rooftopMoM:problem:invalidQuadratureOrder"
    with pytest.raises(TypeError):
        Problem(mesh, 2 * math.pi, order=3)
    for kwargs in ({}, {"wavenumber": 2 * math.pi, "electricalSize": 2}):
        with pytest.raises(RtmError) as e:
            Problem(mesh, **kwargs)
        assert e.value.identifier == "rooftopMoM:problem:invalidWavenumber"
    with pytest.raises(RtmError):
        Problem(mesh, electricalSize=-1)
    with pytest.raises(RtmError):
        Problem.fromElectricalSize(4, density=0)


# Excitation and Solver arguments (tests/+unit/ExcitationTest.m:5-59, SolverTest.m:46-67): every check
# below runs before any device work, and the delta gap of host memory is built on the host.
def test_plane_wave_normalizes_its_vectors():
    from rooftop_mom_b200 import Excitation

    d, p = Excitation.planeWaveVectors([0, 0, -2], [0, 3, 0])
    np.testing.assert_array_equal(d, [0, 0, -1])
    np.testing.assert_array_equal(p, [0, 1, 0])


def test_plane_wave_needs_perpendicular_nonzero_vectors():
    from rooftop_mom_b200 import Excitation

    with pytest.raises(RtmError) as e:
        Excitation.planeWaveVectors([1, 0, 0], [1, 1, 0])
    assert e.value.identifier == "rooftopMoM:excitation:notPerpendicular"
    with pytest.raises(RtmError) as e:
        Excitation.planeWaveVectors([0, 0, -1], [0, 0, 0])
    assert e.value.identifier == "rooftopMoM:excitation:zeroVector"


def test_plane_wave_accepts_a_rotated_frame():
    from rooftop_mom_b200 import Excitation

    a = (0.3, 1.1, 2.5)
    rx = np.array([[1, 0, 0], [0, math.cos(a[0]), -math.sin(a[0])], [0, math.sin(a[0]), math.cos(a[0])]])
    ry = np.array([[math.cos(a[1]), 0, math.sin(a[1])], [0, 1, 0], [-math.sin(a[1]), 0, math.cos(a[1])]])
    rz = np.array([[math.cos(a[2]), -math.sin(a[2]), 0], [math.sin(a[2]), math.cos(a[2]), 0], [0, 0, 1]])
    frame = rz @ ry @ rx
    Excitation.planeWaveVectors(frame[:, 2], frame[:, 0])


def test_delta_gap_defaults_to_the_middle_port():
    from oracle import excitation as EX
    from oracle.geometry import Rooftops
    from rooftop_mom_b200 import Excitation

    problem = Problem(Mesh(6, 1, 0.1, 0.1), 2 * math.pi, quadratureOrder=3)
    e = Excitation.deltaGap(problem, voltage=2)
    assert e.type() == "deltaGap"
    np.testing.assert_array_equal(e.parameters()["port"], [2])
    assert e.parameters()["voltage"] == 2
    np.testing.assert_array_equal(e.vector(), EX.delta_gap(Rooftops(6, 1, 0.1, 0.1, 3), [2], 2))


def test_delta_gap_checks_the_port():
    from rooftop_mom_b200 import Excitation

    problem = Problem(Mesh(6, 1, 0.1, 0.1), 2 * math.pi, quadratureOrder=3)
    for port in ([1, 1], [5]):
        with pytest.raises(RtmError) as e:
            Excitation.deltaGap(problem, port=port)
        assert e.value.identifier == "rooftopMoM:excitation:invalidPort"
    with pytest.raises(RtmError) as e:
        Excitation.deltaGap(problem, direction="y")
    assert e.value.identifier == "rooftopMoM:excitation:noRooftops"


def test_invalid_solvers_and_solver_inputs_raise():
    from rooftop_mom_b200 import Solver

    for kwargs in ({"method": "bicg"}, {"tolerance": 2}):
        with pytest.raises(RtmError):
            Solver(**kwargs)
    with pytest.raises(RtmError) as e:
        Solver(restart=2.5)
    assert e.value.identifier == "rooftopMoM:solver:invalidRestart"
    with pytest.raises(RtmError) as e:
        Solver(method="gmres", gramSchmidtPasses=3)
    assert e.value.identifier == "rooftopMoM:solver:invalidGramSchmidtPasses"
    from rooftop_mom_b200 import PlateBatch

    with pytest.raises(RtmError) as e:
        PlateBatch([])
    assert e.value.identifier == "rooftopMoM:batch:empty"
    with pytest.raises(RtmError) as e:
        Solver(method="fgmres").solveBatch(None, [])
    assert e.value.identifier == "rooftopMoM:solver:invalidMethod"
    solver = Solver()
    with pytest.raises(RtmError) as e:
        solver.solve("matrix", np.ones(3))
    assert e.value.identifier == "rooftopMoM:solver:invalidOperator"
    for rhs in (np.array([1, np.nan, 3]), ["a", "b", "c"], np.array([True, False, True])):
        with pytest.raises(RtmError) as e:
            solver.solve(np.eye(3), rhs)
        assert e.value.identifier == "rooftopMoM:solver:invalidRightHandSide"
    for guess in (np.array([1, np.inf, 1]), ["a", "b", "c"], np.array([True, False, True])):
        with pytest.raises(RtmError) as e:
            solver.solve(np.eye(3), np.ones(3), initialGuess=guess)
        assert e.value.identifier == "rooftopMoM:solver:invalidInitialGuess"


def test_result_quantities_need_their_excitation():
    # tests/+unit/ResultTest.m:13-14, :24, :43: the checks come before any device work
    from rooftop_mom_b200 import Excitation, Result
    from rooftop_mom_b200 import _lib as L

    problem = Problem(Mesh(6, 1, 0.1, 0.1), 2 * math.pi, quadratureOrder=3)
    gap = Result(np.zeros(5, complex), L.SolveStats(), np.array([1.0]), Excitation.deltaGap(problem))
    for quantity in (gap.radarCrossSection, gap.normalizedRadarCrossSection):
        with pytest.raises(RtmError) as e:
            quantity()
        assert e.value.identifier == "rooftopMoM:result:wrongExcitation"
    plain = Result(np.zeros(3, complex), L.SolveStats(), np.array([1.0]), None)
    with pytest.raises(RtmError) as e:
        plain.inputImpedance()
    assert e.value.identifier == "rooftopMoM:result:wrongExcitation"


def test_invalid_preconditioners_raise_before_any_device_work():
    # tests/+unit/PreconditionerTest.m:62-71
    from rooftop_mom_b200 import Preconditioner

    problem = Problem(Mesh(8, 8, 0.05, 0.05), 2 * math.pi, quadratureOrder=3)
    with pytest.raises(RtmError) as e:
        Preconditioner(problem, kernel="jacobi")
    assert e.value.identifier == "rooftopMoM:preconditioner:invalidKernel"
    for bandwidth in ([1, 2, 3], [0, 2], [1.5, 2]):
        with pytest.raises(RtmError) as e:
            Preconditioner(problem, kernel="huckle", bandwidth=bandwidth)
        assert e.value.identifier == "rooftopMoM:preconditioner:invalidBandwidth"


def test_invalid_operators_raise_before_any_device_work():
    # tests/+unit/OperatorTest.m:35-38, and the modifier of Operator.m / Generators.modify
    from rooftop_mom_b200 import Operator

    problem = Problem(Mesh(8, 8, 0.05, 0.05), 2 * math.pi, quadratureOrder=3)
    for kwargs, identifier in (({"product": "dense"}, "rooftopMoM:operator:invalidProduct"),
                               ({"precision": "half"}, "rooftopMoM:operator:invalidPrecision"),
                               ({"modifier": "abs"}, "rooftopMoM:operator:invalidModifier"),
                               ({"modifier": np.abs}, "rooftopMoM:operator:invalidModifier")):
        with pytest.raises(RtmError) as e:
            Operator(problem, **kwargs)
        assert e.value.identifier == identifier


def test_problem_memory_is_zero_before_the_assembly():
    # Problem.m:147-155: the bytes of the generators once assembled, zero before
    problem = Problem(Mesh(4, 3, 0.1, 0.1), 2 * math.pi, quadratureOrder=3)
    assert problem.memory() == 0.0
