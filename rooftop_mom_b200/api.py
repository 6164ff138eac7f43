"""Host-side mirror of the reference's MATLAB API for the solve path, over the C ABI.

The classes keep the names, arguments and error identifiers of src/+rooftopMoM/{Mesh,Problem,
Operator,Preconditioner,Solver,Excitation,Result,Resources}.m; their bodies call librtm.so, which
assembles, transforms and solves on the GPU. Vectors are numpy arrays (host) or CUDA torch tensors
(device, complex128, or complex64 for single-precision products).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import RtmError

Z0 = 376.730313668  # src/+rooftopMoM/+assembler/Constants.m:11
SPEED_OF_LIGHT = 299792458.0  # Constants.m:8


def _err(identifier: str, message: str):
    return RtmError(L.ERR_ARG, message, identifier)


def _is_device(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _vec_in(x, n: int, dtype=np.complex128):
    """(pointer, where, keepalive) of a vector argument of n * nrhs complex entries."""
    if _is_device(x):
        if not x.is_contiguous():
            x = x.contiguous()
        return C.c_void_p(x.data_ptr()), L.DEVICE, x
    a = np.ascontiguousarray(np.asarray(x, dtype=dtype))
    return a.ctypes.data_as(C.c_void_p), L.HOST, a


def format_bytes(count: float) -> str:
    """A byte count as the reference's messages write it (src/+rooftopMoM/+resources/+utils/formatBytes.m)."""
    if math.isinf(count):
        return "unlimited"
    if math.isnan(count):
        return "unknown"
    units = ("B", "kB", "MB", "GB", "TB")
    e = min(max(math.floor(math.log2(max(count, 1.0)) / 10), 0), len(units) - 1)
    return f"{round(count)} B" if e == 0 else f"{count / 1024 ** e:.1f} {units[e]}"


def assembly_bytes(countX: int, countY: int):
    """(generators, working) device bytes of an assembly: the three generators (estimateGenerators.m:11) and
    the 28 lattice-block sums and 7 moment terms of each of the (countX + 1)(countY + 1) blocks."""
    rooftops = (countX - 1) * countY + countX * (countY - 1)
    return 16.0 * (rooftops + countX * countY), 16.0 * 35 * (countX + 1) * (countY + 1)


def fast_fft_size(count: int) -> int:
    """generateFastFFTSize.m:11-15."""
    n = int(count)
    while True:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


class Mesh:
    """src/+rooftopMoM/Mesh.m: countX x countY faces of sizeX x sizeY in the plane z = 0."""

    def __init__(self, countX: int, countY: int, sizeX: float, sizeY: float):
        for v, name in ((countX, "countX"), (countY, "countY")):
            if int(v) != v or v < 1:
                raise _err("rooftopMoM:mesh:invalidCount", f"{name} must be a positive integer.")
        for v in (sizeX, sizeY):
            if not (math.isfinite(v) and v > 0):
                raise _err("rooftopMoM:mesh:invalidSize", "The face sizes must be positive and finite.")
        if countX == 1 and countY == 1:
            raise _err("rooftopMoM:mesh:noRooftops",
                       "A single face has no interior edge, so it carries no rooftop.")
        self._c = (int(countX), int(countY))
        self._s = (float(sizeX), float(sizeY))

    def count(self):
        return self._c

    def faceSize(self):
        return self._s

    def radius(self) -> float:
        return math.hypot(self._c[0] * self._s[0], self._c[1] * self._s[1]) / 2

    # rooftop layout (UniformRooftops.m:31-55)
    def gridSize(self, direction: str):
        cx, cy = self._c
        return (cx - 1, cy) if direction == "x" else (cx, cy - 1)

    def rooftopCount(self) -> int:
        (a, b), (c, d) = self.gridSize("x"), self.gridSize("y")
        return a * b + c * d


def _modifier_key(modifier):
    """'real' or 'imag' for a modifier given by name or as np.real / np.imag (Generators.m:25-37)."""
    if modifier is np.real or modifier == "real":
        return "real"
    if modifier is np.imag or modifier == "imag":
        return "imag"
    raise _err("rooftopMoM:operator:invalidModifier", "The modifier is 'real', 'imag' or None.")


class Generators:
    """Generators.m: the three Toeplitz generators, held on the device."""

    def __init__(self, handle, mesh: Mesh):
        self._h = handle
        self._mesh = mesh

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                L.load().rtm_generators_destroy(self._h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def modify(self, modifier):
        """Generators.modify with 'real' / 'imag' (or np.real / np.imag)."""
        key = _modifier_key(modifier)
        out = C.c_void_p()
        L.call("rtm_generators_modify", self._h, L.MODIFIERS[key], C.byref(out))
        return Generators(out, self._mesh)

    def arrays(self):
        """(magneticXX, magneticYY, electric) as numpy arrays [x, y]; None for a missing direction."""
        cx, cy = self._mesh.count()
        xx = np.zeros((cx - 1) * cy, np.complex128)
        yy = np.zeros(cx * (cy - 1), np.complex128)
        e = np.zeros(cx * cy, np.complex128)
        L.call("rtm_generators_read", self._h, xx.ctypes.data_as(C.c_void_p) if xx.size else None,
               yy.ctypes.data_as(C.c_void_p) if yy.size else None, e.ctypes.data_as(C.c_void_p), L.HOST)
        f = lambda v, r, c: v.reshape(r, c, order="F") if v.size else None
        return f(xx, cx - 1, cy), f(yy, cx, cy - 1), e.reshape(cx, cy, order="F")

    def magneticXX(self):
        return self.arrays()[0]

    def magneticYY(self):
        return self.arrays()[1]

    def electric(self):
        return self.arrays()[2]

    @staticmethod
    def fromArrays(mesh: Mesh, magneticXX, magneticYY, electric):
        """Wraps given generators (the reference's Generators constructor)."""
        cx, cy = mesh.count()
        ptr = lambda a: (np.ascontiguousarray(np.asarray(a, np.complex128).ravel(order="F"))
                         if a is not None and np.size(a) else None)
        xx, yy, e = ptr(magneticXX), ptr(magneticYY), ptr(electric)
        out = C.c_void_p()
        L.call("rtm_generators_create", cx, cy, xx.ctypes.data_as(C.c_void_p) if xx is not None else None,
               yy.ctypes.data_as(C.c_void_p) if yy is not None else None, e.ctypes.data_as(C.c_void_p), L.HOST,
               C.byref(out))
        return Generators(out, mesh)


class Problem:
    """src/+rooftopMoM/Problem.m: the EFIE of a Mesh at one wavenumber; generators assembled lazily."""

    minimumDensity = 10

    def __init__(self, mesh: Mesh, wavenumber=None, electricalSize=None, quadratureOrder=(16, 8), chunkSize=None):
        if (wavenumber is None) == (electricalSize is None):
            raise _err("rooftopMoM:problem:invalidWavenumber",
                       "A problem takes either the wavenumber or the 'electricalSize', not both or neither.")
        if wavenumber is None:
            wavenumber = electricalSize / mesh.radius()
        if not (math.isfinite(wavenumber) and wavenumber > 0):
            raise _err("rooftopMoM:problem:invalidWavenumber", "The wavenumber must be positive and finite.")
        orders = np.atleast_1d(np.asarray(quadratureOrder, dtype=np.float64))
        if orders.size not in (1, 2):
            raise _err("rooftopMoM:problem:invalidQuadratureOrder",
                       "The quadrature order is one order or a pair [near, far].")
        if not np.all((orders >= 1) & (orders == np.floor(orders))):
            raise _err("rooftopMoM:problem:invalidQuadratureOrder", "The quadrature orders are positive integers.")
        self._mesh = mesh
        self._k = float(wavenumber)
        self._orders = (int(orders[0]), int(orders[-1]))
        self._generators = None
        self._require_assembly()

    def _require_assembly(self):
        """Problem.m:77 and :210-219: the generators and the assembly's working arrays must fit below the
        memory ceiling already when the problem is made (the assembly checks the device's free memory too)."""
        ceiling, held = C.c_double(), C.c_double()
        L.call("rtm_budget_query", C.byref(ceiling), C.byref(held))
        gen, work = assembly_bytes(*self._mesh.count())
        if ceiling.value > 0 and held.value + gen + work > ceiling.value:
            raise RtmError(L.ERR_OOM_BUDGET,
                           f"The assembly of {self.rooftopCount()} rooftops (generators {format_bytes(gen)}, chunk "
                           f"{format_bytes(work)}) needs {format_bytes(gen + work)}, but only "
                           f"{format_bytes(max(0.0, ceiling.value - held.value))} of the memory ceiling of "
                           f"{format_bytes(ceiling.value)} are left.", "rooftopMoM:resources:insufficientMemory")

    @staticmethod
    def fromElectricalSize(electricalSize, density=10, aspect=1, quadratureOrder=(16, 8), chunkSize=None):
        """Problem.m:159-206: the fewest faces reaching the density, rounded up to 7-smooth counts, k = 2 pi."""
        for v, name in ((electricalSize, "electricalSize"), (density, "density"), (aspect, "aspect")):
            if not (math.isfinite(v) and v > 0):
                raise _err("rooftopMoM:problem:invalidArgument", f"The {name} must be positive and finite.")
        sides = np.array([aspect, 1.0]) * (electricalSize / math.pi) / math.hypot(aspect, 1.0)
        counts = np.maximum(1, np.ceil((1 - 4 * np.finfo(float).eps) * sides * density)).astype(int)
        counts = [fast_fft_size(c) for c in counts]
        if counts == [1, 1]:
            raise _err("rooftopMoM:problem:singleFace", "The plate is a single face, which carries no rooftop.")
        mesh = Mesh(counts[0], counts[1], sides[0] / counts[0], sides[1] / counts[1])
        return Problem(mesh, 2 * math.pi, quadratureOrder=quadratureOrder)

    def mesh(self):
        return self._mesh

    def wavenumber(self):
        return self._k

    def electricalSize(self):
        return self._k * self._mesh.radius()

    def density(self):
        return 2 * math.pi / (self._k * max(self._mesh.faceSize()))

    def rooftopCount(self):
        return self._mesh.rooftopCount()

    def quadratureOrder(self):
        return self._orders

    def generators(self) -> Generators:
        """Problem.generators: assembled on the first call, on the GPU."""
        if self._generators is None:
            cx, cy = self._mesh.count()
            a, b = self._mesh.faceSize()
            out = C.c_void_p()
            L.call("rtm_generators_assemble", cx, cy, a, b, self._k, self._orders[0], self._orders[1], None,
                   C.byref(out))
            self._generators = Generators(out, self._mesh)
        return self._generators

    def memory(self):
        """Problem.m:147-155: the bytes of the generators, zero before they are assembled."""
        if self._generators is None:
            return 0.0
        return assembly_bytes(*self._mesh.count())[0]

    def setGenerators(self, generators: Generators):
        """Uses given generators instead of assembling them (e.g. the reference's stored ones)."""
        self._generators = generators


class _Product:
    """Product.m: apply with the size check of the reference."""

    _handle = None
    _destroy = None
    _apply_fn = None

    def __del__(self):
        if self._handle:
            try:
                getattr(L.load(), self._destroy)(self._handle)
            except Exception:  # interpreter shutdown
                pass
            self._handle = None

    def apply(self, x, nrhs: int = 1):
        n = self._n
        if _is_device(x):
            total = x.numel()
        else:
            total = np.size(x)
        if total != n * nrhs:
            raise RtmError(L.ERR_SIZE, f"The input must be a numeric {n}x1 vector.", "rooftopMoM:product:sizeMismatch")
        if _is_device(x):
            import torch
            y = torch.empty_like(x)
            xp, where, keep = _vec_in(x, n)
            L.call(self._apply_fn, self._handle, xp, C.c_void_p(y.data_ptr()), n, nrhs, where, None)
            return y
        xp, where, keep = _vec_in(x, n)
        y = np.empty(n * nrhs, np.complex128)
        L.call(self._apply_fn, self._handle, xp, y.ctypes.data_as(C.c_void_p), n, nrhs, where, None)
        return y if nrhs > 1 else y.reshape(np.shape(x)) if np.ndim(x) else y

    @property
    def handle(self):
        return self._handle

    def rooftopCount(self):
        return self._n


class Operator(_Product):
    """src/+rooftopMoM/Operator.m: the matrix-free product with the Green's matrix.

    product: 'fft' | 'splitFFT' (default) | 'leanSplitFFT'; modifier: None | 'real' | 'imag';
    precision: 'double' (default) | 'single' (complex FP32 spectra and transforms).
    """

    _destroy = "rtm_operator_destroy"
    _apply_fn = "rtm_operator_apply"

    def __init__(self, problem: Problem, product="splitFFT", modifier=None, precision="double", maxRhs=1):
        if product not in L.PRODUCTS:
            raise _err("rooftopMoM:operator:invalidProduct", "The product is 'fft', 'splitFFT' or 'leanSplitFFT'.")
        if precision not in L.PRECISIONS:
            raise _err("rooftopMoM:operator:invalidPrecision", "The precision is 'double' or 'single'.")
        if modifier is not None:
            _modifier_key(modifier)
        gen = problem.generators()
        if modifier is not None:
            gen = gen.modify(modifier)
        a, b = problem.mesh().faceSize()
        out = C.c_void_p()
        L.call("rtm_operator_create", gen.handle, a, b, L.PRODUCTS[product], L.PRECISIONS[precision], int(maxRhs),
               C.byref(out))
        self._handle = out
        self._problem = problem
        self._n = problem.rooftopCount()
        self.product = product
        self.precision = precision

    def problem(self):
        return self._problem

    def info(self):
        n = C.c_int64()
        px, py = C.c_int(), C.c_int()
        sb, wb = C.c_double(), C.c_double()
        L.call("rtm_operator_info", self._handle, C.byref(n), C.byref(px), C.byref(py), C.byref(sb), C.byref(wb))
        return {"n": n.value, "fft_x": px.value, "fft_y": py.value, "spectra_bytes": sb.value,
                "working_bytes": wb.value}

    def memory(self):
        return self.info()["spectra_bytes"]

    def spectra(self):
        """The stored spectra as numpy arrays [block][x, y]."""
        cnt = C.c_int()
        L.call("rtm_operator_read_spectra", self._handle, None, C.byref(cnt))
        inf = self.info()
        P, Q = inf["fft_x"], inf["fft_y"]
        buf = np.zeros(cnt.value * P * Q, np.complex128)
        L.call("rtm_operator_read_spectra", self._handle, buf.ctypes.data_as(C.c_void_p), C.byref(cnt))
        return buf.reshape(cnt.value, Q, P).transpose(0, 2, 1)


class DenseOperator(_Product):
    """A dense complex matrix as an operator of the solvers (IterativeMethod accepts matrices)."""

    _destroy = "rtm_operator_destroy"
    _apply_fn = "rtm_operator_apply"

    def __init__(self, matrix):
        A = np.asfortranarray(np.asarray(matrix, np.complex128))
        if A.ndim != 2 or A.shape[0] != A.shape[1]:
            raise _err("rooftopMoM:solver:invalidOperator", "An operator matrix is square.")
        out = C.c_void_p()
        L.call("rtm_operator_create_dense", A.ctypes.data_as(C.c_void_p), A.shape[0], L.HOST, C.byref(out))
        self._handle = out
        self._n = A.shape[0]
        self.precision = "double"


class Preconditioner(_Product):
    """src/+rooftopMoM/Preconditioner.m: circulant preconditioner (inverse of a block-circulant approximation).

    kernel: 'strang' | 'tChan' | 'rChan' (default) | 'huckle' | 'superoptimal';
    builder: 'partwise' (default) | 'blockwise' | 'hybrid'.
    """

    _destroy = "rtm_preconditioner_destroy"
    _apply_fn = "rtm_preconditioner_apply"

    def __init__(self, problem: Problem, kernel="rChan", builder="partwise", bandwidth=None, modifier=None,
                 precision="double"):
        if kernel not in L.KERNELS:
            raise _err("rooftopMoM:preconditioner:invalidKernel",
                       "The kernel is 'strang', 'tChan', 'rChan', 'huckle' or 'superoptimal'.")
        if builder not in L.BUILDERS:
            raise _err("rooftopMoM:preconditioner:invalidBuilder", "The builder is 'partwise', 'blockwise' or 'hybrid'.")
        bw = None
        if bandwidth is not None:
            bw_values = np.asarray(bandwidth, dtype=np.float64).ravel()
            if bw_values.size != 2:
                raise _err("rooftopMoM:preconditioner:invalidBandwidth",
                           "The bandwidth is a pair [bandwidthX, bandwidthY].")
            if not np.all((bw_values >= 1) & (bw_values == np.floor(bw_values))):
                raise _err("rooftopMoM:preconditioner:invalidBandwidth", "The bandwidths are positive integers.")
            bw = (C.c_int * 2)(int(bw_values[0]), int(bw_values[1]))
        if modifier is not None:
            _modifier_key(modifier)
        gen = problem.generators()
        if modifier is not None:
            gen = gen.modify(modifier)
        a, b = problem.mesh().faceSize()
        out = C.c_void_p()
        L.call("rtm_preconditioner_create", gen.handle, a, b, L.KERNELS[kernel], L.BUILDERS[builder],
               C.cast(bw, C.c_void_p) if bw is not None else None, L.PRECISIONS[precision], C.byref(out))
        self._handle = out
        self._problem = problem
        self._n = problem.rooftopCount()
        self.precision = precision

    @classmethod
    def blockJacobi(cls, problem: Problem, block=(2, 2), precision="double"):
        """Block-Jacobi over blocks of block[0] x block[1] faces (not in the reference)."""
        self = cls.__new__(cls)
        gen = problem.generators()
        a, b = problem.mesh().faceSize()
        out = C.c_void_p()
        L.call("rtm_preconditioner_create_block_jacobi", gen.handle, a, b, int(block[0]), int(block[1]),
               L.PRECISIONS[precision], C.byref(out))
        self._handle = out
        self._problem = problem
        self._n = problem.rooftopCount()
        self.precision = precision
        return self

    def problem(self):
        return self._problem


@dataclass
class _Params:
    type: str
    data: dict


class Excitation:
    """src/+rooftopMoM/Excitation.m: plane wave or delta gap, generated on the device."""

    def __init__(self, problem, type_, vector, params):
        self._problem = problem
        self._type = type_
        self._vector = vector
        self._params = params

    @staticmethod
    def _normalize(v, name):
        v = np.asarray(v, np.float64).reshape(3)
        if not np.any(v):
            raise _err("rooftopMoM:excitation:zeroVector", f"The {name} must not be zero.")
        return v / np.linalg.norm(v)

    @classmethod
    def planeWaveVectors(cls, direction, polarization):
        """The unit direction and polarization of a plane wave (Excitation.m:52-62): both normalised, and
        perpendicular to within the rounding of a rotated frame."""
        d = cls._normalize(direction, "direction")
        p = cls._normalize(polarization, "polarization")
        dot = float(d @ p)
        if abs(dot) > 10 * np.finfo(float).eps:
            raise _err("rooftopMoM:excitation:notPerpendicular",
                       f"The polarization must be perpendicular to the direction of propagation, their dot product "
                       f"is {dot:.1e}.")
        return d, p

    @classmethod
    def planeWave(cls, problem: Problem, direction=(0, 0, -1), polarization=(1, 0, 0), intensity=1.0,
                  device=False):
        """device=True keeps the vector on the GPU (a complex128 CUDA tensor)."""
        d, p = cls.planeWaveVectors(direction, polarization)
        cx, cy = problem.mesh().count()
        a, b = problem.mesh().faceSize()
        n = problem.rooftopCount()
        inten = np.array([float(intensity)])
        if device:
            import torch
            out = torch.empty(n, dtype=torch.complex128, device="cuda")
            ptr, where = C.c_void_p(out.data_ptr()), L.DEVICE
        else:
            out = np.zeros(n, np.complex128)
            ptr, where = out.ctypes.data_as(C.c_void_p), L.HOST
        L.call("rtm_plane_wave", cx, cy, a, b, problem.quadratureOrder()[1], problem.wavenumber(),
               d.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p), inten.ctypes.data_as(C.c_void_p), 1,
               ptr, where, None)
        return cls(problem, "planeWave", out, {"direction": d, "polarization": p, "intensity": float(intensity)})

    @classmethod
    def deltaGap(cls, problem: Problem, port=None, direction="x", voltage=1.0):
        """port: 0-based rooftop indices (default: the middle line of edges of the direction)."""
        cx, cy = problem.mesh().count()
        a, b = problem.mesh().faceSize()
        n = problem.rooftopCount()
        out = np.zeros(n, np.complex128)
        if port is None:
            if problem.mesh().gridSize(direction)[0] * problem.mesh().gridSize(direction)[1] == 0:
                raise _err("rooftopMoM:excitation:noRooftops", f"The mesh has no {direction}-directed rooftops.")
            pp = None
            cnt = 0
        else:
            pp = np.ascontiguousarray(np.asarray(port, np.int64).ravel())
            if np.any(pp >= n) or np.any(pp < 0) or np.unique(pp).size < pp.size:
                raise _err("rooftopMoM:excitation:invalidPort",
                           f"The port must hold distinct rooftop indices up to {n}.")
            cnt = pp.size
        L.call("rtm_delta_gap", cx, cy, a, b, pp.ctypes.data_as(C.c_void_p) if pp is not None else None, cnt,
               0 if direction == "x" else 1, float(voltage), out.ctypes.data_as(C.c_void_p), L.HOST)
        if port is None:
            pp = np.flatnonzero(out)
        return cls(problem, "deltaGap", out, {"port": pp, "voltage": float(voltage)})

    def problem(self):
        return self._problem

    def type(self):
        return self._type

    def vector(self):
        return self._vector

    def parameters(self):
        return self._params


class Result:
    """src/+rooftopMoM/Result.m."""

    def __init__(self, solution, stats, history, excitation=None, inner_iterations=None):
        self._x = solution
        self._stats = stats
        self._history = history
        self._excitation = excitation

    def solution(self):
        return self._x

    def converged(self):
        return bool(self._stats.converged)

    def iterationCount(self):
        return int(self._stats.iteration_count)

    def residualNorms(self):
        h = self._history
        return h[: np.count_nonzero(~np.isnan(h))]

    def residualNorm(self):
        return float(self._stats.residual_norm)

    def time(self):
        return float(self._stats.time_s)

    def refinements(self):
        return int(self._stats.refinements)

    def excitation(self):
        return self._excitation

    def _parameters(self, type_):
        if self._excitation is None or self._excitation.type() != type_:
            raise _err("rooftopMoM:result:wrongExcitation", f"This quantity needs a {type_} excitation.")
        return self._excitation.parameters()

    def inputImpedance(self):
        p = self._parameters("deltaGap")
        prob = self._excitation.problem()
        cx, cy = prob.mesh().count()
        a, b = prob.mesh().faceSize()
        xp, where, keep = _vec_in(self._x, prob.rooftopCount())
        port = np.ascontiguousarray(np.asarray(p["port"], np.int64))
        out = (C.c_double * 2)()
        L.call("rtm_input_impedance", cx, cy, a, b, xp, port.ctypes.data_as(C.c_void_p), port.size, p["voltage"],
               where, out)
        return complex(out[0], out[1])

    def radarCrossSection(self):
        p = self._parameters("planeWave")
        prob = self._excitation.problem()
        ev = self._excitation.vector()
        if _is_device(self._x) and not _is_device(ev):
            import torch
            ev = torch.from_numpy(np.ascontiguousarray(ev)).to(self._x.device)
        elif not _is_device(self._x) and _is_device(ev):
            ev = ev.cpu().numpy()
        ep, where, keep1 = _vec_in(ev, prob.rooftopCount())
        xp, where2, keep2 = _vec_in(self._x, prob.rooftopCount())
        out = C.c_double()
        L.call("rtm_radar_cross_section", prob.wavenumber(), ep, xp, prob.rooftopCount(), p["intensity"], where,
               C.byref(out))
        return out.value

    def bistaticRadarCrossSection(self, directions, polarizations):
        """Bistatic RCS (m^2) of the current for observation directions r (unit vectors from the plate to the
        observer) and receive polarisations p (perpendicular to r): (k Z0)^2 |e_r^T J|^2 / (4 pi I^2), with
        e_r the unit plane wave travelling along -r with polarisation p and I the incident intensity.
        At r = -d, p = the incident polarisation it is the monostatic radarCrossSection
        (computeRadarCrossSection.m:18-19); the reference's current code has no bistatic form (its
        obsolete v1 had a far-field pattern), so this one rests on that identity and on reciprocity."""
        p_inc = self._parameters("planeWave")
        prob = self._excitation.problem()
        dirs = np.atleast_2d(np.asarray(directions, dtype=np.float64))
        pols = np.atleast_2d(np.asarray(polarizations, dtype=np.float64))
        if dirs.shape != pols.shape or dirs.shape[1] != 3:
            raise _err("rooftopMoM:result:invalidDirections", "Directions and polarizations are matching 3-vectors.")
        device = _is_device(self._x)
        xp, where, keep = _vec_in(self._x, prob.rooftopCount())
        # intensity' = sqrt(I): the ABI divides by intensity'^4 = I^2 for a unit receive wave
        scale = math.sqrt(p_inc["intensity"])
        out = np.empty(len(dirs))
        for i, (r, p) in enumerate(zip(dirs, pols)):
            e = Excitation.planeWave(prob, direction=-r, polarization=p, device=device).vector()
            ep, _, keep_e = _vec_in(e, prob.rooftopCount())
            v = C.c_double()
            L.call("rtm_radar_cross_section", prob.wavenumber(), ep, xp, prob.rooftopCount(), scale, where,
                   C.byref(v))
            out[i] = v.value
        return out

    def normalizedRadarCrossSection(self):
        wavelength = 2 * math.pi / self._excitation.problem().wavenumber()
        return self.radarCrossSection() / wavelength**2


def _require_finite_rhs(b):
    """Solver.m:162-168: a right-hand side is numeric (which logical arrays are not) and finite."""
    if _is_device(b):
        return
    try:
        a = np.asarray(b)
        finite = a.dtype.kind in "iufc" and bool(np.all(np.isfinite(a)))
    except (TypeError, ValueError):
        finite = False
    if not finite:
        raise _err("rooftopMoM:solver:invalidRightHandSide",
                   "The right-hand side is a rooftopMoM.Excitation or a numeric vector of finite values.")


class Solver:
    """src/+rooftopMoM/Solver.m: 'cg' (COCG) or 'gmres' (restarted GMRES), plus the GPU-only
    precision form 'fgmres' (FP32 flexible GMRES inside FP64 iterative refinement)."""

    def __init__(self, method="cg", tolerance=1e-6, maxIterationCount=1000, restart=50, innerTolerance=1e-4,
                 maxRefinements=20, checkEvery=0, innerMethod="fgmres", side="left", gramSchmidtPasses=0):
        if method not in ("cg", "gmres", "fgmres"):
            raise _err("rooftopMoM:solver:invalidMethod", "The method is 'cg', 'gmres' or 'fgmres'.")
        if not (0 < tolerance < 1):
            raise _err("rooftopMoM:solver:invalidTolerance", "The tolerance lies in (0, 1).")
        if int(maxIterationCount) != maxIterationCount or maxIterationCount < 1:
            raise _err("rooftopMoM:solver:invalidMaxIterationCount", "maxIterationCount is a positive integer.")
        if not (restart == math.inf or (int(restart) == restart and restart > 0)):
            raise _err("rooftopMoM:solver:invalidRestart", "The restart is a positive integer or Inf.")
        self.method = method
        self.tolerance = float(tolerance)
        self.maxIterationCount = int(maxIterationCount)
        self.restart = int(min(restart, 1 << 30))
        self.innerTolerance = innerTolerance
        self.maxRefinements = maxRefinements
        self.checkEvery = checkEvery
        self.innerMethod = innerMethod
        if side not in ("left", "right"):
            raise _err("rooftopMoM:solver:invalidSide", "The preconditioning side is 'left' or 'right'.")
        self.side = side
        if gramSchmidtPasses not in (0, 1, 2):
            raise _err("rooftopMoM:solver:invalidGramSchmidtPasses",
                       "gramSchmidtPasses is 0 (the method's default), 1 or 2.")
        self.gramSchmidtPasses = int(gramSchmidtPasses)

    def solveBatch(self, batch: "PlateBatch", rightHandSides, initialGuesses=None):
        """Solves every entry of a PlateBatch (its operator and preconditioner) for its right-hand side, all
        entries at once, each to this solver's tolerance; 'cg' or 'gmres'. Returns one Result per entry."""
        if self.method not in ("cg", "gmres"):
            raise _err("rooftopMoM:solver:invalidMethod", "A plate batch solves by 'cg' or 'gmres'.")
        excitations = [v if isinstance(v, Excitation) else None for v in rightHandSides]
        vectors = [v.vector() if isinstance(v, Excitation) else v for v in rightHandSides]
        for v, e in zip(vectors, excitations):
            if e is None:
                _require_finite_rhs(v)
        device = _is_device(vectors[0])
        b = batch._pack(vectors, device)
        x0 = batch._pack(initialGuesses, device) if initialGuesses is not None else None
        count = batch.count()
        hist = np.full((count, self.maxIterationCount + 1), np.nan)
        stats = (L.SolveStats * count)()
        cfg = self._config(L.METHODS[self.method])
        if device:
            import torch
            x = torch.empty_like(b)
            ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
            L.call("rtm_plate_batch_solve", batch._handle, C.byref(cfg), ptr(b), ptr(x0), ptr(x), L.DEVICE,
                   hist.ctypes.data_as(C.c_void_p), stats, None)
        else:
            x = np.empty_like(b)
            ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None  # noqa: E731
            L.call("rtm_plate_batch_solve", batch._handle, C.byref(cfg), ptr(b), ptr(x0), ptr(x), L.HOST,
                   hist.ctypes.data_as(C.c_void_p), stats, None)
        return [Result(xk, stats[k], hist[k], excitations[k]) for k, xk in enumerate(batch._unpack(x))]

    def _config(self, method_id):
        return L.SolveConfig(method_id, self.tolerance, self.maxIterationCount, self.restart, self.innerTolerance,
                             self.maxRefinements, self.checkEvery, int(self.side == "right"),
                             self.gramSchmidtPasses)

    def solve(self, operator, rightHandSide, preconditioner=None, initialGuess=None, innerOperator=None,
              innerPreconditioner=None, nrhs: int = 1):
        excitation = None
        if isinstance(rightHandSide, Excitation):
            excitation = rightHandSide
            b = rightHandSide.vector()
        else:
            b = rightHandSide
            _require_finite_rhs(b)
        if initialGuess is not None and not _is_device(initialGuess):
            # Solver.m:62: mustBeNumeric (which rejects logical arrays) and mustBeFinite
            try:
                g = np.asarray(initialGuess)
                finite = g.dtype.kind in "iufc" and bool(np.all(np.isfinite(g)))
            except (TypeError, ValueError):
                finite = False
            if not finite:
                raise _err("rooftopMoM:solver:invalidInitialGuess", "The initial guess is a numeric vector of finite "
                                                                     "values.")
        if not isinstance(operator, (np.ndarray, _Product)):
            raise _err("rooftopMoM:solver:invalidOperator",
                       "The operator is a rooftopMoM.Operator, a DenseOperator or a numeric matrix.")
        if isinstance(operator, np.ndarray):
            operator = DenseOperator(operator)
        if isinstance(preconditioner, np.ndarray):
            preconditioner = DenseOperator(preconditioner)
        count = (b.numel() if _is_device(b) else np.size(b)) // nrhs
        if operator.rooftopCount() != count:
            raise RtmError(L.ERR_SIZE, f"The operator does not match the {count} unknowns of the right-hand side.",
                           "rooftopMoM:solver:sizeMismatch")
        if preconditioner is not None and preconditioner.rooftopCount() != count:
            raise RtmError(L.ERR_SIZE,
                           f"The preconditioner does not match the {count} unknowns of the right-hand side.",
                           "rooftopMoM:solver:sizeMismatch")
        if initialGuess is not None and np.size(initialGuess) != count * nrhs and not _is_device(initialGuess):
            raise RtmError(L.ERR_SIZE, f"The initial guess must have {count} elements.", "rooftopMoM:solver:sizeMismatch")
        device = _is_device(b)
        single = getattr(operator, "precision", "double") == "single"
        dt = np.complex64 if (single and device) else np.complex128
        bp, where, keep_b = _vec_in(b, count, dt)
        x0p = None
        keep_x0 = None
        if initialGuess is not None:
            x0p, _, keep_x0 = _vec_in(initialGuess, count, dt)
        if device:
            import torch
            x = torch.empty_like(b)
            xp = C.c_void_p(x.data_ptr())
        else:
            x = np.empty(count * nrhs, np.complex128)
            xp = x.ctypes.data_as(C.c_void_p)
        hist = np.full((nrhs, self.maxIterationCount + 1), np.nan)
        stats = (L.SolveStats * nrhs)()
        if self.method == "fgmres" or innerOperator is not None:
            method_id = L.METHODS["cg"] if self.innerMethod == "cg" else L.METHODS["fgmres"]
            if innerOperator is None:
                raise _err("rooftopMoM:solver:missingInnerOperator", "The precision form needs an FP32 operator.")
            cfg = self._config(method_id)
            L.call("rtm_solve_mixed", operator.handle, innerOperator.handle,
                   innerPreconditioner.handle if innerPreconditioner is not None else None, C.byref(cfg), bp, x0p, xp,
                   count, nrhs, where, hist.ctypes.data_as(C.c_void_p), stats, None)
        else:
            cfg = self._config(L.METHODS[self.method])
            L.call("rtm_solve", operator.handle, preconditioner.handle if preconditioner is not None else None,
                   C.byref(cfg), bp, x0p, xp, count, nrhs, where, hist.ctypes.data_as(C.c_void_p), stats, None)
        if nrhs == 1:
            return Result(x, stats[0], hist[0], excitation)
        return [Result(x[k * count:(k + 1) * count], stats[k], hist[k], excitation) for k in range(nrhs)]


def tuneProduct(mesh: Mesh, precision="double", nrhs: int = 1, flushL2: bool = True, referenceSizes: bool = False,
                verbose: bool = False):
    """Autotunes the split product of a plate (rtm_tune_product): measures the candidate transform grids (the
    reference's 7-smooth sizes, generateFastFFTSize.m, and the next powers of two) and kernel schedules on the
    device and keeps the fastest for the operators created afterwards for this face grid and precision.
    Returns the choice and its time beside the reference sizes' time."""
    if precision not in L.PRECISIONS:
        raise _err("rooftopMoM:operator:invalidPrecision", "The precision is 'double' or 'single'.")
    cx, cy = mesh.count()
    out = L.TuneResult()
    flags = ((L.TUNE_FLUSH_L2 if flushL2 else 0) | (L.TUNE_REFERENCE_SIZES if referenceSizes else 0)
             | (L.TUNE_VERBOSE if verbose else 0))
    L.call("rtm_tune_product", cx, cy, L.PRECISIONS[precision], int(nrhs), flags, C.byref(out))
    return {"fftSize": (out.fft_x, out.fft_y), "yBlocks": out.y_blocks, "mixKind": out.mix_kind,
            "seconds": out.seconds, "referenceSeconds": out.reference_seconds, "candidates": out.candidates}


def clearTuning():
    """Forgets every autotuner choice (rtm_tune_clear)."""
    L.call("rtm_tune_clear")


def setTransformSize(mesh: Mesh, fftSize, precision="double"):
    """Records fftSize = (P, Q), at least the face counts, as the transform grid of the split products built
    afterwards for this plate's face grid and precision (rtm_tune_set): e.g. powers of two for plates that
    go into one PlateBatch."""
    if precision not in L.PRECISIONS:
        raise _err("rooftopMoM:operator:invalidPrecision", "The precision is 'double' or 'single'.")
    cx, cy = mesh.count()
    L.call("rtm_tune_set", cx, cy, L.PRECISIONS[precision], int(fftSize[0]), int(fftSize[1]))


class PlateBatch:
    """Plates of uneven size solved together (rtm_plate_batch_*; not in the reference): entry k is one
    right-hand side on the plate of operators[k] (an entry may repeat a plate's operator for another
    right-hand side), with preconditioners[k] if given. Split products that share their transform grid
    on the power-of-two path run as one launch of each kernel for the whole batch (fused()); vectors are
    the entries' own vectors, which solve() pads to the batch's stride and crops again."""

    def __init__(self, operators, preconditioners=None):
        self._ops = list(operators)
        self._pcs = list(preconditioners) if preconditioners is not None else None
        if not self._ops:
            raise _err("rooftopMoM:batch:empty", "A plate batch holds at least one entry.")
        if self._pcs is not None and len(self._pcs) != len(self._ops):
            raise _err("rooftopMoM:batch:sizeMismatch", "One preconditioner per entry.")
        count = len(self._ops)
        ops = (C.c_void_p * count)(*[o.handle for o in self._ops])
        pcs = (C.c_void_p * count)(*[p.handle for p in self._pcs]) if self._pcs is not None else None
        out = C.c_void_p()
        L.call("rtm_plate_batch_create", ops, pcs, count, C.byref(out))
        self._handle = out
        stride, n, fused, fused_pc = C.c_int64(), C.c_int(), C.c_int(), C.c_int()
        L.call("rtm_plate_batch_info", out, C.byref(stride), C.byref(n), C.byref(fused), C.byref(fused_pc))
        self._stride, self._fused, self._fused_pc = stride.value, bool(fused.value), bool(fused_pc.value)
        self._counts = [o.rooftopCount() for o in self._ops]
        self.precision = getattr(self._ops[0], "precision", "double")

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                L.load().rtm_plate_batch_destroy(self._handle)
            except Exception:  # interpreter shutdown
                pass
            self._handle = None

    def count(self):
        return len(self._ops)

    def stride(self):
        return self._stride

    def fused(self):
        return self._fused

    def fusedPreconditioner(self):
        return self._fused_pc

    def rooftopCounts(self):
        return list(self._counts)

    def _pack(self, vectors, device):
        if len(vectors) != len(self._ops):
            raise _err("rooftopMoM:batch:sizeMismatch", f"The batch takes {len(self._ops)} vectors.")
        for v, n in zip(vectors, self._counts):
            if (v.numel() if _is_device(v) else np.size(v)) != n:
                raise RtmError(L.ERR_SIZE, f"The input must be a numeric {n}x1 vector.",
                               "rooftopMoM:product:sizeMismatch")
        if device:
            import torch
            dt = torch.complex64 if self.precision == "single" else torch.complex128
            out = torch.zeros(len(vectors) * self._stride, dtype=dt, device=vectors[0].device)
            for k, v in enumerate(vectors):
                out[k * self._stride:k * self._stride + self._counts[k]] = v.reshape(-1).to(dt)
            return out
        out = np.zeros(len(vectors) * self._stride, np.complex128)
        for k, v in enumerate(vectors):
            out[k * self._stride:k * self._stride + self._counts[k]] = np.asarray(v, np.complex128).reshape(-1)
        return out

    def _unpack(self, packed):
        return [packed[k * self._stride:k * self._stride + n] for k, n in enumerate(self._counts)]

    def _apply(self, vectors, which):
        device = _is_device(vectors[0])
        x = self._pack(vectors, device)
        if device:
            import torch
            y = torch.empty_like(x)
            L.call("rtm_plate_batch_apply", self._handle, which, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                   L.DEVICE, None)
        else:
            y = np.empty_like(x)
            L.call("rtm_plate_batch_apply", self._handle, which, x.ctypes.data_as(C.c_void_p),
                   y.ctypes.data_as(C.c_void_p), L.HOST, None)
        return self._unpack(y)

    def apply(self, vectors):
        """y_k = A_k x_k for every entry."""
        return self._apply(vectors, 0)

    def precondition(self, vectors):
        """y_k = M_k x_k for every entry (a batch made with preconditioners)."""
        return self._apply(vectors, 1)


class Resources:
    """src/+rooftopMoM/Resources.m for device memory: the HBM ceiling and the byte models."""

    @staticmethod
    def configure(memory=math.inf):
        L.call("rtm_budget_configure", 0.0 if memory == math.inf else float(memory))

    @staticmethod
    def reset():
        Resources.configure()

    @staticmethod
    def ceiling():
        c, h = C.c_double(), C.c_double()
        L.call("rtm_budget_query", C.byref(c), C.byref(h))
        return math.inf if c.value <= 0 else c.value

    @staticmethod
    def held():
        c, h = C.c_double(), C.c_double()
        L.call("rtm_budget_query", C.byref(c), C.byref(h))
        return h.value

    @staticmethod
    def check(mesh: Mesh, product="splitFFT", preconditioner=True, method="cg", restart=50, maxIterationCount=1000):
        """Resources.check (Resources.m:73-141) for device memory: the bytes of a planned run, estimated before
        anything is built, and rooftopMoM:resources:insufficientMemory if its peak does not fit below the
        ceiling or into the device's free memory. The assembly's working memory ("chunk") is that of the
        device assembly: 28 quadrant sums per far-lattice block and 7 moment terms per face pair offset."""
        est = Resources.estimate(mesh, product, method, preconditioner, restart, maxIterationCount)
        cx, cy = mesh.count()
        report = {"generators": est["generators"],
                  "chunk": 16.0 * (28 * (cx + 1) * (cy + 1) + 7 * cx * cy),
                  "product": est["product"], "productWorking": est["productWorking"],
                  "preconditioner": est["preconditioner"] if preconditioner else 0.0,
                  "preconditionerWorking": est["preconditionerWorking"] if preconditioner else 0.0,
                  "solver": est["solver"]}
        # the assembly and the solve do not overlap; within the solve one product runs at a time
        report["peak"] = max(report["generators"] + report["chunk"],
                             report["generators"] + report["product"] + report["preconditioner"]
                             + max(report["productWorking"], report["preconditionerWorking"]) + report["solver"])
        L.call("rtm_budget_require", float(report["peak"]), identifier="rooftopMoM:resources:insufficientMemory")
        return report

    @staticmethod
    def estimate(mesh: Mesh, product="splitFFT", method="cg", preconditioner=True, restart=50, maxIterationCount=1000):
        out = (C.c_double * 6)()
        cx, cy = mesh.count()
        L.call("rtm_estimate_bytes", cx, cy, L.PRODUCTS[product], L.METHODS[method], int(bool(preconditioner)),
               int(restart), int(maxIterationCount), out)
        keys = ("generators", "product", "productWorking", "preconditioner", "preconditionerWorking", "solver")
        return dict(zip(keys, list(out)))
