"""ctypes binding of librtm.so (the C ABI declared in include/rtm.h).

Loading needs no GPU; every compute call does. There is no CPU fallback: if the library is missing
or a call fails, an RtmError is raised.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RTM_LIBRARY", os.path.join(HERE, "librtm.so"))

OK, ERR_ARG, ERR_SIZE, ERR_OOM_BUDGET, ERR_CUDA, ERR_TIMEOUT, ERR_SINGULAR, ERR_UNSUPPORTED = range(8)
XONLY, YONLY, BOTH = 1, 2, 3
PRODUCTS = {"fft": 0, "splitFFT": 1, "leanSplitFFT": 2}
PRECISIONS = {"double": 0, "single": 1}
HOST, DEVICE = 0, 1
MODIFIERS = {None: 0, "real": 1, "imag": 2}
KERNELS = {"strang": 0, "tChan": 1, "rChan": 2, "huckle": 3, "superoptimal": 4}
BUILDERS = {"partwise": 0, "blockwise": 1, "hybrid": 2}
METHODS = {"cg": 0, "gmres": 1, "fgmres": 2}

# Error identifiers of the reference (src/+rooftopMoM/*.m) for the statuses that have one.
_IDS = {
    ERR_ARG: "rooftopMoM:gpu:invalidArgument",
    ERR_SIZE: "rooftopMoM:product:sizeMismatch",
    ERR_OOM_BUDGET: "rooftopMoM:resources:insufficientMemory",
    ERR_CUDA: "rooftopMoM:gpu:cuda",
    ERR_TIMEOUT: "rooftopMoM:gpu:timeout",
    ERR_SINGULAR: "rooftopMoM:preconditioner:singular",
    ERR_UNSUPPORTED: "rooftopMoM:gpu:unsupported",
}


class RtmError(RuntimeError):
    """A failed librtm call; ``identifier`` follows the reference's error IDs."""

    def __init__(self, status: int, message: str, identifier: str | None = None):
        self.status = status
        self.identifier = identifier or _IDS.get(status, "rooftopMoM:gpu:error")
        super().__init__(f"{self.identifier}: {message}")


class SolveConfig(C.Structure):
    _fields_ = [("method", C.c_int), ("tolerance", C.c_double), ("max_iterations", C.c_int),
                ("restart", C.c_int), ("inner_tolerance", C.c_double), ("max_refinements", C.c_int),
                ("check_every", C.c_int), ("right_preconditioned", C.c_int), ("gram_schmidt_passes", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("iteration_count", C.c_int), ("residual_norm", C.c_double),
                ("time_s", C.c_double), ("refinements", C.c_int), ("matvecs", C.c_int)]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
class TuneResult(C.Structure):
    _fields_ = [("fft_x", C.c_int), ("fft_y", C.c_int), ("y_blocks", C.c_int), ("mix_kind", C.c_int),
                ("seconds", C.c_double), ("reference_seconds", C.c_double), ("candidates", C.c_int)]


TUNE_FLUSH_L2 = 1
TUNE_REFERENCE_SIZES = 2
TUNE_VERBOSE = 4
TRANSFORM_SIZES = {"reference": 0, "powerOfTwo": 1, "autotune": 2}


class ServerConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_double), ("max_active", C.c_int), ("precision", C.c_int), ("device", C.c_int),
                ("transform_sizes", C.c_int), ("max_batch", C.c_int)]


class Request(C.Structure):
    _fields_ = [("count_x", C.c_int), ("count_y", C.c_int), ("size_x", C.c_double), ("size_y", C.c_double),
                ("wavenumber", C.c_double), ("excitation", C.c_int), ("direction", C.c_double * 3),
                ("polarization", C.c_double * 3), ("port_direction", C.c_int), ("voltage", C.c_double),
                ("method", C.c_int), ("preconditioner", C.c_int), ("tolerance", C.c_double),
                ("max_iterations", C.c_int), ("restart", C.c_int), ("keep_current", C.c_int)]


class RequestResult(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("converged", C.c_int), ("iteration_count", C.c_int),
                ("residual_norm", C.c_double), ("rcs", C.c_double), ("impedance", C.c_double * 2),
                ("unknowns", C.c_int64), ("bytes", C.c_double), ("submitted_s", C.c_double),
                ("started_s", C.c_double), ("finished_s", C.c_double), ("solve_s", C.c_double)]


EXCITATIONS = {"planeWave": 0, "deltaGap": 1}
STATES = ("queued", "running", "done", "failed", "cancelled")

_SIGNATURES = {
    "rtm_version": [C.POINTER(C.c_int)] * 3,
    "rtm_last_error": [C.c_char_p, C.c_size_t],
    "rtm_set_device": [C.c_int],
    "rtm_launch_count": [C.POINTER(C.c_int64)],
    "rtm_budget_configure": [C.c_double],
    "rtm_budget_query": [C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "rtm_budget_require": [C.c_double],
    "rtm_estimate_bytes": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)],
    "rtm_generators_assemble": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _P, _PP],
    "rtm_generators_create": [C.c_int, C.c_int, _P, _P, _P, C.c_int, _PP],
    "rtm_generators_modify": [_P, C.c_int, _PP],
    "rtm_generators_read": [_P, _P, _P, _P, C.c_int],
    "rtm_generators_info": [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "rtm_generators_destroy": [_P],
    "rtm_operator_create": [_P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _PP],
    "rtm_operator_apply": [_P, _P, _P, C.c_int64, C.c_int, C.c_int, _P],
    "rtm_operator_apply_fixed_scratch": [_P, _P, _P, C.c_int64, C.c_int, _P],
    "rtm_fixed_scratch_bytes": [_P],
    "rtm_tune_product": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(TuneResult)],
    "rtm_tune_clear": [],
    "rtm_tune_set": [C.c_int] * 5,
    "rtm_plate_batch_create": [_PP, _PP, C.c_int, _PP],
    "rtm_plate_batch_info": [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "rtm_plate_batch_apply": [_P, C.c_int, _P, _P, C.c_int, _P],
    "rtm_plate_batch_solve": [_P, C.POINTER(SolveConfig), _P, _P, _P, C.c_int, _P, C.POINTER(SolveStats), _P],
    "rtm_plate_batch_destroy": [_P],
    "rtm_operator_create_dense": [_P, C.c_int64, C.c_int, _PP],
    "rtm_operator_info": [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                          C.POINTER(C.c_double)],
    "rtm_operator_read_spectra": [_P, _P, C.POINTER(C.c_int)],
    "rtm_operator_destroy": [_P],
    "rtm_preconditioner_create": [_P, C.c_double, C.c_double, C.c_int, C.c_int, _P, C.c_int, _PP],
    "rtm_preconditioner_create_block_jacobi": [_P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _PP],
    "rtm_preconditioner_apply": [_P, _P, _P, C.c_int64, C.c_int, C.c_int, _P],
    "rtm_preconditioner_destroy": [_P],
    "rtm_solve": [_P, _P, C.POINTER(SolveConfig), _P, _P, _P, C.c_int64, C.c_int, C.c_int, _P, C.POINTER(SolveStats),
                  _P],
    "rtm_solve_mixed": [_P, _P, _P, C.POINTER(SolveConfig), _P, _P, _P, C.c_int64, C.c_int, C.c_int, _P,
                        C.POINTER(SolveStats), _P],
    "rtm_plane_wave": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, _P, _P, _P, C.c_int, _P,
                       C.c_int, _P],
    "rtm_delta_gap": [C.c_int, C.c_int, C.c_double, C.c_double, _P, C.c_int, C.c_int, C.c_double, _P, C.c_int],
    "rtm_radar_cross_section": [C.c_double, _P, _P, C.c_int64, C.c_double, C.c_int, C.POINTER(C.c_double)],
    "rtm_input_impedance": [C.c_int, C.c_int, C.c_double, C.c_double, _P, _P, C.c_int, C.c_double, C.c_int,
                            C.POINTER(C.c_double)],
    "rtm_server_create": [C.POINTER(ServerConfig), _PP],
    "rtm_server_submit": [_P, C.POINTER(Request), C.POINTER(C.c_uint64)],
    "rtm_server_poll": [_P, C.c_uint64, C.c_int, C.POINTER(RequestResult), _P, C.c_int64, C.c_int],
    "rtm_server_cancel": [_P, C.c_uint64],
    "rtm_server_destroy": [_P],
}

_lock = threading.Lock()
_lib = None


def load():
    """Returns the loaded library; raises RtmError if librtm.so is absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RtmError(ERR_UNSUPPORTED, f"{LIB_PATH} is missing; build it with "
                                                "`python -m rooftop_mom_b200.build` (no CPU fallback exists)")
            lib = C.CDLL(LIB_PATH)
            for name, args in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = C.c_int
            _lib = lib
        return _lib


def exported_symbols():
    return list(_SIGNATURES)


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    load().rtm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, identifier: str | None = None):
    if status != OK:
        raise RtmError(status, last_error(), identifier)


def call(name: str, *args, identifier: str | None = None):
    check(getattr(load(), name)(*args), identifier)


def launch_count() -> int:
    v = C.c_int64()
    call("rtm_launch_count", C.byref(v))
    return v.value
