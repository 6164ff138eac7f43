"""rooftop-mom on B200: the Green's-matrix assembly, FFT / split-FFT products and COCG / GMRES
solvers of rooftop-mom (MATLAB package +rooftopMoM, 3.5.0) as hand-written sm_100a kernels in
librtm.so, behind a C ABI (include/rtm.h) and this Python mirror of the MATLAB API."""
from ._lib import RtmError, load  # noqa: F401
from .api import (  # noqa: F401
    DenseOperator,
    Excitation,
    Generators,
    Mesh,
    Operator,
    PlateBatch,
    Preconditioner,
    Problem,
    Resources,
    Result,
    Solver,
    clearTuning,
    fast_fft_size,
    setTransformSize,
    tuneProduct,
)
from .server import Request, Server  # noqa: F401

__version__ = "3.5.0"
