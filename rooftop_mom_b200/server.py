"""The serving form over the C ABI (include/rtm.h, rtm_server_*): a request loop of plate solves
admitted by device bytes, with their work overlapping on the device.

    srv = Server(budgetBytes=150e9, maxActive=8, precision="double")
    rid = srv.submit(Request.planeWave(countX, countY, sizeX, sizeY, wavenumber, direction, polarization))
    result = srv.wait(rid)            # dict: state, iterations, residual, rcs / impedance, times
    srv.close()

The reference has no serving loop; its closest analogue is the admission check of its memory ledger
(src/+rooftopMoM/+resources/Budget.m:82-106) on the byte models estimate*.m.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L


PRECONDITIONERS = {None: 0, "blockJacobi": 1, "rChan": 2}


class Request:
    """One plate solve: grid, frequency, excitation and solver settings (rtm_request). preconditioner:
    None, "blockJacobi" (2 x 2 faces) or "rChan" (the reference's default circulant)."""

    def __init__(self, countX, countY, sizeX, sizeY, wavenumber, excitation="planeWave", direction=(0, 0, -1),
                 polarization=(1, 0, 0), portDirection="x", voltage=1.0, method="gmres", preconditioner="blockJacobi",
                 tolerance=1e-6, maxIterationCount=10000, restart=50, keepCurrent=False):
        if excitation == "planeWave":
            from .api import Excitation

            # normalised and checked as Excitation.planeWave does, so a request and a direct solve of the same
            # wave see the same vectors
            direction, polarization = Excitation.planeWaveVectors(direction, polarization)
        r = L.Request()
        r.count_x, r.count_y = int(countX), int(countY)
        r.size_x, r.size_y, r.wavenumber = float(sizeX), float(sizeY), float(wavenumber)
        r.excitation = L.EXCITATIONS[excitation]
        r.direction[:] = [float(v) for v in direction]
        r.polarization[:] = [float(v) for v in polarization]
        r.port_direction = {"x": 0, "y": 1}[portDirection]
        r.voltage = float(voltage)
        r.method = L.METHODS[method]
        r.preconditioner = PRECONDITIONERS[preconditioner]
        r.tolerance = float(tolerance)
        r.max_iterations = int(maxIterationCount)
        r.restart = int(restart)
        r.keep_current = int(bool(keepCurrent))
        self.struct = r

    @classmethod
    def planeWave(cls, countX, countY, sizeX, sizeY, wavenumber, direction, polarization, **kw):
        return cls(countX, countY, sizeX, sizeY, wavenumber, "planeWave", direction=direction,
                   polarization=polarization, **kw)

    @classmethod
    def deltaGap(cls, countX, countY, sizeX, sizeY, wavenumber, portDirection="x", voltage=1.0, **kw):
        return cls(countX, countY, sizeX, sizeY, wavenumber, "deltaGap", portDirection=portDirection,
                   voltage=voltage, **kw)

    def unknowns(self):
        r = self.struct
        return (r.count_x - 1) * r.count_y + r.count_x * (r.count_y - 1)


def _result_dict(res: L.RequestResult):
    return {
        "state": L.STATES[res.state], "status": res.status, "converged": bool(res.converged),
        "iterations": res.iteration_count, "residual": res.residual_norm, "rcs": res.rcs,
        "impedance": complex(res.impedance[0], res.impedance[1]), "unknowns": res.unknowns, "bytes": res.bytes,
        "submitted": res.submitted_s, "started": res.started_s, "finished": res.finished_s,
        "latency": res.finished_s - res.submitted_s, "solveTime": res.solve_s,
    }


class Server:
    """rtm_server: admission by byte budget, maxActive requests on the device at once."""

    def __init__(self, budgetBytes=150e9, maxActive=8, precision="double", device=0, transformSizes="reference",
                 maxBatch=0):
        """transformSizes: "reference" (generateFastFFTSize.m's 7-smooth sizes), "powerOfTwo" (plates: the next
        powers of two where the power-of-two kernels take them) or "autotune" (plates: rtm_tune_product on the
        first request of each face grid). maxBatch > 1 (FP64, "powerOfTwo"): maxActive / maxBatch workers, each
        solving up to maxBatch admitted requests of one transform grid and solver setting as one plate batch."""
        if transformSizes not in L.TRANSFORM_SIZES:
            raise L.RtmError(L.ERR_ARG, "transformSizes is 'reference', 'powerOfTwo' or 'autotune'.",
                             "rooftopMoM:gpu:invalidArgument")
        cfg = L.ServerConfig(float(budgetBytes), int(maxActive), L.PRECISIONS[precision], int(device),
                             L.TRANSFORM_SIZES[transformSizes], int(maxBatch))
        h = C.c_void_p()
        L.call("rtm_server_create", C.byref(cfg), C.byref(h))
        self._h = h
        self._keep = {}

    def submit(self, request: Request) -> int:
        rid = C.c_uint64()
        L.call("rtm_server_submit", self._h, C.byref(request.struct), C.byref(rid))
        if request.struct.keep_current:
            self._keep[rid.value] = request.unknowns()
        return rid.value

    def poll(self, rid: int, wait=0.0, release=False):
        """The request's state and result; waits up to `wait` seconds (math.inf: until it finishes).
        A finished request that kept its current also returns it as "current"."""
        res = L.RequestResult()
        ms = -1 if wait == math.inf else int(wait * 1000)
        n = self._keep.get(rid, 0)
        cur = np.empty(n, np.complex128) if n else None
        L.call("rtm_server_poll", self._h, C.c_uint64(rid), ms, C.byref(res),
               cur.ctypes.data_as(C.c_void_p) if n else None, n, int(bool(release)))
        out = _result_dict(res)
        if n and out["state"] == "done":
            out["current"] = cur
        if release and out["state"] in ("done", "failed", "cancelled"):
            self._keep.pop(rid, None)
        return out

    def wait(self, rid: int, release=False):
        return self.poll(rid, wait=math.inf, release=release)

    def cancel(self, rid: int):
        L.call("rtm_server_cancel", self._h, C.c_uint64(rid))

    def close(self):
        if self._h:
            L.call("rtm_server_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
