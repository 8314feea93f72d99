"""Test infrastructure: the reference's own CUDA sky-model layer
(ObitSystem/Obit/src/ObitCUDASkyModel.cu compiled unmodified for sm_100a into
_ref/libobit_refgpu.so by oracle/Makefile) driven through the same GPUInfo the
host mirror fills, as ObitGPUSkyModel.c would fill it for the reference.

Only tests use this module, as a second, independent implementation to check
against and as a measured comparator; the product never loads the library.

Semantics of the reference kernels that differ from the CPU DFT (and from the
FP64 oracle), handled here so that results are comparable:
  * spectral terms: the kernels use exp(-sum a_t L^(t+1))
    (ObitCUDASkyModel.cu:240,563), the CPU exp(+...): the coefficients are
    negated in the table handed to the reference;
  * phases are FP32 u*X + v*Y + w*Z with __sincosf and frequencies are the FP32
    freqScale, so agreement with the FP64 oracle is at FP32 level and only at
    modest phases;
  * tabulated spectra read a host pointer on the device
    (ObitCUDASkyModel.cu:295): not driven here;
  * DFTShutdown resets the device (ObitCUDASkyModel.cu:780): never called.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libobit_refgpu.so"
SUPPORTED = (0, 10, 1, 11)  # Point, PointSpec, Gauss, GaussSpec (ObitSkyModelCompType)

_lib = None


def available() -> bool:
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(LIB), mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
        for n in ("ObitCUDASkyModelDFTInit", "ObitCUDASkyModelDFTSetMod", "ObitCUDASkyModelDFTCalc"):
            getattr(_lib, n).restype = None
            getattr(_lib, n).argtypes = [C.c_void_p]
    return _lib


def _ref_sky(sky):
    from obit_b200 import uvdata as U

    comps = sky.comps.copy()
    if sky.modType == U.MOD_POINT_SPEC:
        comps[:, 4:4 + sky.nterm] *= -1.0
    elif sky.modType == U.MOD_GAUSS_SPEC:
        comps[:, 7:7 + sky.nterm] *= -1.0
    return U.SkyComps(sky.modType, comps, nterm=sky.nterm, refFreq=sky.refFreq)


class RefGPU:
    """The reference kernels bound to one uv layout and model."""

    def __init__(self, uv, sky, params):
        from obit_b200.skymodel import GPUSkyModel, SkyModelParams

        if sky.modType not in SUPPORTED:
            raise ValueError("tabulated spectra are not driven on the reference kernels")
        self.lib = _load()
        self.uv = uv
        p = SkyModelParams(**{**params.__dict__, "nVisPIO": max(1, uv.nvis)})
        self.gm = GPUSkyModel("reference-kernels")
        self.gm.DFTInit(sky, uv, p, exact_freq=False)
        self.gm.DFTSetMod(_ref_sky(sky))
        self.gi = self.gm.gpuinfo
        self.lib.ObitCUDASkyModelDFTInit(C.cast(self.gi, C.c_void_p))

    def calc(self, vis: np.ndarray) -> np.ndarray:
        """ObitCUDASkyModelDFTCalc on a copy of vis (records x lrec float32)."""
        g = self.gi.contents
        n = vis.shape[0]
        g.nvis = n
        g.h_visInfo.contents.nvis = n
        buf = np.ascontiguousarray(vis, dtype=np.float32)
        C.memmove(g.h_data, buf.ctypes.data, buf.nbytes)
        self.lib.ObitCUDASkyModelDFTCalc(C.cast(self.gi, C.c_void_p))
        out = np.empty_like(buf)
        C.memmove(out.ctypes.data, g.h_data, buf.nbytes)
        return out

    def time_calc(self, vis: np.ndarray, reps: int = 3) -> float:
        """Seconds per ObitCUDASkyModelDFTCalc (host buffer in, host buffer out:
        its 4-stream H2D / kernel / D2H pipeline), best of reps after one warm-up."""
        g = self.gi.contents
        g.nvis = vis.shape[0]
        g.h_visInfo.contents.nvis = vis.shape[0]
        buf = np.ascontiguousarray(vis, dtype=np.float32)
        C.memmove(g.h_data, buf.ctypes.data, buf.nbytes)
        self.lib.ObitCUDASkyModelDFTCalc(C.cast(self.gi, C.c_void_p))
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            self.lib.ObitCUDASkyModelDFTCalc(C.cast(self.gi, C.c_void_p))
            best = min(best, time.perf_counter() - t0)
        return best

    def close(self):
        # the library state of the mirror is released; the reference's own
        # shutdown (a device reset) is not called
        self.gm.DFTShutdown()
        self.gm.close()
