"""Multi-facet batch of the DFT subtract (obit_dft_batch_* in libobit_dft.so):
many facets, each its own device-resident records, layout, frequencies and
component table, applied by one persistent kernel launch per model family
that is captured once in a CUDA graph.  The reference applies such models one
field and one buffer at a time (ObitSystem/Obit/src/ObitGPUSkyModel.c:502-518).

Device memory (records, component tables) belongs to the caller and is passed
as raw device pointers; the batch copies the component tables at creation.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GPUModelInfo, GPUVisInfo, ObitDFTFacet
from .skymodel import SkyModelParams
from .uvdata import SkyComps, UVData


@dataclass
class Facet:
    """One facet: layout and frequencies (uv; uv.vis is not read), model,
    selection and operation, and the device pointers of its nvis records and
    of its component table (sky.ncomp rows of sky.lcomp floats)."""

    uv: UVData
    sky: SkyComps
    params: SkyModelParams
    d_vis: int
    nvis: int
    d_comps: int


def _descriptors(f: Facet, keep: list) -> ObitDFTFacet:
    uv, sky, p = f.uv, f.sky, f.params
    vi = GPUVisInfo()
    vi.nvis, vi.nprod, vi.nrparm, vi.lenvis = f.nvis, uv.ncorr, uv.nrparm, uv.lrec
    vi.nchan, vi.nIF, vi.nstok = uv.nchan, uv.nif, uv.nstok
    vi.ilocu, vi.ilocv, vi.ilocw = uv.ilocu, uv.ilocv, uv.ilocw
    vi.iloct = vi.ilocb = vi.ilocsu = -1
    c0 = (p.startChannel if p.startChannel > 0 else 1) - 1
    nc = p.numberChannel if p.numberChannel > 0 else uv.nchan - c0
    i0 = (p.startIF if p.startIF > 0 else 1) - 1
    ni = p.numberIF if p.numberIF > 0 else uv.nif - i0
    s0 = (p.startPoln if p.startPoln > 0 else 1) - 1
    ns = p.numberPoln if p.numberPoln > 0 else min(2, uv.nstok)
    vi.chanb, vi.chane, vi.IFb, vi.IFe = c0, c0 + nc - 1, i0, i0 + ni - 1
    vi.stokb, vi.stoke = s0, s0 + ns - 1
    vi.incf, vi.incif, vi.incs = uv.incf // 3, uv.incif // 3, uv.incs // 3
    vi.kincf, vi.kincif = uv.kincf, uv.kincif
    vi.stype = 1
    vi.freqScale = None
    mi = GPUModelInfo()
    mi.nterm, mi.size, mi.doSwap, mi.type, mi.opType = sky.nterm, sky.lcomp, 0, sky.gpu_type, p.op
    mi.nmodel[0] = sky.ncomp
    mi.model[0] = f.d_comps
    for i in range(4):
        mi.stokFact[i] = 1.0
    fa = np.ascontiguousarray(uv.freqArr, dtype=np.float64)
    keep += [vi, mi, fa]
    fd = ObitDFTFacet()
    fd.visInfo = C.pointer(vi)
    fd.modelInfo = C.pointer(mi)
    fd.freqArr = fa.ctypes.data_as(C.POINTER(C.c_double))
    fd.uvRefFreq = uv.freq
    fd.modelRefFreq = sky.refFreq if sky.refFreq > 0 else uv.freq
    if sky.is_tspec:
        si = np.ascontiguousarray(sky.specIndex, dtype=np.int32)
        sf = np.ascontiguousarray(sky.specFreq, dtype=np.float64)
        keep += [si, sf]
        mi.specIndex = si.ctypes.data_as(C.POINTER(C.c_int))
        fd.specFreq = sf.ctypes.data_as(C.POINTER(C.c_double))
        fd.nSpec = len(sf)
    fd.cpuRules = 1
    fd.stokFactor = p.stokFactor
    fd.doFlip = int(p.doFlip)
    fd.d_vis = f.d_vis
    fd.nvis = f.nvis
    return fd


class DFTBatch:
    """A batch of facets on the current device (CPU polarization rules and
    FP64 frequencies, as the host mirror uses)."""

    def __init__(self, facets: list[Facet]):
        self._lib = _lib.load()
        keep: list = []
        arr = (ObitDFTFacet * max(1, len(facets)))()
        for i, f in enumerate(facets):
            arr[i] = _descriptors(f, keep)
        h = C.c_void_p()
        _lib.check(self._lib.obit_dft_batch_create(arr, len(facets), C.byref(h)))
        self._h = h

    def autotune(self, stream: int = 0) -> dict:
        best = (C.c_int * 6)()
        _lib.check(self._lib.obit_dft_batch_autotune(self._h, C.c_void_p(stream), best))
        return dict(zip(["K", "ct", "Bt", "R", "threads", "tried"], list(best)))

    def set_tile(self, K: int = 0, ct: int = 0, Bt: int = 0, threads: int = 0) -> None:
        _lib.check(self._lib.obit_dft_batch_set_tile(self._h, K, ct, Bt, threads))

    def run(self, stream: int = 0) -> None:
        _lib.check(self._lib.obit_dft_batch_run(self._h, C.c_void_p(stream)))

    def run_host(self, h_ptrs: list[int], staging_bytes: int, stream: int = 0) -> dict:
        """Streamed run over host records: h_ptrs[i] is facet i's host buffer
        (pinned, nvis x lrec floats); staging_bytes of device staging.  Returns
        {waves, h2d_bytes} of the captured graph."""
        arr = (C.c_void_p * max(1, len(h_ptrs)))(*h_ptrs)
        info = (C.c_longlong * 2)()
        _lib.check(self._lib.obit_dft_batch_run_host(self._h, arr, int(staging_bytes), C.c_void_p(stream), info))
        return {"waves": int(info[0]), "h2d_bytes": int(info[1])}

    def run_per_facet(self, flavor: int = _lib.OBIT_DFT_RECUR, stream: int = 0) -> None:
        _lib.check(self._lib.obit_dft_batch_run_per_facet(self._h, flavor, C.c_void_p(stream)))

    def check(self) -> None:
        _lib.check(self._lib.obit_dft_batch_check(self._h))

    def info(self) -> dict:
        v = (C.c_longlong * 10)()
        _lib.check(self._lib.obit_dft_batch_info(self._h, v, 10))
        return dict(zip(["facets", "launches", "items", "evals", "K", "ct", "Bt", "R", "threads",
                         "grid"], list(v)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.obit_dft_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
