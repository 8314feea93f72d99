"""Python face of the GPU sky model: the class functions of Obit's
ObitGPUSkyModel (Create / DFTInit / DFTSetMod / DFTCalc / DFTShutdown,
ObitSystem/Obit/include/ObitGPUSkyModel.h:95-125) over the C host mirror in
libobit_dft.so, plus the device-resident call used when visibilities already
live in GPU memory.

Errors raise DFTError (the reference pushes them on an ObitErr stack and the
caller tracebacks; there is no silent fallback to a CPU path).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import DFTError, ObitDFTErr, ObitDFTSkyModel, ObitDFTUVData
from .uvdata import SkyComps, UVData

OP_SUB, OP_DIV, OP_REPL = 0, 1, 2


@dataclass
class SkyModelParams:
    """ObitSkyModel members the DFT reads (ObitSkyModelGetInput,
    ObitSkyModel.c:3397-3551; ObitSkyModelSetSelect, :3647-3897)."""

    factor: float = 1.0
    op: int = OP_SUB
    doFlip: bool = False
    stokFactor: float = 1.0
    startChannel: int = 1     # 1-relative, 0 = all
    numberChannel: int = 0
    startIF: int = 1
    numberIF: int = 0
    startPoln: int = 1
    numberPoln: int = 0       # 0 = min(2, nstok) (correlation data)
    GPU_no: int = 0
    nVisPIO: int = 0          # 0 = the reference's 10000


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def uv_struct(uv: UVData, with_buffer: bool, exact_freq: bool, keep: list) -> ObitDFTUVData:
    """The ObitUV / ObitUVDesc fields of uv the C mirror reads (ObitDFTUVData);
    arrays it points to are appended to keep.  with_buffer: point at uv.vis;
    exact_freq: pass the FP64 channel frequencies."""
    d = ObitDFTUVData()
    d.nvis = uv.nvis
    d.numVisBuff = uv.nvis
    d.lrec = uv.lrec
    d.nrparm = uv.nrparm
    d.ncorr = uv.ncorr
    d.ilocu, d.ilocv, d.ilocw = uv.ilocu, uv.ilocv, uv.ilocw
    ax = [3, uv.nstok, uv.nchan, uv.nif, 1, 1, 1]
    for i in range(7):
        d.inaxes[i] = ax[i]
    d.jlocs, d.jlocf, d.jlocif = uv.jlocs, uv.jlocf, uv.jlocif
    d.incs, d.incf, d.incif = uv.incs, uv.incf, uv.incif
    d.crvalStokes = uv.crval_stokes
    d.freq = uv.freq
    fs = np.ascontiguousarray(uv.fscale, dtype=np.float32)
    fa = np.ascontiguousarray(uv.freqArr, dtype=np.float64)
    keep += [fs, fa]
    d.fscale = _ptr(fs, C.c_float)
    d.freqArr = _ptr(fa, C.c_double) if exact_freq else None
    if with_buffer:
        if uv.vis.dtype != np.float32 or not uv.vis.flags.c_contiguous:
            raise DFTError(1, "uv buffer must be C-contiguous float32")
        d.buffer = _ptr(uv.vis, C.c_float)
    return d


class GPUSkyModel:
    """One sky model bound to one uv layout on one GPU."""

    def __init__(self, name: str = "GPUSkyModel"):
        self._lib = _lib.load()
        self._h = self._lib.obit_gpu_skymodel_create(name.encode())
        if not self._h:
            raise DFTError(1, "obit_gpu_skymodel_create failed")
        self._err = ObitDFTErr()
        self._keep = []  # arrays referenced by C structs
        self._sky = None
        self._uvdesc = None

    # -- helpers -----------------------------------------------------------
    def _raise(self):
        msg = self._err.message.decode(errors="replace")
        self._err.error = 0
        raise DFTError(1, msg)

    def _sky_struct(self, sky: SkyComps, p: SkyModelParams, uv: UVData) -> ObitDFTSkyModel:
        s = ObitDFTSkyModel()
        s.modType = sky.modType
        s.nSpecTerm = sky.nterm
        s.factor = p.factor
        s.doDivide = int(p.op == OP_DIV)
        s.doReplace = int(p.op == OP_REPL)
        s.doFlip = int(p.doFlip)
        s.stokFactor = p.stokFactor
        s.startChannelPB = p.startChannel if p.startChannel > 0 else 1
        s.numberChannelPB = p.numberChannel if p.numberChannel > 0 else uv.nchan - s.startChannelPB + 1
        s.startIFPB = p.startIF if p.startIF > 0 else 1
        s.numberIFPB = p.numberIF if p.numberIF > 0 else uv.nif - s.startIFPB + 1
        s.startPoln = p.startPoln if p.startPoln > 0 else 1
        s.numberPoln = p.numberPoln if p.numberPoln > 0 else min(2, uv.nstok)
        s.modelRefFreq = sky.refFreq if sky.refFreq > 0 else uv.freq
        s.isMF = int(sky.is_tspec)
        if sky.is_tspec:
            sf = np.ascontiguousarray(sky.specFreq, dtype=np.float64)
            si = np.ascontiguousarray(sky.specIndex, dtype=np.int32)
            self._keep += [sf, si]
            s.nSpec = len(sf)
            s.specFreq = _ptr(sf, C.c_double)
            s.specIndex = _ptr(si, C.c_int)
        s.GPU_no = p.GPU_no
        s.nVisPIO = p.nVisPIO
        return s

    def _uv_struct(self, uv: UVData, with_buffer: bool, exact_freq: bool) -> ObitDFTUVData:
        return uv_struct(uv, with_buffer, exact_freq, self._keep)

    # -- class functions -----------------------------------------------------
    def DFTInit(self, sky: SkyComps, uv: UVData, params: SkyModelParams | None = None,
                exact_freq: bool = True) -> None:
        """ObitGPUSkyModelDFTInit: buffers, streams and descriptors for `uv`.
        exact_freq passes the FP64 channel frequencies; False keeps only the
        reference's FP32 freqScale."""
        p = params or SkyModelParams()
        self._params = p
        self._sky = self._sky_struct(sky, p, uv)
        self._uvdesc = self._uv_struct(uv, False, exact_freq)
        if self._lib.obit_gpu_skymodel_dft_init(self._h, C.byref(self._sky), C.byref(self._uvdesc),
                                                C.byref(self._err)):
            self._raise()

    def DFTSetMod(self, sky: SkyComps) -> None:
        """ObitGPUSkyModelDFTSetMod: load the component table."""
        comps = np.ascontiguousarray(sky.comps, dtype=np.float32)
        self._keep.append(comps)
        if self._lib.obit_gpu_skymodel_dft_setmod(self._h, C.byref(self._sky), _ptr(comps, C.c_float),
                                                  comps.shape[1], comps.shape[0], C.byref(self._err)):
            self._raise()

    def DFTCalc(self, uv: UVData) -> None:
        """ObitGPUSkyModelDFTCalc: apply the model to uv.vis in place (at most
        nVisPIO records per call, as the reference's buffer)."""
        d = self._uv_struct(uv, True, False)
        if self._lib.obit_gpu_skymodel_dft_calc(self._h, C.byref(d), C.byref(self._err)):
            self._raise()

    def DFTShutdown(self) -> None:
        """ObitGPUSkyModelDFTShutdown: release buffers and library state."""
        if self._h and self._lib.obit_gpu_skymodel_dft_shutdown(self._h, C.byref(self._err)):
            self._raise()

    # -- additions -----------------------------------------------------------
    @property
    def gpuinfo(self):
        return self._lib.obit_gpu_skymodel_info(self._h)

    def set_kernel(self, flavor: int = _lib.OBIT_DFT_RECUR, chan_per_thread: int = 0,
                   comps_per_tile: int = 0, blocks_per_tile: int = 0, threads: int = 0) -> None:
        """Kernel flavor and tile shape (0 keeps the current / planner's choice)."""
        _lib.check(self._lib.obit_dft_set_kernel(self.gpuinfo, flavor, chan_per_thread,
                                                 comps_per_tile))
        if blocks_per_tile or threads:
            _lib.check(self._lib.obit_dft_set_tile(self.gpuinfo, blocks_per_tile, threads))

    def set_positions_fp64(self, xyz) -> None:
        """FP64 X, Y, Z per component (ncomp x 3, the units of table fields 1-3)
        for the phase of the model set by the last DFTSetMod; None drops them."""
        if xyz is None:
            _lib.check(self._lib.obit_dft_set_mod_d(self.gpuinfo, None, 0))
            return
        a = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        _lib.check(self._lib.obit_dft_set_mod_d(self.gpuinfo, a.ctypes.data_as(C.POINTER(C.c_double)),
                                                a.shape[0]))

    def set_beam(self, beam, d_jones: int = 0) -> None:
        """Beam-corrected model (obit_b200.beam.Beam, Jones table at device
        address d_jones) for the following calls; None returns to the plain
        sky model."""
        if beam is None:
            _lib.check(self._lib.obit_dft_set_beam(self.gpuinfo, None))
            return
        self._beam_desc = beam.descriptor(d_jones)
        _lib.check(self._lib.obit_dft_set_beam(self.gpuinfo, C.byref(self._beam_desc)))

    def plan_info(self) -> dict:
        """The kernel plan the next call uses (built on demand)."""
        arr = (C.c_int * 11)()
        _lib.check(self._lib.obit_dft_plan_info(self.gpuinfo, arr, 11))
        keys = ("flavor", "K", "ct", "Bt", "R", "threads", "nblocks", "ndf", "specFactored", "mixed",
                "ncompPoint")
        return dict(zip(keys, list(arr)))

    def beam_info(self) -> dict:
        """The beam kernel the next call uses: form 0 (blocks on the FP32
        pipe), 1 (tensor-core form) or 2 (one thread per channel), components
        per tile, channel runs or blocks per record."""
        arr = (C.c_int * 3)()
        _lib.check(self._lib.obit_dft_beam_info(self.gpuinfo, arr, 3))
        return dict(zip(("form", "ct", "units"), list(arr)))

    def calc_device(self, d_vis_ptr: int, nvis: int, stream_ptr: int = 0) -> None:
        """Apply the model to nvis records already in device memory (async)."""
        _lib.check(self._lib.obit_dft_calc_device(self.gpuinfo, C.c_void_p(d_vis_ptr), nvis,
                                                  C.c_void_p(stream_ptr)))

    def check(self) -> None:
        """Synchronize and raise if a kernel reported an internal error."""
        _lib.check(self._lib.obit_dft_check(self.gpuinfo))

    def close(self) -> None:
        if self._h:
            self._lib.obit_gpu_skymodel_unref(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
