"""Records resident in device memory across CLEAN major cycles
(obit_dft_resident_* in libobit_dft.so): uploaded once, then per cycle a work
copy is reset on the device, models are applied to it with the device-resident
calls (GPUSkyModel.calc_device, DFTBatch facets pointing into it,
GridField.FTGrid_device) and the residual is downloaded.  The reference
re-reads the data and round-trips every buffer each cycle
(ObitSystem/Obit/src/ObitDConCleanVisMF.c:907, ObitGPUSkyModel.c:510-517)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .uvdata import UVData


class ResidentUV:
    """uv's records on the current device, with a work copy."""

    def __init__(self, uv: UVData, stream: int = 0):
        self._lib = _lib.load()
        self.uv = uv
        vis = np.ascontiguousarray(uv.vis, dtype=np.float32)
        h = C.c_void_p()
        _lib.check(self._lib.obit_dft_resident_create(vis.ctypes.data_as(C.c_void_p), uv.nvis, uv.lrec,
                                                      C.c_void_p(stream), C.byref(h)))
        self._h = h

    @property
    def d_records(self) -> int:
        """Device pointer of the work copy."""
        return int(self._lib.obit_dft_resident_records(self._h) or 0)

    def reset(self, stream: int = 0) -> None:
        _lib.check(self._lib.obit_dft_resident_reset(self._h, C.c_void_p(stream)))

    def download(self, stream: int = 0) -> UVData:
        """The work copy as a new UVData (after the work queued on stream)."""
        out = self.uv.copy()
        buf = np.empty_like(out.vis, dtype=np.float32)
        _lib.check(self._lib.obit_dft_resident_download(self._h, buf.ctypes.data_as(C.c_void_p),
                                                        C.c_void_p(stream)))
        out.vis = buf
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.obit_dft_resident_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
