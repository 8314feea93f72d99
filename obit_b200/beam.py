"""Beam-corrected DFT description (obit_dft_set_beam): antenna types, the
Jones plane of each (channel, IF) and the Jones table of ObitCUDABeamModel
(GPUBeamAntInfo, ObitCUDABeamModelInfoDef.h:178-205) for linear feeds and a
Stokes I, Q, U or V sky."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class Beam:
    antType: np.ndarray          # int (numAnt,): type of antenna i + 1
    jchan: np.ndarray            # int (nchan * nIF,): Jones plane per (channel, IF), freqScale order
    jones: np.ndarray            # float32 (numAntType, ncomp, numJChan, 8): XX, XY, YX, YY (re, im)
    ilocb: int = 3               # BASELINE random parameter, or -1 for ANTENNA1 / ANTENNA2
    iloca1: int = -1
    iloca2: int = -1
    stokType: int = 1            # 1 I, 2 Q, 3 U, 4 V
    parAng: float = 0.0          # parallactic angle, radians (Q, U)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def numAnt(self) -> int:
        return int(len(self.antType))

    @property
    def numAntType(self) -> int:
        return int(self.jones.shape[0])

    @property
    def numJChan(self) -> int:
        return int(self.jones.shape[2])

    def descriptor(self, d_jones: int) -> _lib.ObitDFTBeam:
        """The C descriptor, with the Jones table at device address d_jones."""
        at = np.ascontiguousarray(self.antType, dtype=np.int32)
        jc = np.ascontiguousarray(self.jchan, dtype=np.int32)
        self._keep[:] = [at, jc]
        return _lib.ObitDFTBeam(self.numAnt, self.numAntType, self.numJChan,
                                at.ctypes.data_as(C.POINTER(C.c_int)), jc.ctypes.data_as(C.POINTER(C.c_int)),
                                self.ilocb, self.iloca1, self.iloca2, self.stokType, C.c_void_p(d_jones),
                                int(self.jones.shape[1]), float(self.parAng))


def baseline_codes(nant: int, nrow: int) -> np.ndarray:
    """BASELINE = 256 a1 + a2 (1-relative) of rows in the time-major order of
    obit_b200.uvdata.make_uvw (antenna pairs a1 < a2 in row-major order)."""
    a1, a2 = np.triu_indices(nant, k=1)
    code = 256.0 * (a1 + 1) + (a2 + 1)
    reps = (nrow + len(code) - 1) // len(code)
    return np.tile(code, reps)[:nrow].astype(np.float32)
