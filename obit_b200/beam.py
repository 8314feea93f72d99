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
    parAng: float = 0.0          # parallactic angle, radians (linear Q, U)
    circular: bool = False       # circular feeds: records RR, LL, RL, LR; Jones in the R, L basis
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
                                int(self.jones.shape[1]), float(self.parAng), int(bool(self.circular)))


def baseline_codes(nant: int, nrow: int) -> np.ndarray:
    """BASELINE = 256 a1 + a2 (1-relative) of rows in the time-major order of
    obit_b200.uvdata.make_uvw (antenna pairs a1 < a2 in row-major order)."""
    a1, a2 = np.triu_indices(nant, k=1)
    code = 256.0 * (a1 + 1) + (a2 + 1)
    reps = (nrow + len(code) - 1) // len(code)
    return np.tile(code, reps)[:nrow].astype(np.float32)


@dataclass
class BeamImages:
    """Beam images of every antenna type (obit_dft_beam_jones): pixels float32
    (numAntType, 8, nplane, ny, nx) in the order P1 re, P1 im, P2 re, P2 im,
    X1 re, X1 im, X2 re, X2 im; grid geometry in degrees."""
    pixels: np.ndarray
    planeFreq: np.ndarray          # Hz per plane
    crval: tuple = (0.0, 0.0)
    crpix: tuple = (1.0, 1.0)
    cdelt: tuple = (1.0, 1.0)
    projection: int = 0            # 0 linear; 1..8 -SIN -TAN -ARC -NCP -GLS -MER -AIT -STG
    hwidth: int = 2
    fblank: float = -3.0e38
    refSizeFact: float = 0.0
    crota: float = 0.0             # y-axis rotation (deg; -MER and -AIT scales)
    _keep: list = field(default_factory=list, repr=False)

    def descriptor(self, d_pixels: int) -> _lib.ObitDFTBeamImages:
        ntype, _, nplane, ny, nx = self.pixels.shape
        pf = np.ascontiguousarray(self.planeFreq, dtype=np.float32)
        self._keep[:] = [pf]
        return _lib.ObitDFTBeamImages(ntype, nx, ny, nplane, C.c_void_p(d_pixels), float(self.fblank),
                                      int(self.hwidth), int(self.projection), (C.c_double * 2)(*self.crval),
                                      (C.c_float * 2)(*self.crpix), (C.c_float * 2)(*self.cdelt),
                                      pf.ctypes.data_as(C.POINTER(C.c_float)), float(self.refSizeFact),
                                      float(self.crota))


def jones_from_images(images: BeamImages, d_pixels: int, d_pos: int, ncomp: int, par_ang: float,
                      d_jones: int, stream: int = 0) -> None:
    """Fill the device Jones table at d_jones ((numAntType, ncomp, nplane, 8)
    floats) from the device beam images at d_pixels, at the device component
    positions d_pos ((ncomp, 2) degrees), asynchronously on stream."""
    lib = _lib.load()
    desc = images.descriptor(d_pixels)
    _lib.check(lib.obit_dft_beam_jones(C.byref(desc), C.c_void_p(d_pos), ncomp, C.c_float(par_ang),
                                       C.c_void_p(d_jones), C.c_void_p(stream)))
