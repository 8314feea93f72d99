"""CLEAN-component tables to the DFT component table (obit_dft_load_comps in
libobit_dft.so; include/obit_dft_comps.h): the host step Obit runs before each
DFT pass (ObitSkyModelLoadComps, ObitSystem/Obit/src/ObitSkyModel.c:1682-2121,
with ObitTableCCUtilMergeSel, ObitTableCCUtil.c:1238-1361)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ObitDFTCCField, ObitDFTCCModel
from .uvdata import SkyComps


@dataclass
class CCField:
    """One field: CC-table columns and the image keywords the geometry needs."""

    flux: np.ndarray
    deltaX: np.ndarray            # deg
    deltaY: np.ndarray            # deg
    crvalRA: float                # deg
    crvalDec: float               # deg
    rotation: float = 0.0         # CROTA of the declination axis, deg
    do3D: bool = True
    deltaZ: np.ndarray | None = None
    parms: np.ndarray | None = None   # (nrow, nparms)
    status: np.ndarray | None = None
    startComp: int = 1
    endComp: int = 0
    xPxOff: float = 0.0
    yPxOff: float = 0.0
    cdeltX: float = 0.0
    cdeltY: float = 0.0
    xShift: float = 0.0
    yShift: float = 0.0
    ncp: bool = False


@dataclass
class CCModel:
    uvRA: float
    uvDec: float
    uvRotation: float = 0.0
    factor: float = 1.0
    minFlux: float = 0.0
    minDFT: float = 0.0
    noNeg: bool = False
    do3D: bool = False


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _field_array(fields: list[CCField], keep: list):
    arr = (ObitDFTCCField * max(1, len(fields)))()
    for i, f in enumerate(fields):
        cols = [_f32(f.flux), _f32(f.deltaX), _f32(f.deltaY), _f32(f.deltaZ), _f32(f.parms)]
        st = None if f.status is None else np.ascontiguousarray(f.status, dtype=np.int32)
        keep += cols + [st]
        d = arr[i]
        d.nrow = len(cols[0])
        d.flux, d.deltaX, d.deltaY = (c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols[:3])
        if cols[3] is not None:
            d.deltaZ = cols[3].ctypes.data_as(C.POINTER(C.c_float))
        if cols[4] is not None:
            d.parms = cols[4].ctypes.data_as(C.POINTER(C.c_float))
            d.nparms = cols[4].shape[1]
        if st is not None:
            d.status = st.ctypes.data_as(C.POINTER(C.c_int))
        d.startComp, d.endComp = f.startComp, f.endComp
        d.crvalRA, d.crvalDec, d.rotation, d.do3D = f.crvalRA, f.crvalDec, f.rotation, int(f.do3D)
        d.xPxOff, d.yPxOff, d.cdeltX, d.cdeltY = f.xPxOff, f.yPxOff, f.cdeltX, f.cdeltY
        d.xShift, d.yShift, d.ncpProjection = f.xShift, f.yShift, int(f.ncp)
    return arr


def _model(model: CCModel) -> ObitDFTCCModel:
    return ObitDFTCCModel(model.uvRA, model.uvDec, model.uvRotation, model.factor, model.minFlux,
                          model.minDFT, int(model.noNeg), int(model.do3D))


def load_comps(fields: list[CCField], model: CCModel, ref_freq: float = 0.0):
    """Returns (SkyComps of the components, rows allocated incl. zero rows)."""
    lib = _lib.load()
    keep: list = []
    arr = _field_array(fields, keep)
    m = _model(model)
    nrow, ncomp, lcomp, mtype, nterm = (C.c_int() for _ in range(5))
    _lib.check(lib.obit_dft_load_comps(arr, len(fields), C.byref(m), None, 0, C.byref(nrow),
                                       C.byref(ncomp), C.byref(lcomp), C.byref(mtype), C.byref(nterm)))
    table = np.zeros((max(1, nrow.value), lcomp.value), np.float32)
    xyz = np.zeros((table.shape[0], 3), np.float64)
    _lib.check(lib.obit_dft_load_comps_d(arr, len(fields), C.byref(m),
                                         table.ctypes.data_as(C.POINTER(C.c_float)), table.size,
                                         C.byref(nrow), C.byref(ncomp), C.byref(lcomp), C.byref(mtype),
                                         C.byref(nterm), xyz.ctypes.data_as(C.POINTER(C.c_double))))
    comps = np.ascontiguousarray(table[:ncomp.value])
    sky = SkyComps(mtype.value, comps, nterm=nterm.value, refFreq=ref_freq,
                   xyz=np.ascontiguousarray(xyz[:ncomp.value]))
    return sky, nrow.value


@dataclass
class MFModel:
    """Tabulated-spectrum settings of an MF sky model (ObitSkyModelMF)."""

    specFreq: np.ndarray          # Hz per coarse plane
    noSIfit: bool = False
    doAlphaCorr: bool = False
    priorAlpha: float = 0.0
    priorAlphaRefF: float = 1.0e9


def load_comps_mf(fields: list[CCField], model: CCModel, mf: MFModel, spec_index=None):
    """obit_dft_load_comps_mf: components with tabulated spectra (CC types 20,
    21; PARMS[4..] per-plane fluxes) and fitted spectral indices.  Returns
    (SkyComps of type 20 or 21, rows allocated).  spec_index: the plane of each
    (channel, IF), kept on the result for the DFT."""
    from .uvdata import MOD_GAUSS_TSPEC, MOD_POINT_TSPEC

    lib = _lib.load()
    keep: list = []
    arr = _field_array(fields, keep)
    m = _model(model)
    sf = np.ascontiguousarray(mf.specFreq, dtype=np.float64)
    mm = _lib.ObitDFTCCModelMF(len(sf), sf.ctypes.data_as(C.POINTER(C.c_double)), int(mf.noSIfit),
                               int(mf.doAlphaCorr), float(mf.priorAlpha), float(mf.priorAlphaRefF))
    nrow, ncomp, lcomp, mtype = (C.c_int() for _ in range(4))
    _lib.check(lib.obit_dft_load_comps_mf(arr, len(fields), C.byref(m), C.byref(mm), None, 0, C.byref(nrow),
                                          C.byref(ncomp), C.byref(lcomp), C.byref(mtype)))
    table = np.zeros((max(1, nrow.value), lcomp.value), np.float32)
    _lib.check(lib.obit_dft_load_comps_mf(arr, len(fields), C.byref(m), C.byref(mm),
                                          table.ctypes.data_as(C.POINTER(C.c_float)), table.size,
                                          C.byref(nrow), C.byref(ncomp), C.byref(lcomp), C.byref(mtype)))
    kind = MOD_POINT_TSPEC if mtype.value == 20 else MOD_GAUSS_TSPEC
    comps = np.ascontiguousarray(table[:ncomp.value])
    return SkyComps(kind, comps, specFreq=sf, specIndex=spec_index), nrow.value
