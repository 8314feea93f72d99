"""The caller of the model path: ObitSkyModelSubUV's pass structure
(ObitSystem/Obit/src/ObitSkyModel.c:850-1087) over this library's GPU paths,
run natively by obit_dft_sub_uv (include/obit_dft_subuv.h).  The mode is chosen
as ObitSkyModelChose does (or from the measured rates); the DFT loads every
field's components into one table and applies them in one pass (nload = -1,
:986-987), the gridded model applies each field in its own pass, in field order
(:974-995); data I/O, calibration and selection of the reference's ObitUV layer
are the caller's."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib
from . import grid as GR
from ._lib import ObitDFTErr, ObitDFTGridImage, ObitDFTSkyModel
from .comps import CCField, CCModel, _field_array, _model
from .skymodel import OP_DIV, OP_REPL, SkyModelParams, uv_struct
from .uvdata import UVData


@dataclass
class SubUVResult:
    uv: UVData
    mode: int            # grid.MODE_DFT, MODE_GRID or MODE_MIXED
    ncomp: int           # components applied (DFT: merged rows; grid: rows gridded; Mixed: both)


def _sky_fields(p: SkyModelParams, uv: UVData) -> ObitDFTSkyModel:
    """The ObitSkyModel settings of params (operation, factor, selection); the
    model type and spectral terms come from the loaded table."""
    s = ObitDFTSkyModel()
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
    s.modelRefFreq = uv.freq
    s.GPU_no = p.GPU_no
    return s


def sub_uv(uv: UVData, fields: list[CCField], images: list[GR.GridImage], model: CCModel,
           params: SkyModelParams | None = None, mode: int = GR.MODE_FASTEST, measured: bool = False,
           maxGrid: float = 1e20, kernel: int = GR.KERNEL_REFERENCE, exact_freq: bool = False) -> SubUVResult:
    """Applies the CLEAN model of `fields` to a copy of uv's records with the
    operation of params.  mode: MODE_FASTEST chooses (the reference's time
    model, or this library's measured rates with measured=True), MODE_DFT or
    MODE_GRID force one, MODE_MIXED runs per field the DFT of the components
    above model.minDFT and the gridded model of those of at most maxGrid.
    exact_freq: the DFT forms its phase from FP64 channel frequencies (the
    gridded model, as the reference's, uses FP32 freqScale)."""
    p = params or SkyModelParams()
    if mode not in (GR.MODE_FASTEST, GR.MODE_DFT, GR.MODE_GRID, GR.MODE_MIXED):
        raise ValueError(f"unknown mode {mode}")
    lib = _lib.load()
    keep: list = []
    out = uv.copy()
    arr = _field_array(fields, keep)
    imgs = (ObitDFTGridImage * max(1, len(images)))()
    for i, im in enumerate(images):
        imgs[i] = ObitDFTGridImage(int(im.nx), int(im.ny), float(im.crpixX), float(im.crpixY))
    m = _model(model)
    s = _sky_fields(p, out)
    d = uv_struct(out, True, exact_freq, keep)
    used, ncomp = C.c_int(), C.c_int()
    err = ObitDFTErr()
    rc = lib.obit_dft_sub_uv(arr, len(fields), imgs if images else None, C.byref(m), C.byref(s), C.byref(d),
                             int(mode), int(bool(measured)), float(maxGrid), int(kernel), C.byref(used),
                             C.byref(ncomp), C.byref(err))
    if rc:
        raise _lib.DFTError(rc, err.message.decode(errors="replace"))
    return SubUVResult(out, used.value, ncomp.value)


def sub_uv_image(uv: UVData, pixels: list, fblank: float, fields: list[CCField], images: list[GR.GridImage],
                 model: CCModel, params: SkyModelParams | None = None,
                 kernel: int = GR.KERNEL_REFERENCE) -> SubUVResult:
    """The pass structure for image models (obit_dft_sub_uv_image): per field
    the model image pixels[f] ((ny, nx) float32; fields[f] gives the geometry
    only) gridded and applied to a copy of uv's records.  ncomp of the result
    counts the pixels gridded."""
    import numpy as np

    p = params or SkyModelParams()
    if not (len(pixels) == len(fields) == len(images)):
        raise ValueError("one image per field")
    lib = _lib.load()
    keep: list = []
    out = uv.copy()
    arr = _field_array(fields, keep)
    imgs = (ObitDFTGridImage * max(1, len(images)))()
    pix = (C.c_void_p * max(1, len(pixels)))()
    for i, (im, px) in enumerate(zip(images, pixels)):
        imgs[i] = ObitDFTGridImage(int(im.nx), int(im.ny), float(im.crpixX), float(im.crpixY))
        a = np.ascontiguousarray(px, dtype=np.float32)
        if a.shape != (im.ny, im.nx):
            raise ValueError("pixels must be (ny, nx)")
        keep.append(a)
        pix[i] = a.ctypes.data
    m = _model(model)
    s = _sky_fields(p, out)
    d = uv_struct(out, True, False, keep)
    n = C.c_longlong()
    err = ObitDFTErr()
    rc = lib.obit_dft_sub_uv_image(pix, float(fblank), arr, len(fields), imgs, C.byref(m), C.byref(s), C.byref(d),
                                   int(kernel), C.byref(n), C.byref(err))
    if rc:
        raise _lib.DFTError(rc, err.message.decode(errors="replace"))
    return SubUVResult(out, GR.MODE_GRID, n.value)
