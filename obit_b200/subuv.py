"""The caller of the model path: ObitSkyModelSubUV's pass structure
(ObitSystem/Obit/src/ObitSkyModel.c:850-1087) over this library's GPU paths.
The mode is chosen as ObitSkyModelChose does (or from the measured rates);
the DFT loads every field's components into one table and applies them in one
pass (nload = -1, :986-987), the gridded model applies each field in its own
pass, in field order (:974-995); data I/O, calibration and selection of the
reference's ObitUV layer are the caller's."""
from __future__ import annotations

from dataclasses import dataclass

from . import grid as GR
from .comps import CCField, CCModel, load_comps
from .skymodel import GPUSkyModel, SkyModelParams
from .uvdata import UVData


@dataclass
class SubUVResult:
    uv: UVData
    mode: int            # grid.MODE_DFT or grid.MODE_GRID
    ncomp: int           # components applied (DFT: merged rows; grid: rows gridded)


def sub_uv(uv: UVData, fields: list[CCField], images: list[GR.GridImage], model: CCModel,
           params: SkyModelParams | None = None, mode: int = GR.MODE_FASTEST, measured: bool = False,
           maxGrid: float = 1e20, kernel: int = GR.KERNEL_REFERENCE, exact_freq: bool = False) -> SubUVResult:
    """Applies the CLEAN model of `fields` to uv's records (a copy) with the
    operation of params.  mode: MODE_FASTEST chooses (the reference's time model,
    or this library's measured rates with measured=True), MODE_DFT or MODE_GRID
    force one.  exact_freq: the DFT forms its phase from FP64 channel
    frequencies (the gridded model, as the reference's, uses FP32 freqScale)."""
    p = params or SkyModelParams()
    ncc = []
    for f in fields:
        first = f.startComp if f.startComp > 0 else 1
        last = f.endComp if f.endComp > 0 else len(f.flux)
        ncc.append(max(0, last - first + 1))
    nx = [im.nx for im in images]
    ny = [im.ny for im in images]
    chan = uv.nchan * uv.nif
    if mode == GR.MODE_FASTEST:
        choose = GR.choose_mode_measured if measured else (lambda *a: GR.choose_mode(GR.MODE_FASTEST, *a))
        use = choose(GR.TYPE_COMPS, ncc, nx, ny, uv.nvis, chan)
    else:
        use = mode
    if use == GR.MODE_DFT:
        sky, _ = load_comps(fields, model)
        out = uv.copy()
        if sky.ncomp > 0 and uv.nvis > 0:
            q = SkyModelParams(**{**p.__dict__, "nVisPIO": max(1, uv.nvis)})
            gm = GPUSkyModel("subuv")
            try:
                gm.DFTInit(sky, out, q, exact_freq=exact_freq)
                gm.DFTSetMod(sky)
                gm.DFTCalc(out)
                gm.DFTShutdown()
            finally:
                gm.close()
        return SubUVResult(out, GR.MODE_DFT, sky.ncomp)
    if use != GR.MODE_GRID:
        raise ValueError(f"mode {use} is not supported (Mixed: the DFT with minDFT plus the grid with maxGrid)")
    out = uv
    total = 0
    for f, im in zip(fields, images):
        with GR.GridField(f, im, model, maxGrid=maxGrid, kernel=kernel) as gf:
            total += gf.info()["ncomp"]
            out = gf.FTGrid(out, p)
    if out is uv:
        out = uv.copy()
    return SubUVResult(out, GR.MODE_GRID, total)
