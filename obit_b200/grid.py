"""Gridded model Fourier transform on the GPU (obit_dft_grid_* in
libobit_dft.so; include/obit_dft_grid.h): the reference's second way of
predicting a CLEAN model, ObitSkyModelGridFTComps (grid, FFT, taper,
conjugate columns; ObitSystem/Obit/src/ObitSkyModel.c:4243-4371) and
ObitSkyModelFTGrid / ThreadSkyModelFTGrid (interpolation and subtract /
divide / replace per record and channel; :2878-3232), with the mode choice of
ObitSkyModelChose (:3560-3620)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GPUVisInfo, ObitDFTGridImage
from .comps import CCField, CCModel, _field_array, _model
from .skymodel import SkyModelParams
from .uvdata import UVData

KERNEL_REFERENCE = _lib.OBIT_DFT_GRID_KERNEL_REFERENCE
KERNEL_EXACT = _lib.OBIT_DFT_GRID_KERNEL_EXACT
MODE_FASTEST, MODE_DFT, MODE_GRID, MODE_MIXED = 0, 1, 2, 3
TYPE_COMPS, TYPE_IMAGE, TYPE_POINT = 0, 1, 2


@dataclass
class GridImage:
    """Image keywords of a field besides those of CCField."""

    nx: int
    ny: int
    crpixX: float
    crpixY: float


def vis_info(uv: UVData, params: SkyModelParams | None = None, nvis: int | None = None,
             keep: list | None = None):
    """(GPUVisInfo, freqScale array): uv's layout and the selection of params,
    freqScale pointing at a host FP32 copy of uv.fscale (also kept in `keep`)."""
    p = params or SkyModelParams()
    vi = GPUVisInfo()
    vi.nvis = uv.nvis if nvis is None else nvis
    vi.nprod, vi.nrparm, vi.lenvis = uv.ncorr, uv.nrparm, uv.lrec
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
    fs = np.ascontiguousarray(uv.fscale, dtype=np.float32)
    if keep is not None:
        keep.append(fs)
    vi.freqScale = fs.ctypes.data
    return vi, fs


class GridField:
    """One field's gridded model on the current device: the grid of its CLEAN
    components, its FFT and the interpolator's plane (ObitSkyModelGridFTComps),
    applied to records by FTGrid / FTGrid_device (ObitSkyModelFTGrid)."""

    def __init__(self, field: CCField, image: GridImage, model: CCModel, maxGrid: float = 1e20,
                 kernel: int = KERNEL_REFERENCE, stream: int = 0):
        self._lib = _lib.load()
        keep: list = []
        arr = _field_array([field], keep)
        m = _model(model)
        im = ObitDFTGridImage(image.nx, image.ny, image.crpixX, image.crpixY)
        h = C.c_void_p()
        _lib.check(self._lib.obit_dft_grid_create(arr, C.byref(im), C.byref(m), float(maxGrid), int(kernel),
                                                  C.c_void_p(stream), C.byref(h)))
        self._h = h

    @classmethod
    def from_image(cls, pixels: np.ndarray, fblank: float, field: CCField, image: GridImage, model: CCModel,
                   kernel: int = KERNEL_REFERENCE, stream: int = 0) -> "GridField":
        """An image model (ObitSkyModelLoadImage): pixels (ny, nx) float32 in
        place of components; field gives the geometry only."""
        self = cls.__new__(cls)
        self._lib = _lib.load()
        keep: list = []
        arr = _field_array([field], keep)
        m = _model(model)
        im = ObitDFTGridImage(image.nx, image.ny, image.crpixX, image.crpixY)
        pix = np.ascontiguousarray(pixels, dtype=np.float32)
        if pix.shape != (image.ny, image.nx):
            raise ValueError("pixels must be (ny, nx)")
        h = C.c_void_p()
        _lib.check(self._lib.obit_dft_grid_create_image(pix.ctypes.data_as(C.c_void_p), float(fblank), arr,
                                                        C.byref(im), C.byref(m), int(kernel), C.c_void_p(stream),
                                                        C.byref(h)))
        self._h = h
        return self

    def info(self) -> dict:
        a = (C.c_longlong * 10)()
        _lib.check(self._lib.obit_dft_grid_info(self._h, a, 10))
        keys = ["ncomp", "bad", "nx", "ny", "nxp", "gauss", "do3Dmul", "doPC", "doRot", "kernel"]
        return dict(zip(keys, (int(x) for x in a)))

    def plane(self) -> np.ndarray:
        """The interpolator's plane: complex64 (ny, nx / 2 + 13)."""
        i = self.info()
        out = np.zeros((i["ny"], i["nxp"]), np.complex64)
        _lib.check(self._lib.obit_dft_grid_plane(self._h, out.view(np.float32).ctypes.data_as(
            C.POINTER(C.c_float)), out.size * 2))
        return out

    def FTGrid(self, uv: UVData, params: SkyModelParams | None = None, stream: int = 0) -> UVData:
        """Applies the field to a copy of uv's records (host records through
        obit_dft_grid_apply_host); returns the new UVData."""
        p = params or SkyModelParams()
        out = uv.copy()
        keep: list = []
        vi, _ = vis_info(out, p, keep=keep)
        vis = np.ascontiguousarray(out.vis, dtype=np.float32)
        _lib.check(self._lib.obit_dft_grid_apply_host(
            self._h, C.byref(vi), p.op, float(p.stokFactor), int(p.doFlip),
            vis.ctypes.data_as(C.c_void_p), out.nvis, C.c_void_p(stream)))
        out.vis = vis
        return out

    def FTGrid_device(self, uv: UVData, d_vis: int, nvis: int, params: SkyModelParams | None = None,
                      d_fscale: int | None = None, stream: int = 0) -> None:
        """Applies the field to nvis device-resident records at d_vis (layout
        of uv), asynchronously on `stream`; d_fscale: device FP32 freqScale
        (None: uv.fscale is copied from the host)."""
        p = params or SkyModelParams()
        keep: list = []
        vi, _ = vis_info(uv, p, nvis=nvis, keep=keep)
        if d_fscale is not None:
            vi.freqScale = int(d_fscale)
        _lib.check(self._lib.obit_dft_grid_apply(self._h, C.byref(vi), p.op, float(p.stokFactor),
                                                 int(p.doFlip), C.c_void_p(d_vis), int(nvis),
                                                 C.c_void_p(stream)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.obit_dft_grid_destroy(self._h)
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


def choose_mode(model_mode: int, model_type: int, ncc, nx, ny, nvis: int, nchan: int) -> int:
    """ObitSkyModelChose: MODE_DFT or MODE_GRID for MODE_FASTEST (other modes
    are returned unchanged)."""
    lib = _lib.load()
    n = len(ncc)
    a = (C.c_int * max(1, n))(*[int(x) for x in ncc])
    b = (C.c_int * max(1, n))(*[int(x) for x in nx])
    c = (C.c_int * max(1, n))(*[int(x) for x in ny])
    return int(lib.obit_dft_choose_mode(int(model_mode), int(model_type), a, b, c, n, int(nvis), int(nchan)))


def choose_mode_measured(model_type: int, ncc, nx, ny, nvis: int, nchan: int, dft_rate: float = 0.0,
                         grid_rate: float = 0.0, grid_setup: float = 0.0) -> int:
    """MODE_DFT or MODE_GRID from this library's own rates (0: the measured
    B200 defaults); obit_dft_choose_mode_measured."""
    lib = _lib.load()
    n = len(ncc)
    a = (C.c_int * max(1, n))(*[int(x) for x in ncc])
    b = (C.c_int * max(1, n))(*[int(x) for x in nx])
    c = (C.c_int * max(1, n))(*[int(x) for x in ny])
    return int(lib.obit_dft_choose_mode_measured(int(model_type), a, b, c, n, int(nvis), int(nchan),
                                                 float(dft_rate), float(grid_rate), float(grid_setup)))
