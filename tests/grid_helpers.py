"""Seeded cases of the gridded model FT: a field of CLEAN components on the
cells of an image, the uv records that sample it, and the DFT component table
of the same field (through the component loader) for the DFT oracle."""
from __future__ import annotations

import math

import numpy as np

import oracle_grid as G
from obit_b200 import uvdata as U
from obit_b200.comps import CCField, CCModel, load_comps


def field_case(N: int = 64, ncomp: int = 150, seed: int = 3, gauss=None, shift3d: bool = False,
               nchan: int = 8, nif: int = 2, nint: int = 4, reach: float = 0.8, cell_asec: float = 2.0,
               neg_frac: float = 0.0, nstok: int = 2, flag_frac: float = 0.0, Ny: int | None = None,
               rotation: float = 0.0, uv_rotation: float = 0.0):
    """Returns (CCField, GridImage, CCModel, UVData).  Components on cells
    within the central half of an N x N image of cell_asec pixels; baselines
    reach `reach` x a quarter of the grid's uv half-width.  gauss: (maj, min
    arcsec, PA deg) of every component.  Ny: image rows (default N); rotation,
    uv_rotation: the image's and the uv data's CROTA (a 3-D field)."""
    rng = np.random.default_rng(seed)
    cell = cell_asec / 3600.0
    Ny = Ny or N
    ix = rng.integers(-N // 4, N // 4, ncomp)
    iy = rng.integers(-Ny // 4, Ny // 4, ncomp)
    flux = rng.uniform(0.01, 1.0, ncomp).astype(np.float32)
    if neg_frac > 0:
        flux[rng.random(ncomp) < neg_frac] *= -0.1
    cdx, cdy = -cell, cell
    parms = None
    if gauss is not None:
        parms = np.zeros((ncomp, 4), np.float32)
        parms[:, 0] = gauss[0] / 3600.0
        parms[:, 1] = gauss[1] / 3600.0
        parms[:, 2] = gauss[2]
        parms[:, 3] = 1.0
    f = CCField(flux=flux, deltaX=(ix * cdx).astype(np.float32), deltaY=(iy * cdy).astype(np.float32),
                crvalRA=150.0, crvalDec=45.0, do3D=shift3d, cdeltX=cdx, cdeltY=cdy, parms=parms)
    m = CCModel(uvRA=150.0, uvDec=45.0, do3D=shift3d, uvRotation=uv_rotation)
    f.rotation = rotation
    if shift3d:
        f.crvalRA = 150.0 + 0.05 / math.cos(math.radians(45.0))
        f.crvalDec = 45.03
    img = G.GridImage(N, Ny, N / 2 + 1, Ny / 2 + 1)
    umax = 1.0 / (cell * math.pi / 180.0) / 4.0
    freq = 1.4e9
    lam = 299792458.0 / freq
    pos = U.array_layout(12, umax * lam * reach, rng)
    uvw = U.make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)
    fa = U.freq_axis(nchan, nif, freq * 0.98, 2e6)
    uv = U.make_uvdata(uvw, nstok, nchan, nif, freq, fa, rng, flag_frac=flag_frac)
    return f, img, m, uv


def dft_sky(field: CCField, model: CCModel):
    """The DFT component table of the same field (merged, as the DFT reads it)."""
    sky, _ = load_comps([field], model)
    return sky


def with_pa(field: CCField, pa: float) -> CCField:
    """A copy of a Gaussian field with every component at position angle pa."""
    parms = field.parms.copy()
    parms[:, 2] = pa
    return CCField(**{**field.__dict__, "parms": parms})


def cell_bound(field: CCField, image: G.GridImage) -> float:
    """Worst relative difference between the reference kernel's model and the
    exact one: a shift of at most 0.0075 cell (0.005 offset + 0.0025
    tabulation) in u and v moves component c's phase by at most
    2 pi 0.0075 (|x_c| / nx + |y_c| / ny), x, y its cell offsets."""
    nx, ny = 2 * image.nx, 2 * image.ny
    x = np.abs(np.asarray(field.deltaX, np.float64) / field.cdeltX)
    y = np.abs(np.asarray(field.deltaY, np.float64) / field.cdeltY)
    a = np.abs(np.asarray(field.flux, np.float64))
    return float(np.sum(a * 2 * math.pi * 0.0075 * (x / nx + y / ny)) / a.sum())
