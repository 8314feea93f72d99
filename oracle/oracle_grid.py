"""Test infrastructure: CPU oracle of the gridded model Fourier transform.

Restates, in numpy, the reference's gridded path of ObitSkyModel (mode
OBIT_SkyModel_Grid), per field:

  ObitTableCCUtilGrid        ObitTableCCUtil.c:106-302   components summed into a
                                                         grid of OverSample x the image
  ObitSkyModelFTImage        ObitSkyModel.c:4475-4498    quadrant swap, real-to-half-
                                                         complex FFT, row swap
  ObitSkyModelGridFTComps    ObitSkyModel.c:4243-4371    Gaussian taper, conjugate
                                                         columns, interpolator set-up
  ObitCArrayAddConjg         ObitCArray.c:1660-1726
  ObitCInterpolate           ObitCInterpolate.c:128-206, 359-455, 557-580, 699-830
                                                         Lagrange kernel table and
                                                         interpolation at a uv offset
  ThreadSkyModelFTGrid       ObitSkyModel.c:2970-3232    per visibility and channel:
                                                         uvw scaling, re-projection or
                                                         rotation, half-plane conjugation,
                                                         interpolation, field-offset phase,
                                                         subtract / divide / replace

Discrete choices (grid cell of a component, kernel-table row, window start)
follow the reference's single-precision arithmetic step by step (numpy float32
scalars round every operation as C float does), so that they match the
reference exactly; the FFT and the interpolation sums are FP64.  The kernel
table is the reference's: 201 rows tabulated every 0.005 cell, selected with
an offset of one row, so that the interpolated point lies 0.005 cell below the
exact one (plus up to 0.0025 cell of tabulation step) -- the reference's own
accuracy, which the test bounds against the DFT oracle account for.

Only tests, the smoke check and bench.py's CPU-baseline leg import this module;
the product never does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

F32 = np.float32
OVERSAMPLE = 2          # ObitSkyModel.c:71
HWIDTH = 12             # ObitSkyModel.c:75
IWID = 2 * HWIDTH + 1
G_PI = math.pi
GAUSS_TYPES = (1, 2, 11, 12, 21, 22)     # OBIT_CC_(C)GaussMod(Spec|TSpec)
DISK_TYPES = (4, 14, 24)                 # OBIT_CC_expDiskMod*
SPHERE_TYPES = (3, 13, 23)               # OBIT_CC_USphereMod*


@dataclass
class GridImage:
    """The image keywords the gridded model reads besides those of CCField."""

    nx: int          # pixels along the RA axis (inaxes)
    ny: int          # pixels along the declination axis
    crpixX: float    # reference pixel, 1-relative
    crpixY: float


# ---- ObitTableCCUtilGrid ----------------------------------------------------


def grid_comps(field, image: GridImage, factor: float = 1.0, minFlux: float = 0.0,
               maxGrid: float = 1e20, noNeg: bool = False):
    """ObitTableCCUtilGrid (ObitTableCCUtil.c:106-302): returns (grid float32
    (ny2, nx2), ncomp, gparm float32[3], bad-cell count).  field: CCField."""
    nx = OVERSAMPLE * image.nx
    ny = OVERSAMPLE * image.ny
    grid = np.zeros((ny, nx), F32)
    cdx, cdy = F32(field.cdeltX), F32(field.cdeltY)
    fNx, fNy = float(F32(nx)), float(F32(ny))
    minX = F32((-fNx / 2.0) * abs(float(cdx)))
    maxX = F32(((fNx / 2.0) - 1.0) * abs(float(cdx)))
    minY = F32((-fNy / 2.0) * abs(float(cdy)))
    maxY = F32(((fNy / 2.0) - 1.0) * abs(float(cdy)))
    iCellX = F32(1.0 / float(cdx)) if cdx != 0 else F32(1.0)
    iCellY = F32(1.0 / float(cdy)) if cdy != 0 else F32(1.0)
    xpoff = F32(F32(F32(image.crpixX) - F32(image.nx // 2)) - F32(1)) * cdx
    ypoff = F32(F32(F32(image.crpixY) - F32(image.ny // 2)) - F32(1)) * cdy
    flux = np.asarray(field.flux, F32)
    dX = np.asarray(field.deltaX, F32)
    dY = np.asarray(field.deltaY, F32)
    parms = None if field.parms is None else np.asarray(field.parms, F32)
    nrow = len(flux)
    first = field.startComp if field.startComp > 0 else 1
    last = field.endComp if field.endComp > 0 else nrow
    last = min(last, nrow)
    gparm = np.full(3, -1.0, F32)
    is_gauss = False
    count = bad = 0
    fac = F32(factor)
    for j in range(first, last + 1):
        k = j - 1
        if j == first and parms is not None and parms.shape[1] >= 4:
            mtype = int(parms[k, 3])
            if mtype in DISK_TYPES or mtype in SPHERE_TYPES:
                raise ValueError("exponential disks and uniform spheres are not gridded")
            if mtype in GAUSS_TYPES:
                gparm[:] = parms[k, :3]
                is_gauss = True
        elif is_gauss and np.any(parms[k, :3] != gparm):
            raise ValueError("All Gaussians MUST have same size")
        if noNeg and flux[k] < 0.0:
            break
        f = F32(flux[k] * fac)
        x = F32(dX[k] + xpoff)
        y = F32(dY[k] + ypoff)
        if abs(float(f)) < minFlux or f == 0.0:
            continue
        if abs(float(f)) > maxGrid:
            continue
        tx, ty = F32(x * iCellX), F32(y * iCellY)
        ix = int(float(tx) + 0.5) if tx > 0 else int(float(tx) - 0.5)
        iy = int(float(ty) + 0.5) if ty > 0 else int(float(ty) - 0.5)
        if float(tx) - ix > 0.1 or float(ty) - iy > 0.1:   # the reference's test (no abs)
            bad += 1
        x = min(maxX, max(x, minX))
        y = min(maxY, max(y, minY))
        x = F32(x * iCellX)
        y = F32(y * iCellY)
        xPix = int(float(F32(x + F32(nx // 2))) + 0.5)
        yPix = int(float(F32(y + F32(ny // 2))) + 0.5)
        # the reference's clip admits one cell past the grid's last column or
        # row (cdelt < 0); such a component is kept on the edge
        xPix = min(max(xPix, 0), nx - 1)
        yPix = min(max(yPix, 0), ny - 1)
        grid[yPix, xPix] = F32(grid[yPix, xPix] + f)
        count += 1
    return grid, count, gparm, bad


def grid_image(pixels: np.ndarray, fblank: float, factor: float = 1.0, minFlux: float = 0.0) -> np.ndarray:
    """ObitSkyModelLoadImage's grid (ObitSkyModel.c:2163-2260): ObitFArrayClip
    (values below minFlux or above 1e20 to 0, blanks kept), then ObitFArrayPad
    (ObitFArray.c:3512-3530: zero grid of twice the size, the image times
    factor added with pixel n/2 on grid pixel n by the blank-skipping
    ObitFArrayShiftAdd, then blanks to 0).  float32 (2n, 2n)."""
    p = np.asarray(pixels, F32)
    n = p.shape[0]
    assert p.shape == (n, n)
    blank = p == F32(fblank)
    clip = (~blank) & ((p < F32(minFlux)) | (p > F32(1e20)))
    v = np.where(clip, F32(0.0), p)
    v = np.where(blank, F32(0.0), (F32(factor) * v).astype(F32))
    g = np.zeros((2 * n, 2 * n), F32)
    off = n - n // 2
    g[off:off + n, off:off + n] = v
    return g


# ---- ObitSkyModelFTImage / GridFTComps ---------------------------------------


def ft_plane(grid: np.ndarray, gparm, field, image: GridImage) -> np.ndarray:
    """Quadrant swap, FP64 real-to-half-complex FFT, row swap, Gaussian taper
    and conjugate columns: the interpolator's plane, complex128
    (ny2, nx2 // 2 + 1 + HWIDTH)."""
    ny, nx = grid.shape
    g = np.roll(grid.astype(np.float64), (-(ny // 2), -(nx // 2)), axis=(0, 1))  # ObitFArray2DCenter
    F = np.fft.rfft2(g)                       # forward, exp(-2 pi i k x / n), unnormalized
    F = np.roll(F, ny // 2, axis=0)           # ObitCArray2DCenter: row r holds ky = r - ny/2
    if gparm[0] > 0.0 or gparm[1] > 0.0:
        F = F * taper(gparm, field, image, nx, ny)
    return add_conjg(F, HWIDTH)


def taper(gparm, field, image: GridImage, nx: int, ny: int) -> np.ndarray:
    """Gaussian taper of ObitSkyModelGridFTComps (ObitSkyModel.c:4291-4331) in
    its single-precision steps, float32 (ny, nx // 2 + 1)."""
    d2r = G_PI / 180.0
    r2d = 180.0 / G_PI
    dU = F32(r2d / (nx * abs(float(F32(field.cdeltX)))))
    dV = F32(r2d / (ny * abs(float(F32(field.cdeltY)))))
    konst = F32(d2r * G_PI * math.sqrt(0.5) / 1.17741022)
    xmaj = F32(F32(gparm[0]) * konst)
    xmin = F32(F32(gparm[1]) * konst)
    cpa = F32(math.cos(d2r * (90.0 + float(F32(gparm[2])))))
    spa = F32(math.sin(d2r * (90.0 + float(F32(gparm[2])))))
    b1 = -F32(F32(F32(cpa * xmaj) * F32(cpa * xmaj)) + F32(F32(spa * xmin) * F32(spa * xmin)))
    b2 = -F32(F32(F32(spa * xmaj) * F32(spa * xmaj)) + F32(F32(cpa * xmin) * F32(cpa * xmin)))
    b3 = F32(((-2.0 * float(spa)) * float(cpa)) * float(F32(F32(xmaj * xmaj) - F32(xmin * xmin))))
    nu = nx // 2 + 1
    UU = np.zeros(nu, F32)
    acc = F32(0.0)
    for j in range(nu):       # UU accumulates by repeated single-precision addition
        UU[j] = acc
        acc = F32(acc + dU)
    out = np.zeros((ny, nu), F32)
    for i in range(ny):
        VV = F32(dV * F32(i - nx // 2))
        bb2 = F32(F32(b2 * VV) * VV)
        bb3 = F32(b3 * VV)
        texp = ((b1 * UU) * UU + bb2) + bb3 * UU            # float32 arrays, left to right
        t = np.exp(texp.astype(np.float64)).astype(F32)
        out[i] = np.where(texp > F32(-14.0), t, F32(0.0))
    return out


def add_conjg(F: np.ndarray, ncc: int) -> np.ndarray:
    """ObitCArrayAddConjg (ObitCArray.c:1660-1726): ncc columns of conjugate
    values on the negative-u side; row 0 takes its values from columns
    ncc + 1 .. 2 ncc of itself, as the reference does."""
    ny, nu = F.shape
    out = np.zeros((ny, nu + ncc), F.dtype)
    out[:, ncc:] = F
    for r in range(1, ny):
        src = F[ny - r]
        for m in range(ncc):
            out[r, ncc - 1 - m] = np.conj(src[1 + m])
    for m in range(ncc):
        out[0, ncc - 1 - m] = np.conj(F[0, ncc + 1 + m])
    return out


# ---- ObitCInterpolate ---------------------------------------------------------


def kernel_table() -> np.ndarray:
    """InitConvKernal / CalcConvKernal (ObitCInterpolate.c:747-830): 201 rows of
    25 Lagrange weights in the reference's single-precision arithmetic."""
    denom = np.zeros(IWID, F32)
    for j in range(1, IWID + 1):
        prod = F32(1.0)
        for i in range(1, IWID + 1):
            if i != j:
                prod = F32(prod * F32(j - i))
        denom[j - 1] = F32(1.0 / float(prod))
    ks = F32(0.005)
    num = int(1 + (1.0 / float(ks)) + 0.5)
    tab = np.zeros((num, IWID), F32)
    for k in range(num):
        xx = F32(float(F32(F32(HWIDTH) + F32(ks * F32(k - 1)))) + 0.5)
        ipos = int(float(xx) + 0.5)
        cen = max(1, min(ipos - HWIDTH, 1024 - IWID)) - 1
        x = F32(float(F32(xx - F32(cen))) + 1.0)
        for j in range(IWID):
            prod = denom[j]
            for i in range(IWID):
                if i != j:
                    prod = F32(prod * F32(x - F32(i + 1)))
            tab[k, j] = prod
    return tab


def conv_setup(pixel: np.ndarray, naxis: int, ntab: int):
    """SetConvKernal (ObitCInterpolate.c:699-745), vectorized over float32
    pixels: (start 0-rel, first kernel tap, taps, table row)."""
    p = pixel.astype(np.float64)
    ipos = np.trunc(p + 0.5).astype(np.int64)
    cen = np.clip(ipos - HWIDTH, 1, naxis - IWID)
    off = ((pixel - cen.astype(F32)).astype(F32) - F32(HWIDTH)).astype(F32)
    o = off.astype(np.float64)
    ioff = np.where(o > 0.0, np.trunc(o + 0.5), np.trunc(o - 0.5)).astype(np.int64)
    off = (off - ioff.astype(F32)).astype(F32)
    itab = np.trunc((0.5 + off.astype(np.float64)) * ntab + 0.5).astype(np.int64)
    itab = np.clip(itab, 0, ntab)
    k0 = np.abs(ioff)
    return cen - 1, k0, IWID - k0, itab


@dataclass
class Interp:
    """The interpolator of newObitCInterpolateCreate (ObitCInterpolate.c:128-206)
    on the conjugate-extended plane."""

    plane: np.ndarray        # complex128 (ny2, nx2 // 2 + 1 + HWIDTH)
    crpix: tuple             # float32 (x, y), 1-relative
    cdelt: tuple             # float32 (x, y), wavelengths per pixel
    table: np.ndarray        # float32 (201, 25)


def make_interp(plane: np.ndarray, field, image: GridImage) -> Interp:
    ny = plane.shape[0]
    c0 = F32(1.0 / ((((-G_PI) / 180.0) * float(F32(OVERSAMPLE))) * float(F32(field.cdeltX)) * image.nx))
    c1 = F32(1.0 / ((((-G_PI) / 180.0) * float(F32(OVERSAMPLE))) * float(F32(field.cdeltY)) * image.ny))
    return Interp(plane, (F32(HWIDTH), F32(ny // 2)), (c0, c1), kernel_table())


def lagrange_weights(t: np.ndarray) -> np.ndarray:
    """FP64 weights of the 25-point Lagrange interpolant on nodes 0..24 at
    positions t (n,): (n, 25)."""
    nodes = np.arange(IWID, dtype=np.float64)
    w = np.ones((len(t), IWID))
    for j in range(IWID):
        for k in range(IWID):
            if k != j:
                w[:, j] *= (t - nodes[k]) / (j - k)
    return w


def interpolate(ip: Interp, u: np.ndarray, v: np.ndarray, chunk: int = 8192, exact: bool = False):
    """ObitCInterpolateOffset at float32 offsets (u, v): complex128 values,
    NaN where the reference returns its blank (outside the plane, or weight
    sum <= 0.5).  exact: 25-point Lagrange weights at the requested point
    itself (0-relative plane position = the reference's 1-relative pixel),
    the window centred on it; a point whose window would leave the plane is
    blanked."""
    ny, nxp = ip.plane.shape
    ntab = ip.table.shape[0] - 1
    px = (ip.crpix[0] + (u / ip.cdelt[0]).astype(F32)).astype(F32)
    py = (ip.crpix[1] + (v / ip.cdelt[1]).astype(F32)).astype(F32)
    out = np.full(u.shape, np.nan + 0j)
    inside = (px >= 1.0) & (px <= nxp) & (py >= 1.0) & (py <= ny)
    idx = np.nonzero(inside)[0]
    tab = ip.table.astype(np.float64)
    ar = np.arange(IWID)
    for s in range(0, len(idx), chunk):
        ii = idx[s:s + chunk]
        if exact:
            X, Y = px[ii].astype(np.float64), py[ii].astype(np.float64)
            sx = np.floor(px[ii].astype(np.float32) + np.float32(0.5)).astype(np.int64) - HWIDTH
            sy = np.floor(py[ii].astype(np.float32) + np.float32(0.5)).astype(np.int64) - HWIDTH
            fits = (sx >= 0) & (sx + IWID <= nxp) & (sy >= 0) & (sy + IWID <= ny)
            sx, sy = np.clip(sx, 0, nxp - IWID), np.clip(sy, 0, ny - IWID)
            wx = lagrange_weights(X - sx) * fits[:, None]
            wy = lagrange_weights(Y - sy) * fits[:, None]
        else:
            sx, k0x, ntx, tx = conv_setup(px[ii], nxp, ntab)
            sy, k0y, nty, ty = conv_setup(py[ii], ny, ntab)
            wx = tab[tx[:, None], np.minimum(k0x[:, None] + ar, IWID - 1)] * (ar < ntx[:, None])
            wy = tab[ty[:, None], np.minimum(k0y[:, None] + ar, IWID - 1)] * (ar < nty[:, None])
        cols = np.minimum(sx[:, None] + ar, nxp - 1)
        rows = np.minimum(sy[:, None] + ar, ny - 1)
        win = ip.plane[rows[:, :, None], cols[:, None, :]]          # (n, 25, 25)
        s_ = np.einsum("nj,nji,ni->n", wy, win, wx)
        sw = wy.sum(1) * wx.sum(1)
        val = np.where(sw > 0.5, s_ / np.where(sw > 0.5, sw, 1.0), np.nan)
        out[ii] = val
    return out


# ---- field geometry (ThreadSkyModelFTGrid set-up) ------------------------------


def shift_sin(ra, dec, rotate, xra, xdec):
    """ObitSkyGeomShiftSIN (ObitSkyGeom.c:177-205): float32 2 pi (l, m, n - 1)."""
    maprr = F32(float(F32(rotate)) * G_PI / 180.0)
    d2r = G_PI / 180.0
    xx = math.cos(d2r * xdec) * math.sin(d2r * (xra - ra))
    yy = math.sin(d2r * xdec) * math.cos(d2r * dec) - \
        math.cos(d2r * xdec) * math.sin(d2r * dec) * math.cos(d2r * (xra - ra))
    xs = F32(math.cos(float(maprr)) * xx + math.sin(float(maprr)) * yy)
    ys = F32(-math.sin(float(maprr)) * xx + math.cos(float(maprr)) * yy)
    dz = math.sqrt(1.0 - float(F32(xs * xs)) - float(F32(ys * ys)))
    return np.array([2.0 * G_PI * float(xs), 2.0 * G_PI * float(ys), 2.0 * G_PI * (dz - 1.0)], F32)


def _rot(r, sign):
    m = np.zeros((3, 3))
    m[2, 2] = 1.0
    m[0, 0] = m[1, 1] = math.cos(r)
    m[1, 0] = -sign * math.sin(r)
    m[0, 1] = sign * math.sin(r)
    return m


def shift3d_matrices(ra, dec, xra, xdec, mrot, urot):
    """ObitUVDescShift3DMatrix, 3-D branch (ObitUVDesc.c:913-1020): float32
    URot3D and PRot3D, indexed [j][i] as the reference stores them."""
    d2r = G_PI / 180.0
    sa, ca = math.sin(d2r * (xra - ra)), math.cos(d2r * (xra - ra))
    sd, cd = math.sin(d2r * xdec), math.cos(d2r * xdec)
    sd0, cd0 = math.sin(d2r * dec), math.cos(d2r * dec)

    def prod(x, rm1, rm2):
        t = np.zeros((3, 3))
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    t[j][i] += x[k][i] * rm1[j][k]
        out = np.zeros((3, 3))
        for i in range(3):
            for j in range(3):
                r = 0.0
                for k in range(3):
                    r += rm2[k][i] * t[j][k]
                out[j][i] = r
        return out.astype(F32)

    x = np.zeros((3, 3))
    x[0][0], x[1][0], x[2][0] = ca, -sd * sa, cd * sa
    x[0][1], x[1][1], x[2][1] = sd0 * sa, cd * cd0 + sd * sd0 * ca, sd * cd0 - cd * sd0 * ca
    x[0][2], x[1][2], x[2][2] = -cd0 * sa, cd * sd0 - sd * cd0 * ca, sd * sd0 + cd * cd0 * ca
    U = prod(x, _rot(d2r * float(F32(mrot)), 1.0), _rot(d2r * float(F32(urot)), -1.0))
    x = np.zeros((3, 3))
    x[0][0], x[1][0], x[2][0] = ca, sd0 * sa, -cd0 * sa
    x[0][1], x[1][1], x[2][1] = -sd * sa, cd * cd0 + sd * sd0 * ca, sd0 * cd - cd0 * sd * ca
    x[0][2], x[1][2], x[2][2] = cd * sa, cd0 * sd - sd0 * cd * ca, sd * sd0 + cd * cd0 * ca
    P = prod(x, _rot(d2r * float(F32(urot)), 1.0), _rot(d2r * float(F32(mrot)), -1.0))
    return U, P


@dataclass
class GridGeom:
    flip: float
    do3Dmul: bool
    umat: np.ndarray
    doRot: bool
    ccrot: np.float32
    ssrot: np.float32
    doPC: bool
    dxyzc: np.ndarray


def field_geometry(field, model) -> GridGeom:
    """The set-up of ThreadSkyModelFTGrid (ObitSkyModel.c:3037-3101) for a
    -SIN field: 3-D images, and 2-D images centred on the uv phase centre
    without rotation or pixel offset."""
    maprot, uvrot = float(F32(field.rotation)), float(F32(model.uvRotation))
    d2r = G_PI / 180.0
    ssrot = F32(math.sin(d2r * float(F32(uvrot - maprot))))
    ccrot = F32(math.cos(d2r * float(F32(uvrot - maprot))))
    flip = -1.0 if field.cdeltX > 0.0 else 1.0
    dxyzc = shift_sin(model.uvRA, model.uvDec, maprot, field.crvalRA, field.crvalDec)
    doPC = bool(np.any(np.abs(dxyzc.astype(np.float64)) > 1e-12))
    do3Dmul = False
    umat = np.eye(3, dtype=F32)
    if model.do3D:
        do3Dmul = (maprot != 0.0 or uvrot != 0.0 or abs(field.crvalRA - model.uvRA) > 1e-10 or
                   abs(field.crvalDec - model.uvDec) > 1e-10 or abs(field.xPxOff) > 1e-20 or
                   abs(field.yPxOff) > 1e-20)
        umat, pmat = shift3d_matrices(model.uvRA, model.uvDec, field.crvalRA, field.crvalDec, maprot, uvrot)
        if doPC:
            rmat = np.zeros((3, 3), F32)
            rmat[0][0], rmat[1][0], rmat[2][0] = ccrot, ssrot, 0.0
            rmat[0][1], rmat[1][1], rmat[2][1] = -ssrot, ccrot, 0.0
            rmat[2][2] = 1.0
            dmat = np.zeros((3, 3), F32)
            for i in range(3):
                for j in range(3):
                    acc = F32(0.0)
                    for k in range(3):
                        acc = F32(acc + F32(pmat[k][i] * rmat[j][k]))
                    dmat[j][i] = acc
            d = dxyzc
            t = [F32(F32(F32(d[0] * dmat[0][c]) + F32(d[1] * dmat[1][c])) + F32(d[2] * dmat[2][c]))
                 for c in range(3)]
            dxyzc = np.array(t, F32)
    doRot = abs(float(ssrot)) > 1e-10 or abs(float(ccrot) - 1.0) > 1e-4
    return GridGeom(flip, do3Dmul, umat, doRot, ccrot, ssrot, doPC, dxyzc)


# ---- the per-visibility loop ---------------------------------------------------


@dataclass
class GridModel:
    interp: Interp
    geom: GridGeom
    ncomp: int
    l1: float               # sum of |flux| gridded (bound of every plane value)


def build(field, image: GridImage, model, maxGrid: float = 1e20) -> GridModel:
    """ObitSkyModelLoadGridComps + ObitSkyModelGridFTComps for one field."""
    grid, ncomp, gparm, _ = grid_comps(field, image, model.factor, model.minFlux, maxGrid, model.noNeg)
    plane = ft_plane(grid, gparm, field, image)
    return GridModel(make_interp(plane, field, image), field_geometry(field, model), ncomp,
                     float(np.abs(grid.astype(np.float64)).sum()))


def build_image(pixels, fblank, field, image: GridImage, model) -> GridModel:
    """ObitSkyModelLoadImage for one field: the image model's interpolator."""
    grid = grid_image(pixels, fblank, model.factor, model.minFlux)
    plane = ft_plane(grid, np.full(3, -1.0, F32), field, image)
    return GridModel(make_interp(plane, field, image), field_geometry(field, model), grid.size // 4,
                     float(np.abs(grid.astype(np.float64)).sum()))


def model_values(gm: GridModel, uv, params=None, exact: bool = False):
    """The complex model of every (record, IF, channel) the reference's grid
    path forms before it touches the data (after conjugating back and doFlip);
    NaN where it blanks.  Returns complex128 (nvis, nif, nchan).  exact: the
    Lagrange weights at the requested point (see interpolate)."""
    from obit_b200.skymodel import SkyModelParams
    p = params or SkyModelParams()
    g = gm.geom
    fs = uv.fscale.reshape(uv.nif, uv.nchan)                    # float32, kincf = 1, kincif = nchan
    rec = uv.vis.astype(F32)
    u0 = rec[:, uv.ilocu][:, None, None]
    v0 = rec[:, uv.ilocv][:, None, None]
    w0 = rec[:, uv.ilocw][:, None, None]
    u = (fs[None] * u0).astype(F32)
    v = (fs[None] * v0).astype(F32)
    w = (fs[None] * w0).astype(F32)
    if g.do3Dmul:
        m = g.umat
        ut = ((u * m[0][0]).astype(F32) + (v * m[0][1]).astype(F32)).astype(F32) + (w * m[0][2]).astype(F32)
        vt = ((u * m[1][0]).astype(F32) + (v * m[1][1]).astype(F32)).astype(F32) + (w * m[1][2]).astype(F32)
        wt = ((u * m[2][0]).astype(F32) + (v * m[2][1]).astype(F32)).astype(F32) + (w * m[2][2]).astype(F32)
        u, v, w = ut.astype(F32), vt.astype(F32), wt.astype(F32)
    elif g.doRot:
        ut = ((g.ccrot * u).astype(F32) - (g.ssrot * v).astype(F32)).astype(F32)
        vt = ((g.ccrot * v).astype(F32) + (g.ssrot * u).astype(F32)).astype(F32)
        u, v = ut, vt
    conj = (F32(g.flip) * u) < 0.0
    u = np.where(conj, -u, u).astype(F32)
    v = np.where(conj, -v, v).astype(F32)
    w = np.where(conj, -w, w).astype(F32)
    val = interpolate(gm.interp, u.ravel(), v.ravel(), exact=exact).reshape(u.shape)
    if g.doPC:
        d = g.dxyzc
        pc = (((u * d[0]).astype(F32) + (v * d[1]).astype(F32)).astype(F32) + (w * d[2]).astype(F32)).astype(F32)
        val = val * np.exp(1j * pc.astype(np.float64))
    val = np.where(conj, np.conj(val), val)
    if p.doFlip:
        val = 1j * val
    return val


def apply(gm: GridModel, uv, params=None, exact: bool = False) -> np.ndarray:
    """ThreadSkyModelFTGrid's operation on a copy of the records (float32),
    with the model of model_values in FP64."""
    from obit_b200.skymodel import OP_DIV, OP_REPL, SkyModelParams
    p = params or SkyModelParams()
    out = uv.vis.astype(F32).copy()
    val = model_values(gm, uv, p, exact=exact)
    c0 = (p.startChannel if p.startChannel > 0 else 1) - 1
    nc = p.numberChannel if p.numberChannel > 0 else uv.nchan - c0
    i0 = (p.startIF if p.startIF > 0 else 1) - 1
    ni = p.numberIF if p.numberIF > 0 else uv.nif - i0
    s0 = (p.startPoln if p.startPoln > 0 else 1) - 1
    ns = p.numberPoln if p.numberPoln > 0 else min(2, uv.nstok)
    vv = out[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    for iv in range(uv.nvis):
        for ii in range(i0, i0 + ni):
            for ic in range(c0, c0 + nc):
                m = val[iv, ii, ic]
                bad = np.isnan(m)
                wt = 1.0
                if p.op == OP_DIV and not bad:
                    wt = abs(m) ** 2
                    m = m / wt
                    wt = math.sqrt(wt)
                for s in range(s0, s0 + ns):
                    c = vv[iv, ii, ic, s]
                    if c[2] <= 0.0 and p.op != OP_REPL:
                        continue
                    if bad:
                        c[:] = 0.0
                    elif p.op == OP_DIV:
                        d = complex(c[0], c[1]) * np.conj(m)
                        c[0], c[1] = d.real, d.imag
                        c[2] = c[2] * wt
                    elif p.op == OP_REPL:
                        c[0], c[1] = m.real, m.imag
                    else:
                        c[0] -= m.real
                        c[1] -= m.imag
                    m = m * p.stokFactor
    return out


def choose_mode(model_mode: int, model_type: int, ncc, nx, ny, nvis: int, nchan: int) -> int:
    """ObitSkyModelChose (ObitSkyModel.c:3560-3620): 1 (DFT) or 2 (grid).
    model_mode 0 = fastest, 1 = DFT, 2 = grid; model_type 0 components,
    1 image, 2 point."""
    if model_mode != 0:
        return model_mode
    if model_type == 2:
        return 1
    tpvgrd, tfft, tpcgrd, tpvpc = F32(1.0e-5), F32(0.8e-6), F32(1.0e-4), F32(6.6e-7)
    sumcc = t1 = t2 = t3 = 0
    for n, a, b in zip(ncc, nx, ny):
        if n > 0:
            x = 4 if not (a > 2048 or b > 2048) else 2
            sumcc += n
            t1 += nvis
            t2 += x * a * b
            t3 += n
    timfft = F32(F32(F32(F32(t1) * tpvgrd) + F32(F32(t2) * tfft)) + F32(F32(t3) * tpcgrd)) * F32(nchan)
    timfft = F32(timfft * F32(0.5))
    timdft = F32(F32(F32(tpvpc * F32(nvis)) * F32(sumcc)) * F32(nchan))
    mode = 1 if timdft <= timfft else 2
    if model_type == 1:
        mode = 2
    return mode


# ---- the single-precision C restatement (refcpu_grid.c) -------------------------

import ctypes as _C  # noqa: E402


class RefGridJob(_C.Structure):
    _fields_ = [
        ("plane", _C.POINTER(_C.c_float)), ("nxp", _C.c_int), ("ny", _C.c_int),
        ("table", _C.POINTER(_C.c_float)), ("ntab", _C.c_int),
        ("crpix0", _C.c_float), ("crpix1", _C.c_float), ("cdelt0", _C.c_float), ("cdelt1", _C.c_float),
        ("flip", _C.c_float), ("do3Dmul", _C.c_int), ("umat", _C.c_float * 9), ("doRot", _C.c_int),
        ("ccrot", _C.c_float), ("ssrot", _C.c_float), ("doPC", _C.c_int), ("dxyzc", _C.c_float * 3),
        ("lrec", _C.c_int), ("nrparm", _C.c_int), ("ilocu", _C.c_int), ("ilocv", _C.c_int),
        ("ilocw", _C.c_int), ("fscale", _C.POINTER(_C.c_float)), ("kincf", _C.c_int), ("kincif", _C.c_int),
        ("chanb", _C.c_int), ("nchan", _C.c_int), ("ifb", _C.c_int), ("nif", _C.c_int),
        ("incf", _C.c_int), ("incif", _C.c_int), ("incs", _C.c_int), ("stokb", _C.c_int),
        ("nstok", _C.c_int), ("doDivide", _C.c_int), ("doReplace", _C.c_int), ("doFlip", _C.c_int),
        ("stokFactor", _C.c_float),
    ]


def _lib_c():
    import oracle
    lib = oracle.lib_a()
    if not getattr(lib, "_grid_bound", False):
        lib.refcpu_grid_apply.restype = _C.c_int
        lib.refcpu_grid_apply.argtypes = [_C.POINTER(RefGridJob), _C.POINTER(_C.c_float), _C.c_long, _C.c_int]
        lib._grid_bound = True
    return lib


class CJob:
    """A RefGridJob for a GridModel, a record layout and SkyModelParams, with
    the arrays it points into."""

    def __init__(self, gm: GridModel, uv, params=None):
        from obit_b200.skymodel import OP_DIV, OP_REPL, SkyModelParams
        p = params or SkyModelParams()
        j = RefGridJob()
        self.plane = np.ascontiguousarray(gm.interp.plane.astype(np.complex64))
        self.table = np.ascontiguousarray(gm.interp.table, dtype=F32)
        self.fscale = np.ascontiguousarray(uv.fscale, dtype=F32)
        j.plane = self.plane.view(F32).ctypes.data_as(_C.POINTER(_C.c_float))
        j.ny, j.nxp = self.plane.shape
        j.table = self.table.ctypes.data_as(_C.POINTER(_C.c_float))
        j.ntab = self.table.shape[0] - 1
        j.crpix0, j.crpix1 = gm.interp.crpix
        j.cdelt0, j.cdelt1 = gm.interp.cdelt
        g = gm.geom
        j.flip, j.do3Dmul, j.doRot, j.doPC = g.flip, int(g.do3Dmul), int(g.doRot), int(g.doPC)
        for i in range(9):
            j.umat[i] = float(g.umat.ravel()[i])
        j.ccrot, j.ssrot = float(g.ccrot), float(g.ssrot)
        for i in range(3):
            j.dxyzc[i] = float(g.dxyzc[i])
        j.lrec, j.nrparm, j.ilocu, j.ilocv, j.ilocw = uv.lrec, uv.nrparm, uv.ilocu, uv.ilocv, uv.ilocw
        j.fscale = self.fscale.ctypes.data_as(_C.POINTER(_C.c_float))
        j.kincf, j.kincif = uv.kincf, uv.kincif
        c0 = (p.startChannel if p.startChannel > 0 else 1) - 1
        i0 = (p.startIF if p.startIF > 0 else 1) - 1
        s0 = (p.startPoln if p.startPoln > 0 else 1) - 1
        j.chanb, j.nchan = c0, p.numberChannel if p.numberChannel > 0 else uv.nchan - c0
        j.ifb, j.nif = i0, p.numberIF if p.numberIF > 0 else uv.nif - i0
        j.stokb, j.nstok = s0, p.numberPoln if p.numberPoln > 0 else min(2, uv.nstok)
        j.incf, j.incif, j.incs = uv.incf, uv.incif, uv.incs
        j.doDivide, j.doReplace, j.doFlip = int(p.op == OP_DIV), int(p.op == OP_REPL), int(p.doFlip)
        j.stokFactor = p.stokFactor
        self.job = j


def apply_c(gm: GridModel, uv, params=None, nthreads: int = 1, vis: np.ndarray | None = None) -> np.ndarray:
    """refcpu_grid_apply on a copy of the records (or in place on `vis`)."""
    jb = CJob(gm, uv, params)
    out = np.ascontiguousarray(uv.vis, dtype=F32).copy() if vis is None else vis
    rc = _lib_c().refcpu_grid_apply(_C.byref(jb.job), out.ctypes.data_as(_C.POINTER(_C.c_float)),
                                    out.shape[0], int(nthreads))
    if rc:
        raise ValueError(f"refcpu_grid_apply returned {rc}")
    return out
