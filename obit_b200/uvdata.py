"""Obit-layout visibility buffers and component tables, and seeded synthetic
workloads of the shapes the DFT path is measured on.

Record layout (ObitUVDesc, ObitSystem/Obit/src/ObitUVDesc.c:370-452): `nrparm`
random parameters (u, v, w in wavelengths at the reference frequency, then
baseline and time) followed by {re, im, weight} per correlation, with the
regular axes ordered COMPLEX, STOKES, FREQ, IF.  Channel frequencies follow
ObitUVDescGetFreq (ObitUVDesc.c:506-617): per IF, nu = nu_IF + (ch + 1 - crpix)
* dnu, and fscale = nu / nu_ref in FP32.

Component tables use the reference field order (ObitSkyModel.c:1965-2063,
ObitSkyModelMF.c:1497-1514):
  point        [flux, X, Y, Z]
  point+spec   [flux, X, Y, Z, a_1..a_nterm]
  point+tspec  [flux, X, Y, Z, alpha, S_plane0..]
  gauss        [flux, X, Y, Z, g1, g2, g3]
  gauss+spec   [flux, X, Y, Z, g1, g2, g3, a_1..a_nterm]
  gauss+tspec  [flux, X, Y, Z, g1, g2, g3, alpha, S_plane0..]
with X, Y, Z = 2 pi (l, m, n - 1) and g1..g3 from the FWHM/PA formula of
ObitSkyModelLoadComps (ObitSkyModel.c:1719-1722, 1938-1947).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C_LIGHT = 299792458.0
DG2RAD = math.pi / 180.0

# ObitSkyModelCompType numbering (ObitSkyModel.h:130-164)
MOD_POINT, MOD_GAUSS = 0, 1
MOD_POINT_SPEC, MOD_GAUSS_SPEC = 10, 11
MOD_POINT_TSPEC, MOD_GAUSS_TSPEC = 20, 21
# GPUModType numbering (ObitCUDASkyModelInfoDef.h:44-52)
GPU_TYPE = {MOD_POINT: 0, MOD_POINT_SPEC: 1, MOD_POINT_TSPEC: 2, MOD_GAUSS: 3,
            MOD_GAUSS_SPEC: 4, MOD_GAUSS_TSPEC: 5}


@dataclass
class UVData:
    """A buffer of Obit random-group records plus its descriptor fields."""

    vis: np.ndarray          # float32 (nvis, lrec)
    nstok: int
    nchan: int
    nif: int
    freq: float              # reference frequency, Hz
    freqArr: np.ndarray      # float64 Hz, index ichan*kincf + iIF*kincif
    crval_stokes: float = -1.0
    nrparm: int = 5
    ilocu: int = 0
    ilocv: int = 1
    ilocw: int = 2

    @property
    def nvis(self) -> int:
        return self.vis.shape[0]

    @property
    def lrec(self) -> int:
        return self.vis.shape[1]

    @property
    def ncorr(self) -> int:
        return self.nstok * self.nchan * self.nif

    # axis order COMPLEX(0), STOKES(1), FREQ(2), IF(3)
    jlocs, jlocf, jlocif = 1, 2, 3

    @property
    def incs(self) -> int:
        return 3

    @property
    def incf(self) -> int:
        return 3 * self.nstok

    @property
    def incif(self) -> int:
        return 3 * self.nstok * self.nchan

    # frequency-table increments (frequency axis before IF: ObitGPUSkyModel.c:263-275)
    kincf = 1

    @property
    def kincif(self) -> int:
        return self.nchan

    @property
    def fscale(self) -> np.ndarray:
        return (self.freqArr / self.freq).astype(np.float32)

    def copy(self) -> "UVData":
        return UVData(self.vis.copy(), self.nstok, self.nchan, self.nif, self.freq,
                      self.freqArr.copy(), self.crval_stokes, self.nrparm, self.ilocu,
                      self.ilocv, self.ilocw)

    def rows(self, lo: int, hi: int) -> "UVData":
        return UVData(self.vis[lo:hi].copy(), self.nstok, self.nchan, self.nif, self.freq,
                      self.freqArr, self.crval_stokes, self.nrparm, self.ilocu, self.ilocv,
                      self.ilocw)

    def vis_view(self) -> np.ndarray:
        """(nvis, nif, nchan, nstok, 3) view of the correlations."""
        return self.vis[:, self.nrparm:].reshape(self.nvis, self.nif, self.nchan, self.nstok, 3)


@dataclass
class SkyComps:
    """A CLEAN-component table in the reference field order."""

    modType: int             # ObitSkyModelCompType
    comps: np.ndarray        # float32 (ncomp, lcomp)
    nterm: int = 0           # spectral terms (Spec types)
    refFreq: float = 0.0     # reference frequency of polynomial spectra, Hz
    specFreq: np.ndarray | None = None   # coarse-plane frequencies (TSpec), Hz
    specIndex: np.ndarray | None = None  # plane per (chan, IF) (TSpec)
    xyz: np.ndarray | None = None        # FP64 X, Y, Z per component (ncomp, 3), if known

    @property
    def ncomp(self) -> int:
        return self.comps.shape[0]

    @property
    def lcomp(self) -> int:
        return self.comps.shape[1]

    @property
    def gpu_type(self) -> int:
        return GPU_TYPE[self.modType]

    @property
    def is_tspec(self) -> bool:
        return self.modType in (MOD_POINT_TSPEC, MOD_GAUSS_TSPEC)

    @property
    def nspec(self) -> int:
        return 0 if self.specFreq is None else len(self.specFreq)


# ---- frequency axes ----------------------------------------------------------


def freq_axis(nchan: int, nif: int, f_first: float, dnu: float, if_step: float | None = None):
    """Channel frequencies (Hz) in data order: IF-major blocks of nchan, as
    ObitUVDescGetFreq fills freqArr when FREQ precedes IF."""
    if if_step is None:
        if_step = nchan * dnu
    f = np.empty(nchan * nif, dtype=np.float64)
    for i in range(nif):
        f[i * nchan:(i + 1) * nchan] = f_first + i * if_step + np.arange(nchan) * dnu
    return f


# ---- uvw -------------------------------------------------------------------


def array_layout(nant: int, max_baseline_m: float, rng: np.random.Generator) -> np.ndarray:
    """Random east-west arm plus north arm; local (east, north, up) metres."""
    n_ew = nant - nant // 3
    n_n = nant - n_ew
    half = 0.5 * max_baseline_m
    ew = np.sort(rng.uniform(-half, half, n_ew))
    ew[0], ew[-1] = -half, half
    north = np.sort(rng.uniform(0.0, half, n_n))
    pos = np.zeros((nant, 3))
    pos[:n_ew, 0] = ew
    pos[n_ew:, 1] = north
    return pos


def make_uvw(pos_enu: np.ndarray, nint: int, dec_deg: float, ha_hours: float,
             lat_deg: float, freq: float) -> np.ndarray:
    """(nint * nbl, 3) u, v, w in wavelengths at `freq`, time-major (Obit 'TB')."""
    lat = lat_deg * DG2RAD
    e, n, u_ = pos_enu[:, 0], pos_enu[:, 1], pos_enu[:, 2]
    X = -math.sin(lat) * n + math.cos(lat) * u_
    Y = e
    Z = math.cos(lat) * n + math.sin(lat) * u_
    xyz = np.stack([X, Y, Z], axis=1)
    nant = len(pos_enu)
    a1, a2 = np.triu_indices(nant, k=1)
    b = xyz[a2] - xyz[a1]
    lam = C_LIGHT / freq
    dec = dec_deg * DG2RAD
    has = np.linspace(-ha_hours, ha_hours, nint) * (math.pi / 12.0)
    out = np.empty((nint, len(a1), 3))
    for i, H in enumerate(has):
        sH, cH = math.sin(H), math.cos(H)
        sd, cd = math.sin(dec), math.cos(dec)
        out[i, :, 0] = sH * b[:, 0] + cH * b[:, 1]
        out[i, :, 1] = -sd * cH * b[:, 0] + sd * sH * b[:, 1] + cd * b[:, 2]
        out[i, :, 2] = cd * cH * b[:, 0] - cd * sH * b[:, 1] + sd * b[:, 2]
    return (out / lam).reshape(-1, 3)


def make_uvdata(uvw: np.ndarray, nstok: int, nchan: int, nif: int, freq: float,
                freqArr: np.ndarray, rng: np.random.Generator, noise: float = 0.01,
                flag_frac: float = 0.0) -> UVData:
    nvis = uvw.shape[0]
    nrparm = 5
    ncorr = nstok * nchan * nif
    vis = np.empty((nvis, nrparm + 3 * ncorr), dtype=np.float32)
    vis[:, 0:3] = uvw.astype(np.float32)
    vis[:, 3] = 256.0  # baseline code placeholder
    vis[:, 4] = 0.0    # time placeholder
    c = vis[:, nrparm:].reshape(nvis, ncorr, 3)
    c[:, :, 0] = rng.normal(0.0, noise, size=(nvis, ncorr)).astype(np.float32)
    c[:, :, 1] = rng.normal(0.0, noise, size=(nvis, ncorr)).astype(np.float32)
    c[:, :, 2] = 1.0
    if flag_frac > 0:
        m = rng.random((nvis, ncorr)) < flag_frac
        c[:, :, 2][m] = -1.0
    return UVData(vis, nstok, nchan, nif, freq, freqArr)


# ---- components --------------------------------------------------------------


def lm_disk(n: int, radius_deg: float, rng: np.random.Generator, center=(0.0, 0.0)):
    r = radius_deg * DG2RAD * np.sqrt(rng.random(n))
    th = rng.uniform(0, 2 * math.pi, n)
    return center[0] + r * np.cos(th), center[1] + r * np.sin(th)


def xyz_from_lm(l: np.ndarray, m: np.ndarray):
    n = np.sqrt(1.0 - l * l - m * m)
    return 2 * math.pi * l, 2 * math.pi * m, 2 * math.pi * (n - 1.0)


def gauss_coeffs(maj_deg, min_deg, pa_deg):
    """g1, g2, g3 of ObitSkyModelLoadComps (ObitSkyModel.c:1722, 1938-1947)."""
    konst2 = DG2RAD * math.sqrt(2.0) * math.pi / 2.35482044
    cpa = np.cos(DG2RAD * pa_deg)
    spa = np.sin(DG2RAD * pa_deg)
    xmaj = maj_deg * konst2
    xmin = min_deg * konst2
    g1 = -((cpa * xmaj) ** 2 + (spa * xmin) ** 2)
    g2 = -((spa * xmaj) ** 2 + (cpa * xmin) ** 2)
    g3 = -2.0 * cpa * spa * (xmaj * xmaj - xmin * xmin)
    return g1, g2, g3


def make_comps(modType: int, n: int, rng: np.random.Generator, radius_deg: float = 0.5,
               flux=(1e-3, 1.0), alpha=(-1.5, 0.5), nterm: int = 1, center=(0.0, 0.0),
               gauss_frac: float = 1.0, maj_arcsec=(1.0, 60.0), ratio=(0.3, 1.0),
               ref_freq: float = 1.4e9, spec_freq=None, spec_index=None) -> SkyComps:
    l, m = lm_disk(n, radius_deg, rng, center)
    X, Y, Z = xyz_from_lm(l, m)
    S = np.exp(rng.uniform(math.log(flux[0]), math.log(flux[1]), n))
    cols = [S, X, Y, Z]
    gauss = modType in (MOD_GAUSS, MOD_GAUSS_SPEC, MOD_GAUSS_TSPEC)
    if gauss:
        maj = rng.uniform(maj_arcsec[0], maj_arcsec[1], n) / 3600.0
        mn = maj * rng.uniform(ratio[0], ratio[1], n)
        pa = rng.uniform(0.0, 180.0, n)
        g1, g2, g3 = gauss_coeffs(maj, mn, pa)
        is_g = rng.random(n) < gauss_frac
        cols += [np.where(is_g, g1, 0.0), np.where(is_g, g2, 0.0), np.where(is_g, g3, 0.0)]
    if modType in (MOD_POINT_SPEC, MOD_GAUSS_SPEC):
        a = rng.uniform(alpha[0], alpha[1], n)
        cols.append(a)
        for _ in range(1, nterm):
            cols.append(rng.uniform(-0.1, 0.1, n))
    if modType in (MOD_POINT_TSPEC, MOD_GAUSS_TSPEC):
        a = rng.uniform(alpha[0], alpha[1], n)
        cols.append(a)
        sf = np.asarray(spec_freq)
        for f in sf:
            cols.append(S * (f / ref_freq) ** a)
    comps = np.stack(cols, axis=1).astype(np.float32)
    # order by decreasing flux, as merged CC tables are (ObitTableCCUtil.c:1238-1361)
    order = np.argsort(-np.abs(comps[:, 0]), kind="stable")
    comps = comps[order]
    xyz = np.stack([X, Y, Z], axis=1)[order]
    return SkyComps(modType, np.ascontiguousarray(comps), xyz=np.ascontiguousarray(xyz),
                    nterm=nterm if modType in (MOD_POINT_SPEC, MOD_GAUSS_SPEC) else 0,
                    refFreq=ref_freq, specFreq=None if spec_freq is None else np.asarray(spec_freq, np.float64),
                    specIndex=None if spec_index is None else np.asarray(spec_index, np.int32))


# ---- named workloads ---------------------------------------------------------


@dataclass
class Workload:
    name: str
    uv: UVData
    sky: SkyComps
    notes: dict = field(default_factory=dict)

    @property
    def evals(self) -> int:
        """Component-visibility evaluations: components x rows x channels x IFs."""
        return int(self.sky.ncomp) * self.uv.nvis * self.uv.nchan * self.uv.nif


def config1(nint: int = 120, ncomp: int = 1000, seed: int = 1) -> Workload:
    """27 antennas (351 baselines) x nint integrations, 1 IF x 64 channels of
    1 MHz about 1.4 GHz, RR/LL, 1000 points within 0.5 deg."""
    rng = np.random.default_rng(seed)
    pos = array_layout(27, 36e3, rng)
    freq = 1.4e9
    fa = freq_axis(64, 1, freq - 32e6, 1e6)
    uvw = make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)
    uv = make_uvdata(uvw, 2, 64, 1, freq, fa, np.random.default_rng(seed + 1))
    sky = make_comps(MOD_POINT, ncomp, np.random.default_rng(seed + 2), radius_deg=0.5)
    return Workload("config1", uv, sky)


def config2(nint: int = 2000, ncomp: int = 20000, seed: int = 2, nant: int = 64) -> Workload:
    """64 antennas (2016 baselines) x nint integrations, 4 IFs x 256 channels of
    1 MHz contiguous about 1.4 GHz, 4 polarizations, 20000 points with spectral
    index in [-1.5, 0.5] about 1.4 GHz, w-term, field radius 1 deg."""
    rng = np.random.default_rng(seed)
    pos = array_layout(nant, 36e3, rng)
    freq = 1.4e9
    fa = freq_axis(256, 4, freq - 512e6, 1e6)
    uvw = make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)
    uv = make_uvdata(uvw, 4, 256, 4, freq, fa, np.random.default_rng(seed + 1))
    sky = make_comps(MOD_POINT_SPEC, ncomp, np.random.default_rng(seed + 2), radius_deg=1.0,
                     nterm=1, ref_freq=freq)
    return Workload("config2", uv, sky)


def config3(nint: int = 2000, ncomp: int = 50000, seed: int = 3, nant: int = 64) -> Workload:
    """config2's uv coverage with 50000 components, 70 % points and 30 %
    elliptical Gaussians (major 1-60 arcsec, axial ratio 0.3-1, random PA),
    each with a spectral index; Gaussian+spectrum table with g = 0 for points."""
    rng = np.random.default_rng(seed)
    pos = array_layout(nant, 36e3, rng)
    freq = 1.4e9
    fa = freq_axis(256, 4, freq - 512e6, 1e6)
    uvw = make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)
    uv = make_uvdata(uvw, 4, 256, 4, freq, fa, np.random.default_rng(seed + 1))
    sky = make_comps(MOD_GAUSS_SPEC, ncomp, np.random.default_rng(seed + 2), radius_deg=1.0,
                     nterm=1, gauss_frac=0.3, ref_freq=freq)
    return Workload("config3", uv, sky)


def config4(nint: int = 240, ncomp: int = 10000, seed: int = 4) -> Workload:
    """32 antennas with baselines to 8000 km at 22 GHz, 8 IFs x 64 channels of
    2 MHz, RR/LL, 10000 points within 2 arcmin of a position 0.3 deg from the
    phase centre."""
    rng = np.random.default_rng(seed)
    pos = array_layout(32, 8.0e6, rng)
    freq = 22e9
    fa = freq_axis(64, 8, freq - 512e6, 2e6)
    uvw = make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)
    uv = make_uvdata(uvw, 2, 64, 8, freq, fa, np.random.default_rng(seed + 1))
    c = 0.3 * DG2RAD / math.sqrt(2.0)
    sky = make_comps(MOD_POINT, ncomp, np.random.default_rng(seed + 2), radius_deg=2.0 / 60.0,
                     center=(c, c))
    return Workload("config4", uv, sky)


def config5_facets(nfacet: int = 96, seed: int = 5, row_scale: float = 1.0,
                   comp_scale: float = 1.0):
    """Seeded draw of the uneven multi-facet workload: per facet components
    log-uniform in [500, 60000], rows log-uniform in [1e5, 1e7], 1-8 IFs x
    32-512 channels, 2 polarizations.  Returns a list of (nrow, ncomp, nif,
    nchan) without materializing data; row_scale/comp_scale shrink the draw."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nfacet):
        nc = int(round(math.exp(rng.uniform(math.log(500), math.log(60000)))))
        nr = int(round(math.exp(rng.uniform(math.log(1e5), math.log(1e7)))))
        nif = int(rng.integers(1, 9))
        nch = int(2 ** rng.integers(5, 10))
        out.append((max(1, int(nr * row_scale)), max(1, int(nc * comp_scale)), nif, nch))
    return out
