"""Shared helpers for the parity tests: run the GPU path through the C ABI and
compare with the FP64 oracle."""
from __future__ import annotations

import numpy as np

import oracle
from obit_b200 import uvdata as U
from obit_b200._lib import OBIT_DFT_PLAIN, OBIT_DFT_RECUR
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, GPUSkyModel, SkyModelParams

# |V_gpu - V_oracle| / sum_c |A_c|, per visibility
TOL_REL = 1e-5


def run_gpu(uv: U.UVData, sky: U.SkyComps, params: SkyModelParams | None = None,
            flavor: int = OBIT_DFT_RECUR, K: int = 0, ct: int = 0, exact: bool = True,
            Bt: int = 0, threads: int = 0) -> U.UVData:
    """Apply the model with the GPU path; returns a new UVData."""
    p = params or SkyModelParams()
    if p.nVisPIO <= 0:
        p.nVisPIO = max(1, uv.nvis)
    out = uv.copy()
    gm = GPUSkyModel("test")
    try:
        gm.DFTInit(sky, out, p, exact_freq=exact)
        if flavor != OBIT_DFT_RECUR or K or ct or Bt or threads:
            gm.set_kernel(flavor, K, ct, Bt, threads)
        gm.DFTSetMod(sky)
        if uv.nvis > 0:
            gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    return out


def gpu_model(uv, sky, params=None, **kw):
    """GPU model of the first selected polarization via the replace operation:
    complex (nvis, nif, nchan)."""
    p = params or SkyModelParams()
    q = SkyModelParams(**{**p.__dict__, "op": OP_REPL, "doFlip": False, "stokFactor": 1.0})
    out = run_gpu(uv, sky, q, **kw)
    pol0 = (q.startPoln if q.startPoln > 0 else 1) - 1
    v = out.vis_view()[..., pol0, :]
    return v[..., 0].astype(np.float64) + 1j * v[..., 1].astype(np.float64)


def model_error(uv, sky, params=None, exact=True, **kw):
    """(max, rms) of |V_gpu - V_fp64| / sum|A| over selected visibilities."""
    g = gpu_model(uv, sky, params, exact=exact, **kw)
    m, l1 = oracle.model_fp64(uv, sky, params, exact=exact)
    sel = ~np.isnan(l1)
    rel = np.abs(g - m)[sel] / np.maximum(l1[sel], 1e-30)
    return float(rel.max()), float(np.sqrt(np.mean(rel ** 2)))


def small(modType=U.MOD_POINT, nrow=64, nchan=48, nif=2, nstok=2, ncomp=300, seed=11,
          radius_deg=0.5, max_bl=36e3, freq=1.4e9, dnu=1e6, nterm=1, flag_frac=0.0,
          nplanes=3, gauss_frac=0.5, alpha=(-1.5, 0.5)):
    """A small seeded workload of any model family."""
    rng = np.random.default_rng(seed)
    pos = U.array_layout(12, max_bl, rng)
    nbl = 12 * 11 // 2
    nint = max(1, (nrow + nbl - 1) // nbl)
    uvw = U.make_uvw(pos, nint, 45.0, 4.0, 34.0, freq)[:nrow]
    fa = U.freq_axis(nchan, nif, freq - 0.5 * nchan * nif * dnu, dnu)
    uv = U.make_uvdata(uvw, nstok, nchan, nif, freq, fa, np.random.default_rng(seed + 1),
                       flag_frac=flag_frac)
    kw = {}
    if modType in (U.MOD_POINT_TSPEC, U.MOD_GAUSS_TSPEC):
        lo, hi = fa.min(), fa.max()
        edges = np.linspace(lo, hi + 1.0, nplanes + 1)
        spec_freq = 0.5 * (edges[:-1] + edges[1:])
        idx = np.clip(np.searchsorted(edges, fa, side="right") - 1, 0, nplanes - 1)
        kw = dict(spec_freq=spec_freq, spec_index=idx)
    sky = U.make_comps(modType, ncomp, np.random.default_rng(seed + 2), radius_deg=radius_deg,
                       nterm=nterm, ref_freq=freq, gauss_frac=gauss_frac, alpha=alpha, **kw)
    return uv, sky


__all__ = ["run_gpu", "gpu_model", "model_error", "small", "TOL_REL", "OP_SUB", "OP_DIV",
           "OP_REPL", "SkyModelParams", "OBIT_DFT_PLAIN", "OBIT_DFT_RECUR"]
