"""The oracles themselves, on CPU: the FP64 oracle (A, oracle_dft.c) against an
independent numpy statement of the reference CPU DFT, and the reference-faithful
restatement (B, refcpu_dft.c with the reference's ObitSinCosVec/ObitExpVec)
against (A) where FP32 phases are accurate.

numpy statement followed here (reference CPU DFT):
  ThreadSkyModelFTDFT    ObitSystem/Obit/src/ObitSkyModel.c:2354-2857
  ThreadSkyModelMFFTDFT  ObitSystem/Obit/src/ObitSkyModelMF.c:1971-2440
"""
import numpy as np
import pytest

import oracle
from helpers import small
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

ALL_TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC,
             U.MOD_GAUSS_TSPEC]


def np_model(uv, sky):
    """complex128 (nvis, nif, nchan) model and its L1 norm, all channels."""
    c = sky.comps.astype(np.float64)
    uvw = uv.vis[:, :3].astype(np.float64)
    fs = (uv.freqArr / uv.freq).reshape(uv.nif, uv.nchan)           # [IF, chan]
    u = uvw[:, 0, None, None] * fs                                   # [row, IF, chan]
    v = uvw[:, 1, None, None] * fs
    w = uvw[:, 2, None, None] * fs
    nu = uv.freqArr.reshape(uv.nif, uv.nchan)
    gauss = sky.modType in (U.MOD_GAUSS, U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC)
    out = np.zeros(u.shape, np.complex128)
    l1 = np.zeros(u.shape)
    for k in range(sky.ncomp):
        expo = np.zeros(u.shape)
        amp = np.full(u.shape, c[k, 0])
        base = 7 if gauss else 4
        if gauss:
            expo += c[k, 4] * u * u + c[k, 5] * v * v + c[k, 6] * u * v
        if sky.modType in (U.MOD_POINT_SPEC, U.MOD_GAUSS_SPEC):
            L = np.log(nu / sky.refFreq)
            for t in range(sky.nterm):
                expo += c[k, base + t] * L ** (t + 1)
        if sky.is_tspec:
            plane = sky.specIndex.reshape(uv.nif, uv.nchan)
            amp = c[k, base + 1 + plane] * np.ones(u.shape)
            expo += c[k, base] * np.log(nu / sky.specFreq[plane])
        amp = amp * np.exp(expo)
        out += amp * np.exp(1j * (c[k, 1] * u + c[k, 2] * v + c[k, 3] * w))
        l1 += np.abs(amp)
    return out, l1


@pytest.mark.parametrize("mt", ALL_TYPES)
def test_oracle_model_matches_numpy(mt):
    uv, sky = small(mt, nrow=9, nchan=7, nif=2, nstok=2, ncomp=11, seed=3, nterm=2)
    m, l1 = oracle.model_fp64(uv, sky, nthreads=3)
    want, wl1 = np_model(uv, sky)
    assert np.max(np.abs(m - want) / wl1) < 1e-12
    assert np.allclose(l1, wl1, rtol=1e-12)


def np_apply(uv, sky, params):
    """Records after the reference CPU application rules (ObitSkyModel.c:2787-2849)."""
    m, _ = np_model(uv, sky)
    out = uv.copy()
    v = out.vis_view()                                              # [row, IF, chan, pol, 3]
    p0 = (params.startPoln if params.startPoln > 0 else 1) - 1
    npol = params.numberPoln if params.numberPoln > 0 else min(2, uv.nstok)
    for r in range(uv.nvis):
        for i in range(uv.nif):
            for ch in range(uv.nchan):
                wt = v[r, i, ch, p0:p0 + npol, 2]
                if not np.any(wt > 0) and params.op != OP_REPL:
                    continue
                cum = 1.0
                for jp in range(npol):
                    rec = v[r, i, ch, p0 + jp]
                    if rec[2] <= 0 and params.op != OP_REPL:
                        continue
                    mod = cum * m[r, i, ch] * (1j if params.doFlip else 1.0)
                    if params.op == OP_DIV:
                        q = complex(rec[0], rec[1]) / mod
                        rec[0], rec[1], rec[2] = q.real, q.imag, rec[2] * abs(mod)
                    elif params.op == OP_REPL:
                        rec[0], rec[1] = mod.real, mod.imag
                    else:
                        rec[0] -= mod.real
                        rec[1] -= mod.imag
                    cum *= params.stokFactor
    return out.vis


@pytest.mark.parametrize("op", [OP_SUB, OP_DIV, OP_REPL])
@pytest.mark.parametrize("flip", [False, True])
def test_oracle_apply_matches_numpy(op, flip):
    uv, sky = small(U.MOD_GAUSS_SPEC, nrow=13, nchan=5, nif=2, nstok=4, ncomp=7, seed=4,
                    flag_frac=0.3)
    p = SkyModelParams(op=op, doFlip=flip, stokFactor=-0.5, startPoln=1, numberPoln=2)
    got = oracle.apply_fp64(uv, sky, p, nthreads=2)
    want = np_apply(uv, sky, p)
    assert np.allclose(got, want, rtol=2e-6, atol=1e-6)
    # cross-hand correlations (polarizations 3-4) stay untouched
    cross = got[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., 2:, :]
    assert np.array_equal(cross, uv.vis_view()[..., 2:, :])


def test_oracle_thread_split_is_deterministic():
    uv, sky = small(U.MOD_POINT_SPEC, nrow=37, nchan=6, nif=1, ncomp=23, seed=5)
    a = oracle.apply_fp64(uv, sky, nthreads=1)
    b = oracle.apply_fp64(uv, sky, nthreads=5)
    assert np.array_equal(a, b)


@pytest.mark.skipif(not oracle.have_refcpu(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mt", ALL_TYPES)
def test_refcpu_agrees_with_fp64_at_low_phase(mt):
    """(B) uses FP32 phases and the reference's SIMD sin/cos/exp: on short
    baselines and a 1-arcmin field it must agree with (A) well below 1e-5 of
    the L1 norm."""
    uv, sky = small(mt, nrow=66, nchan=16, nif=2, nstok=2, ncomp=120, seed=6, max_bl=300.0,
                    radius_deg=1.0 / 60.0)
    _, l1 = oracle.model_fp64(uv, sky)
    p = SkyModelParams(op=OP_REPL)
    a = oracle.apply_fp64(uv, sky, p)[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = oracle.apply_refcpu(uv, sky, p)[:, uv.nrparm:].reshape(uv.vis_view().shape)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))[..., :2]
    assert float(np.max(d / l1[..., None])) < 1e-6


@pytest.mark.skipif(not oracle.have_refcpu(), reason="oracle/_ref not built")
def test_refcpu_subtract_matches_fp64_model():
    uv, sky = small(U.MOD_POINT, nrow=40, nchan=8, nif=1, ncomp=50, seed=7, max_bl=300.0,
                    radius_deg=1.0 / 60.0, flag_frac=0.2)
    a = oracle.apply_fp64(uv, sky, SkyModelParams(op=OP_SUB))
    b = oracle.apply_refcpu(uv, sky, SkyModelParams(op=OP_SUB))
    assert np.max(np.abs(a - b)) < 1e-5 * np.max(np.abs(sky.comps[:, 0])) * sky.ncomp
    # flagged records are untouched by both
    wt = uv.vis_view()[..., 2]
    va, vb = (x[:, uv.nrparm:].reshape(uv.vis_view().shape) for x in (a, b))
    assert np.array_equal(va[wt <= 0], uv.vis_view()[wt <= 0])
    assert np.array_equal(vb[wt <= 0], uv.vis_view()[wt <= 0])


def test_oracle_fp64_positions():
    """Optional FP64 positions: the FP32 table's own values promoted give the
    table result exactly; the FP64 values move the phase (here a 22 GHz,
    8000 km array, components 0.3 deg out) by far more than the tolerance."""
    w = U.config4(nint=2, ncomp=200)
    uv = w.uv.rows(0, 40)
    sky = w.sky
    p = SkyModelParams(op=OP_REPL)
    a = oracle.apply_fp64(uv, sky, p)
    b = oracle.apply_fp64(uv, sky, p, xyz=sky.comps[:, 1:4].astype(np.float64))
    assert np.array_equal(a, b)
    m64, l1 = oracle.model_fp64(uv, sky, p, xyz=sky.xyz)
    m32, _ = oracle.model_fp64(uv, sky, p)
    assert np.nanmax(np.abs(m64 - m32) / l1) > 1e-3
    assert np.max(np.abs(sky.xyz - sky.comps[:, 1:4])) < 1e-6 * np.max(np.abs(sky.xyz))
