"""The literal drop-in path on the GPU: the reference's own host glue
(ObitSystem/Obit/src/ObitGPUSkyModel.c, compiled unmodified; oracle/refglue.py)
fills GPUInfo exactly as the reference does -- stokFact = factor on every
polarization, doSwap = doFlip, the FP32 freqScale only, the first two
polarizations, buffers of at most 10,000 records -- and calls this library's
void ObitCUDASkyModelDFTInit / SetMod / Calc / Shutdown, with none of the
library's status-returning additions.  The records must match the FP64 oracle
evaluated under the reference GPU plug-in's polarization rules within the
parity tolerance, for every model family and operation, a negative Factor
included; at low phase they must also match the reference's own CUDA kernels
driven by the same glue."""
import numpy as np
import pytest

import oracle
import refglue
from helpers import TOL_REL, small
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refglue.available("ours"), reason="oracle/_ref/libobit_refglue.so not built")]

FAMILIES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC,
            U.MOD_GAUSS_TSPEC]


def _table(sky, factor):
    """The component table as ObitSkyModelLoadComps writes it: flux x Factor
    (ObitSkyModel.c:1965); tabulated spectra scale every plane's flux."""
    t = sky.comps.copy()
    t[:, 0] *= factor
    if sky.modType == U.MOD_POINT_TSPEC:
        t[:, 5:] *= factor
    elif sky.modType == U.MOD_GAUSS_TSPEC:
        t[:, 8:] *= factor
    return U.SkyComps(sky.modType, t, nterm=sky.nterm, refFreq=sky.refFreq, specFreq=sky.specFreq,
                      specIndex=sky.specIndex)


def _oracle(uv, sky, factor, op, chans=None, ifs=None):
    """FP64 oracle under the reference GPU rules, with the glue's selection
    (first two polarizations, FP32 freqScale)."""
    kw = {}
    if chans:
        kw.update(startChannel=chans[0], numberChannel=chans[1])
    if ifs:
        kw.update(startIF=ifs[0], numberIF=ifs[1])
    p = SkyModelParams(op=op, startPoln=1, numberPoln=min(2, uv.nstok), **kw)
    want = oracle.apply_fp64(uv, sky, p, exact=False, gpu_rules=([factor] * 4, False))
    _, l1 = oracle.model_fp64(uv, sky, p, exact=False)
    return want, l1


def _max_rel(got, want, l1, uv, pols=2):
    x = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    y = want[:, uv.nrparm:].reshape(x.shape)
    d = np.abs((x[..., 0] - y[..., 0]) + 1j * (x[..., 1] - y[..., 1]))[..., :pols]
    sel = ~np.isnan(l1)
    return float(np.max((d / np.where(sel, l1, np.inf)[..., None])))


@pytest.mark.parametrize("mt", FAMILIES)
@pytest.mark.parametrize("op,factor", [(OP_SUB, 1.0), (OP_SUB, -1.0), (OP_REPL, 0.5), (OP_DIV, 1.0)])
def test_reference_glue_over_this_library(mt, op, factor):
    flag = 0.2 if op == OP_SUB else 0.0
    uv, sky = small(mt, nrow=70, nchan=24, nif=2, nstok=4, ncomp=160, seed=71 + mt, flag_frac=flag,
                    nterm=2)
    t = _table(sky, factor)
    got, per = refglue.run(uv, t, factor=factor, op=op)
    assert per == uv.nvis  # one buffer
    want, l1 = _oracle(uv, t, factor, op)
    assert not np.array_equal(got, uv.vis)
    assert _max_rel(got, want, l1, uv) < TOL_REL
    # polarizations 3-4 are never touched by the reference's selection
    v = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    assert np.array_equal(v[..., 2:, :], uv.vis_view()[..., 2:, :])
    if op != OP_DIV:  # weights unchanged
        assert np.array_equal(v[..., 2], uv.vis_view()[..., 2])


def test_reference_glue_buffers_and_selection():
    """More records than one glue buffer (10,000), a channel and IF selection."""
    uv, sky = small(U.MOD_POINT_SPEC, nrow=12345, nchan=16, nif=3, nstok=2, ncomp=40, seed=81,
                    flag_frac=0.1)
    got, per = refglue.run(uv, sky, op=OP_SUB, startChann=3, numberChann=11, startIF=2, numberIF=2)
    assert per == 10000
    want, l1 = _oracle(uv, sky, 1.0, OP_SUB, chans=(3, 11), ifs=(2, 2))
    assert _max_rel(got, want, l1, uv) < TOL_REL
    # outside the selection: untouched
    v = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    o = uv.vis_view()
    assert np.array_equal(v[:, 0], o[:, 0])
    assert np.array_equal(v[:, :, :2], o[:, :, :2])
    assert np.array_equal(v[:, :, 13:], o[:, :, 13:])


@pytest.mark.skipif(not refglue.available("ref"), reason="oracle/_ref/libobit_refglue_ref.so not built")
@pytest.mark.parametrize("mt", [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC])
@pytest.mark.parametrize("factor", [1.0, -1.0])
def test_reference_glue_same_records_as_reference_kernels_at_low_phase(mt, factor):
    """The same glue over the reference's own ObitCUDASkyModel.cu: at modest
    phases (its FP32 phase and __sincosf are accurate there) both layers give
    the same records.  The reference kernels use exp(-sum a_t L^(t+1)) for
    polynomial spectra (ObitCUDASkyModel.cu:240,563); their table carries the
    negated coefficients so that both evaluate the same sky."""
    uv, sky = small(mt, nrow=66, nchan=24, nif=2, nstok=4, ncomp=150, seed=91 + mt, max_bl=300.0,
                    radius_deg=1.0 / 60.0, nterm=2, flag_frac=0.2)
    t = _table(sky, factor)
    ours, _ = refglue.run(uv, t, factor=factor, op=OP_SUB, which="ours")
    tr = U.SkyComps(t.modType, t.comps.copy(), nterm=t.nterm, refFreq=t.refFreq)
    if mt == U.MOD_POINT_SPEC:
        tr.comps[:, 4:4 + t.nterm] *= -1.0
    elif mt == U.MOD_GAUSS_SPEC:
        tr.comps[:, 7:7 + t.nterm] *= -1.0
    ref, _ = refglue.run(uv, tr, factor=factor, op=OP_SUB, which="ref")
    want, l1 = _oracle(uv, t, factor, OP_SUB)
    assert _max_rel(ref, want, l1, uv) < TOL_REL
    assert _max_rel(ours, ref, l1, uv) < TOL_REL
