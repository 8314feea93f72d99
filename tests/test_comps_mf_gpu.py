"""The multi-frequency loader's table (obit_dft_load_comps_mf: tabulated
spectra with fitted spectral indices) through the DFT on the GPU, against the
FP64 oracle on the same table: CC rows -> component table -> model."""
import numpy as np
import pytest

import oracle
from helpers import TOL_REL, small
from obit_b200 import uvdata as U
from obit_b200.comps import CCField, CCModel, MFModel, load_comps_mf
from obit_b200.skymodel import OP_REPL, GPUSkyModel, SkyModelParams

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gauss", [False, True])
def test_loaded_tabulated_spectra_through_the_dft(gauss):
    uv, _ = small(U.MOD_POINT, nrow=60, nchan=48, nif=2, nstok=2, ncomp=10, seed=91)
    nplane = 4
    edges = np.linspace(uv.freqArr.min(), uv.freqArr.max() + 1.0, nplane + 1)
    spec_freq = 0.5 * (edges[:-1] + edges[1:])
    spec_index = np.clip(np.searchsorted(edges, uv.freqArr, side="right") - 1, 0, nplane - 1).astype(np.int32)
    rng = np.random.default_rng(92)
    n = 400
    x, y = rng.uniform(-0.4, 0.4, n), rng.uniform(-0.4, 0.4, n)
    s0 = np.exp(rng.uniform(np.log(0.01), 0.0, n))
    a = rng.uniform(-1.2, 1.0, n)
    planes = s0[:, None] * (spec_freq[None, :] / spec_freq[0]) ** a[:, None]
    parms = np.zeros((n, 4 + nplane), np.float32)
    if gauss:
        parms[:, 0:3] = (4.0 / 3600, 2.5 / 3600, 60.0)
    parms[:, 3] = 21 if gauss else 20
    parms[:, 4:] = planes
    ra, dec = 150.0, 35.0
    f = CCField(flux=planes.mean(axis=1), deltaX=x, deltaY=y, crvalRA=ra, crvalDec=dec, parms=parms)
    sky, _ = load_comps_mf([f], CCModel(uvRA=ra, uvDec=dec), MFModel(spec_freq), spec_index=spec_index)
    assert sky.ncomp == n and np.count_nonzero(sky.comps[:, 8 if gauss else 5 - 1]) > n // 2
    p = SkyModelParams(op=OP_REPL, nVisPIO=uv.nvis)
    out = uv.copy()
    gm = GPUSkyModel("mf-loader")
    try:
        gm.DFTInit(sky, out, p)
        gm.DFTSetMod(sky)
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    want = oracle.apply_fp64(uv, sky, p)
    _, l1 = oracle.model_fp64(uv, sky, p)
    A = out.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    B = want[:, uv.nrparm:].reshape(A.shape)
    d = np.abs((A[..., 0] - B[..., 0]) + 1j * (A[..., 1] - B[..., 1]))
    # the float32 records cannot hold a model whose every term is below the
    # FP32 normal range (strongly resolved Gaussians on the longest baselines)
    ok = l1 > 1e-30
    assert ok.mean() > 0.9
    assert float(np.nanmax(np.where(ok[..., None], d / l1[..., None], 0.0))) < TOL_REL
