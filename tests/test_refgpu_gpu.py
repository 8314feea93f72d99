"""The reference's own CUDA kernels (ObitCUDASkyModel.cu compiled for sm_100a,
oracle/refgpu.py) as a second implementation: at modest phases, where their
FP32 phase and __sincosf are accurate, they must agree with the FP64 oracle and
with this library within the parity tolerance -- an independent pin of the
oracle's model families and application rules on the reference's own code.
At config-2 phases their FP32 error is measured and printed ("REFGPU {json}")
beside their throughput through ObitCUDASkyModelDFTCalc."""
import json
import sys
import time
from pathlib import Path

import numpy as np
import pytest

import oracle
import refgpu
from helpers import TOL_REL, run_gpu, small
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_REPL, OP_SUB, SkyModelParams

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref/libobit_refgpu.so not built")]


def _rel(a, b, l1, uv):
    shape = uv.vis_view().shape
    x = a[:, uv.nrparm:].reshape(shape)[..., :2, :]
    y = b[:, uv.nrparm:].reshape(shape)[..., :2, :]
    d = np.abs((x[..., 0] - y[..., 0]) + 1j * (x[..., 1] - y[..., 1])) / l1[..., None]
    return float(d.max()), float(np.sqrt(np.mean(d ** 2)))


@pytest.mark.parametrize("mt", [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC])
def test_reference_kernels_agree_with_oracle_at_low_phase(mt):
    uv, sky = small(mt, nrow=66, nchan=24, nif=2, nstok=4, ncomp=150, seed=51, max_bl=300.0,
                    radius_deg=1.0 / 60.0, nterm=2)
    p = SkyModelParams(op=OP_REPL)
    ref = refgpu.RefGPU(uv, sky, p)
    try:
        got = ref.calc(uv.vis)
    finally:
        ref.close()
    # FP32 freqScale on both sides: the reference carries only that
    _, l1 = oracle.model_fp64(uv, sky, p, exact=False)
    want = oracle.apply_fp64(uv, sky, p, exact=False)
    mx, _ = _rel(got, want, l1, uv)
    assert mx < TOL_REL
    ours = run_gpu(uv, sky, p, exact=False).vis
    assert _rel(ours, got, l1, uv)[0] < TOL_REL
    # polarizations 3-4 untouched by both
    shape = uv.vis_view().shape
    assert np.array_equal(got[:, 5:].reshape(shape)[..., 2:, :], uv.vis_view()[..., 2:, :])


def test_reference_kernels_subtract_skips_flagged_data():
    uv, sky = small(U.MOD_POINT, nrow=40, nchan=16, nif=1, nstok=2, ncomp=60, seed=52, max_bl=300.0,
                    radius_deg=1.0 / 60.0, flag_frac=0.3)
    p = SkyModelParams(op=OP_SUB)
    ref = refgpu.RefGPU(uv, sky, p)
    try:
        got = ref.calc(uv.vis)
    finally:
        ref.close()
    want = oracle.apply_fp64(uv, sky, p, exact=False)
    _, l1 = oracle.model_fp64(uv, sky, p, exact=False)
    assert _rel(got, want, l1, uv)[0] < TOL_REL
    wt = uv.vis_view()[..., 2]
    v = got[:, 5:].reshape(uv.vis_view().shape)
    assert np.array_equal(v[wt <= 0], uv.vis_view()[wt <= 0])


def test_reference_kernels_on_config2_chunk():
    """Accuracy of the reference kernels at config-2 phases (FP32 phase) and
    their throughput through ObitCUDASkyModelDFTCalc (host buffers, its own
    four-stream pipeline) on 2016 records (one integration) of config 2."""
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    from bench import workload_geometry

    g = workload_geometry("config2", 0, 2016, None)
    uv = U.make_uvdata(g.uvw, g.nstok, g.nchan, g.nif, g.freq, g.fa, np.random.default_rng(8))
    p = SkyModelParams(op=OP_REPL, numberPoln=2)
    ref = refgpu.RefGPU(uv, g.sky, p)
    try:
        rows = np.linspace(0, uv.nvis - 1, 12).astype(int)
        got = ref.calc(uv.vis)[rows]
        secs = ref.time_calc(uv.vis, reps=3)
    finally:
        ref.close()
    sub = uv.rows(0, 0)
    sub.vis = uv.vis[rows].copy()
    _, l1 = oracle.model_fp64(sub, g.sky, p, exact=False)
    want = oracle.apply_fp64(sub, g.sky, p, exact=False)
    mx, rms = _rel(got, want, l1, sub)
    evals = uv.nvis * g.channels * g.sky.ncomp
    print("REFGPU " + json.dumps({"workload": "config2, 2016 records x 1024 channels x 20000 "
                                              "PointSpec components", "evals": evals,
                                  "seconds_per_calc": secs, "gevals_per_s": evals / secs / 1e9,
                                  "max_rel_err_vs_fp64": mx, "rms_rel_err_vs_fp64": rms}))
    assert mx < 1e-1  # FP32 phase of ~1e4 rad: far from 1e-5, but the model is right
