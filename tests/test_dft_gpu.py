"""GPU parity: the sm_100a kernels through the C ABI against the FP64 oracle.

Metric: |V_gpu - V_fp64| / sum_c |A_c| per visibility, bound 1e-5 (TOL_REL)."""
import numpy as np
import pytest

import oracle
from helpers import (OBIT_DFT_PLAIN, OBIT_DFT_RECUR, OP_DIV, OP_REPL, OP_SUB, TOL_REL,
                     SkyModelParams, gpu_model, model_error, run_gpu, small)
from obit_b200 import uvdata as U

pytestmark = pytest.mark.gpu

ALL_TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC,
             U.MOD_GAUSS_TSPEC]


@pytest.mark.parametrize("mod", ALL_TYPES)
@pytest.mark.parametrize("K", [32, 16, 8])
def test_model_types_recur(mod, K):
    uv, sky = small(mod, nrow=80, nchan=40, nif=2, ncomp=257)
    mx, rms = model_error(uv, sky, K=K)
    assert mx < TOL_REL, (mx, rms)


@pytest.mark.parametrize("mod", ALL_TYPES)
def test_model_types_plain(mod):
    uv, sky = small(mod, nrow=48, nchan=24, nif=2, ncomp=130)
    mx, rms = model_error(uv, sky, flavor=OBIT_DFT_PLAIN, K=8)
    assert mx < TOL_REL, (mx, rms)


@pytest.mark.parametrize("K", [2, 4, 32])
def test_channels_per_thread(K):
    uv, sky = small(U.MOD_POINT_SPEC, nrow=40, nchan=70, nif=1, ncomp=100)
    mx, _ = model_error(uv, sky, K=K)
    assert mx < TOL_REL


@pytest.mark.parametrize("Bt", [1, 4, 32])
def test_tile_shapes(Bt):
    uv, sky = small(U.MOD_GAUSS_TSPEC, nrow=70, nchan=64, nif=3, ncomp=90)
    mx, _ = model_error(uv, sky, Bt=Bt, K=8)
    assert mx < TOL_REL


@pytest.mark.parametrize("mod", [U.MOD_POINT, U.MOD_GAUSS_SPEC])
def test_plain_one_channel_blocks(mod):
    uv, sky = small(mod, nrow=20, nchan=9, nif=1, ncomp=40)
    mx, _ = model_error(uv, sky, flavor=OBIT_DFT_PLAIN, K=1)
    assert mx < TOL_REL


def test_two_spectral_terms():
    uv, sky = small(U.MOD_POINT_SPEC, nterm=2, nrow=40, nchan=33, nif=2, ncomp=90)
    mx, _ = model_error(uv, sky)
    assert mx < TOL_REL


@pytest.mark.parametrize("op", [OP_SUB, OP_DIV, OP_REPL])
def test_operations_match_oracle(op):
    uv, sky = small(U.MOD_GAUSS_SPEC, nrow=50, nchan=20, nif=2, nstok=4, ncomp=120, flag_frac=0.1)
    if op == OP_DIV:
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    p = SkyModelParams(op=op)
    got = run_gpu(uv, sky, p).vis
    want = oracle.apply_fp64(uv, sky, p)
    m, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    b = want[:, uv.nrparm:].reshape(a.shape)
    # polarizations 3,4 are never touched for a correlation model
    assert np.array_equal(a[..., 2:, :], uv.vis_view()[..., 2:, :])
    # weights: unchanged for sub/repl, x|M| for divide
    if op != OP_DIV:
        assert np.array_equal(a[..., 2], b[..., 2])
    if op == OP_DIV:
        # data 1+0i divided by M gives 1/M: compare the implied model
        sel = b[..., :2, 2] > 0
        ga = 1.0 / (a[..., :2, 0] + 1j * a[..., :2, 1])
        wa = 1.0 / (b[..., :2, 0] + 1j * b[..., :2, 1])
        rel = np.abs(ga - wa) / l1[..., None]
        assert np.nanmax(np.where(sel, rel, 0)) < TOL_REL
        wrel = np.abs(a[..., :2, 2] - b[..., :2, 2]) / np.maximum(l1[..., None], 1e-30)
        assert np.nanmax(np.where(sel, wrel, 0)) < TOL_REL
    else:
        d = np.abs((a[..., :2, 0] - b[..., :2, 0]) + 1j * (a[..., :2, 1] - b[..., :2, 1]))
        assert np.nanmax(d / l1[..., None]) < TOL_REL + 1e-6


def test_flagged_data_untouched_for_subtract():
    uv, sky = small(U.MOD_POINT, nrow=30, nchan=16, ncomp=40, flag_frac=0.3)
    got = run_gpu(uv, sky, SkyModelParams(op=OP_SUB)).vis_view()
    src = uv.vis_view()
    flagged = src[..., 2] <= 0
    assert flagged.any()
    assert np.array_equal(got[flagged], src[flagged])


def test_stokfactor_and_flip_cpu_rules():
    uv, sky = small(U.MOD_POINT, nrow=30, nchan=16, ncomp=40, flag_frac=0.3)
    p = SkyModelParams(op=OP_SUB, doFlip=True, stokFactor=-1.0)
    got = run_gpu(uv, sky, p).vis
    want = oracle.apply_fp64(uv, sky, p)
    m, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    b = want[:, uv.nrparm:].reshape(a.shape)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert np.max(d / l1[..., None]) < TOL_REL + 1e-6


def test_channel_if_poln_selection():
    uv, sky = small(U.MOD_POINT_SPEC, nrow=40, nchan=37, nif=3, nstok=4, ncomp=64)
    p = SkyModelParams(op=OP_SUB, startChannel=5, numberChannel=21, startIF=2, numberIF=2,
                       startPoln=2, numberPoln=2)
    got = run_gpu(uv, sky, p).vis
    want = oracle.apply_fp64(uv, sky, p)
    m, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    b = want[:, uv.nrparm:].reshape(a.shape)
    src = uv.vis_view()
    # outside the selection nothing changes
    mask = np.zeros(a.shape[:-1], bool)
    mask[:, 1:3, 4:25, 1:3] = True
    assert np.array_equal(a[~mask], src[~mask])
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))[mask].reshape(uv.nvis, 2, 21, 2)
    assert np.max(d / l1[:, 1:3, 4:25, None]) < TOL_REL + 1e-6


def test_empty_model_is_noop():
    uv, sky = small(U.MOD_POINT, nrow=10, nchan=8, ncomp=5)
    sky.comps[:, 0] = 0.0
    for op in (OP_SUB, OP_DIV, OP_REPL):
        got = run_gpu(uv, sky, SkyModelParams(op=op))
        assert np.array_equal(got.vis, uv.vis)


def test_single_row_single_channel():
    uv, sky = small(U.MOD_POINT, nrow=1, nchan=1, nif=1, ncomp=17)
    mx, _ = model_error(uv, sky)
    assert mx < TOL_REL


def test_nonlinear_frequency_table():
    uv, sky = small(U.MOD_POINT, nrow=30, nchan=24, nif=1, ncomp=50)
    rng = np.random.default_rng(3)
    uv.freqArr = np.sort(uv.freqArr + rng.uniform(-3e5, 3e5, uv.freqArr.shape))
    mx, _ = model_error(uv, sky)
    assert mx < TOL_REL


def test_fp32_freqscale_interface():
    """Without the FP64 side table the kernels see only FP32 freqScale; the
    result matches the oracle fed the same FP32 ratios."""
    uv, sky = small(U.MOD_POINT, nrow=40, nchan=32, nif=2, ncomp=80)
    mx, _ = model_error(uv, sky, exact=False)
    assert mx < TOL_REL


@pytest.mark.parametrize("K", [0, 16])
def test_high_phase_precision(K):
    """8000 km baselines at 22 GHz, field 0.3 deg off centre: phases ~1e7 rad."""
    rng = np.random.default_rng(4)
    pos = U.array_layout(10, 8.0e6, rng)
    freq = 22e9
    fa = U.freq_axis(64, 2, freq - 64e6, 2e6)
    uvw = U.make_uvw(pos, 4, 45.0, 4.0, 34.0, freq)
    uv = U.make_uvdata(uvw, 2, 64, 2, freq, fa, np.random.default_rng(5))
    c = 0.3 * U.DG2RAD / np.sqrt(2.0)
    sky = U.make_comps(U.MOD_POINT, 200, np.random.default_rng(6), radius_deg=2 / 60, center=(c, c))
    mx, rms = model_error(uv, sky, K=K)
    assert mx < TOL_REL, (mx, rms)


@pytest.mark.parametrize("K", [0, 16])
def test_sampled_rows_config2_shape(K):
    """Full config-2 channel/IF/polarization layout and component count on a
    few rows (the dataset's size-independent part)."""
    w = U.config2(nint=1, ncomp=20000, nant=6)
    mx, rms = model_error(w.uv, w.sky, K=K)
    assert mx < TOL_REL, (mx, rms)


@pytest.mark.parametrize("Bt", [2, 16])
def test_128_thread_ctas(Bt):
    uv, sky = small(U.MOD_POINT_SPEC, nrow=70, nchan=64, nif=3, ncomp=90)
    mx, _ = model_error(uv, sky, Bt=Bt, threads=128)
    assert mx < TOL_REL


def test_host_buffer_path_pipelines_large_buffers():
    """40,003 records through obit_dft_calc in one call: four stream buffers of
    10,001 records, each cut into quarter-buffer chunks with a short last one
    (the pipelined host-buffer path), subtract with flags."""
    uv, sky = small(U.MOD_POINT_SPEC, nrow=40003, nchan=8, nif=2, nstok=2, ncomp=40, seed=71,
                    flag_frac=0.05)
    mx, _ = model_error(uv, sky)
    assert mx < TOL_REL
    p = SkyModelParams(op=OP_SUB)
    got = run_gpu(uv, sky, p).vis
    want = oracle.apply_fp64(uv, sky, p)
    _, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(a.shape)
    d = np.abs((a[..., :2, 0] - b[..., :2, 0]) + 1j * (a[..., :2, 1] - b[..., :2, 1]))
    assert np.nanmax(d / l1[..., None]) < TOL_REL + 1e-6
    assert np.array_equal(a[..., 2], b[..., 2])
