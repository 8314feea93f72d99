"""The reference's golden test of the DFT path (Obit/testScripts/testUVSub.py):
divide the DFT of a 13-component CC model (entered twice at half flux) into
real VLA data and compare with the reference's master output with the metric of
ObitUVUtilVisCompare.  tests/golden/make_uvsub_fixture.py made the fixture from
the reference's test data (a row subset, the component table after the
reference's geometry, and the full-data RMS values).

The master was written by an Obit build with FP32 phases and positions, so it
agrees with an exact evaluation only to the FP32 level: the fractional RMS is
5.4e-4 over all rows, growing linearly with baseline length (the size of an
FP32 position/phase rounding), against 1.9 for the undivided input."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import TOL_REL
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, SkyModelParams

GOLD = Path(__file__).resolve().parent / "golden"
PIN_RMS = 1.0e-3  # fractional RMS vs the master; the full-data value is 5.4e-4


def _vis_compare(a, b, nrparm=5):
    """ObitUVUtilVisCompare (ObitSystem/Obit/src/ObitUVUtil.c:1455-1503):
    sqrt(mean over real and imaginary parts of (delta^2 / |master|)) over
    correlations with positive weight in both."""
    x = a[:, nrparm:].reshape(len(a), -1, 3).astype(np.float64)
    y = b[:, nrparm:].reshape(len(b), -1, 3).astype(np.float64)
    amp = np.sqrt(y[..., 0] ** 2 + y[..., 1] ** 2)
    ok = (x[..., 2] > 0) & (y[..., 2] > 0) & (amp > 0)
    s = ((x[..., 0] - y[..., 0]) ** 2 + (x[..., 1] - y[..., 1]) ** 2)[ok] / amp[ok]
    return float(np.sqrt(s.sum() / (2 * ok.sum())))


def _fixture():
    d = np.load(GOLD / "uvsub_fixture.npz")
    nstok, nchan, nif = (int(v) for v in d["axes"])
    uv = U.UVData(d["input"].copy(), nstok, nchan, nif, float(d["ref_freq"]),
                  d["freq_arr"].copy(), crval_stokes=float(d["crval_stokes"]))
    sky = U.SkyComps(U.MOD_POINT, d["comps"].copy())
    params = SkyModelParams(op=OP_DIV, startPoln=1, numberPoln=2)
    return uv, sky, params, d["master"].copy()


def test_fixture_records_the_full_data_pin():
    info = json.loads((GOLD / "uvsub_fixture.json").read_text())
    assert info["records"] == 15949 and info["components"] == 26
    assert info["visCompare_fp64_oracle_vs_master"] < PIN_RMS
    assert info["visCompare_input_vs_master"] > 1.0


def test_oracle_divide_reproduces_master():
    uv, sky, params, master = _fixture()
    assert _vis_compare(uv.vis, master) > 1.0          # undivided data is far off
    out = oracle.apply_fp64(uv, sky, params)
    assert _vis_compare(out, master) < PIN_RMS
    # cross-hand correlations and their weights are untouched, as in the master
    v, m = (x[:, 5:].reshape(len(x), uv.nif, uv.nchan, uv.nstok, 3) for x in (out, master))
    assert np.array_equal(v[..., 2:, :], m[..., 2:, :])
    # divide scales weights by |model|
    assert np.allclose(v[..., :2, 2], m[..., :2, 2], rtol=2e-3)


def test_pin_detects_a_position_error():
    """A mistake planted in the oracle's input (every component moved by 2e-9
    rad, below an arcsecond's thousandth) must break the pin."""
    uv, sky, params, master = _fixture()
    sky.comps[:, 1] += np.float32(2 * np.pi * 2e-9)
    assert _vis_compare(oracle.apply_fp64(uv, sky, params), master) > 3 * PIN_RMS


@pytest.mark.skipif(not oracle.have_refcpu(), reason="oracle/_ref not built")
def test_reference_restatement_reproduces_master():
    uv, sky, params, master = _fixture()
    assert _vis_compare(oracle.apply_refcpu(uv, sky, params), master) < PIN_RMS


@pytest.mark.gpu
def test_gpu_divide_reproduces_master_and_oracle():
    from helpers import run_gpu

    uv, sky, params, master = _fixture()
    out = run_gpu(uv, sky, params)
    assert _vis_compare(out.vis, master) < PIN_RMS
    want = oracle.apply_fp64(uv, sky, params)
    _, l1 = oracle.model_fp64(uv, sky, params)
    a = out.vis[:, 5:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)[..., :2, :]
    b = want[:, 5:].reshape(a.shape[:-2] + (uv.nstok, 3))[..., :2, :]
    # divided values are V/M with |M| ~ 2.5 Jy = sum|A|: compare the quotient
    # error scaled back to model units
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    vm = np.abs(b[..., 0] + 1j * b[..., 1])
    assert float(np.max(d / np.maximum(vm, 1e-30))) < 10 * TOL_REL
