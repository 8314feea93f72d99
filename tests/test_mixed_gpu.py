"""GPU parity of the mixed recurrence: a Gaussian-family model with one spectral
index whose untapered components (g1 = g2 = g3 = 0, the reference's encoding
of points in a Gaussian table) the library moves into a point sub-table that
runs in the spectral-factored form, the Gaussian components then running the
chain form into the same compensated totals in one launch.  Every operation
stays exact in one pass (divide included).

Each case checks the plan (plan info: mixed, number of point components) and
compares with the FP64 oracle, |V_gpu - V_fp64| / sum_c |A_c| < 1e-5."""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import OP_DIV, OP_REPL, OP_SUB, TOL_REL, SkyModelParams, small
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import GPUSkyModel

pytestmark = pytest.mark.gpu

GAUSS_TYPES = [U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC]


def _run(uv, sky, p, flavor=_lib.OBIT_DFT_RECUR, K=0, xyz=None, exact=True):
    out = uv.copy()
    q = SkyModelParams(**{**p.__dict__, "nVisPIO": max(1, uv.nvis)})
    gm = GPUSkyModel("mixed")
    try:
        gm.DFTInit(sky, out, q, exact_freq=exact)
        gm.set_kernel(flavor, K, 0)
        gm.DFTSetMod(sky)
        if xyz is not None:
            gm.set_positions_fp64(xyz)
        info = gm.plan_info()
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    return out, info


def _errors(got, uv, sky, p, xyz=None, exact=True):
    """Max error of the selected polarizations against the oracle's result."""
    want = oracle.apply_fp64(uv, sky, p, xyz=xyz, exact=exact)
    _, l1 = oracle.model_fp64(uv, sky, p, xyz=xyz, exact=exact)
    a = got.vis_view()[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    if p.op == OP_DIV:  # data 1 + 0i: the divided data is 1 / M
        sel = b[..., 2] > 0
        ga = 1.0 / (a[..., 0] + 1j * a[..., 1])
        wa = 1.0 / (b[..., 0] + 1j * b[..., 1])
        e = np.nanmax(np.where(sel, np.abs(ga - wa) / l1[..., None], 0))
        w = np.nanmax(np.where(sel, np.abs(a[..., 2] - b[..., 2]) / np.maximum(l1[..., None], 1e-30), 0))
        return float(max(e, w))
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert np.array_equal(a[..., 2], b[..., 2])  # weights untouched
    return float(np.nanmax(d / l1[..., None]))


def _mixed(mod, seed=21, **kw):
    args = dict(nrow=40, nchan=64, nif=2, ncomp=2500, seed=seed, alpha=(-0.9, -0.3), gauss_frac=0.3)
    args.update(kw)
    return small(mod, **args)


@pytest.mark.parametrize("mod", GAUSS_TYPES)
@pytest.mark.parametrize("K", [32, 16])
def test_mixed_matches_the_oracle(mod, K):
    uv, sky = _mixed(mod)
    npt = int(np.sum(np.all(sky.comps[:, 4:7] == 0, axis=1)))
    out, info = _run(uv, sky, SkyModelParams(op=OP_REPL), K=K)
    assert info["mixed"] == 1 and info["ncompPoint"] == npt and info["K"] == K, info
    assert 0 < npt < sky.ncomp
    assert _errors(out, uv, sky, SkyModelParams(op=OP_REPL)) < TOL_REL


@pytest.mark.parametrize("op", [OP_SUB, OP_DIV, OP_REPL])
def test_mixed_operations_with_flags(op):
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=22, flag_frac=0.1)
    if op == OP_DIV:
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    p = SkyModelParams(op=op)
    out, info = _run(uv, sky, p)
    assert info["mixed"] == 1
    assert _errors(out, uv, sky, p) < TOL_REL


def test_chain_comparator_keeps_one_table():
    """OBIT_DFT_RECUR_CHAIN runs the whole Gaussian table in the chain form;
    both agree within the bound."""
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=23)
    p = SkyModelParams(op=OP_REPL)
    a, ia = _run(uv, sky, p)
    b, ib = _run(uv, sky, p, flavor=_lib.OBIT_DFT_RECUR_CHAIN)
    assert ia["mixed"] == 1 and ib["mixed"] == 0 and ib["specFactored"] == 0
    assert _errors(a, uv, sky, p) < TOL_REL
    assert _errors(b, uv, sky, p) < TOL_REL


def test_all_points_in_a_gaussian_table():
    """A Gaussian table whose components are all untapered runs as the point
    family in the spectral-factored form."""
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=24, gauss_frac=0.0)
    p = SkyModelParams(op=OP_REPL)
    out, info = _run(uv, sky, p)
    assert info["mixed"] == 0 and info["specFactored"] == 1
    assert _errors(out, uv, sky, p) < TOL_REL


def test_only_gaussians_keep_the_chain_form():
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=25, gauss_frac=1.0, ncomp=600)
    p = SkyModelParams(op=OP_SUB)
    out, info = _run(uv, sky, p)
    assert info["mixed"] == 0 and info["specFactored"] == 0
    assert _errors(out, uv, sky, p) < TOL_REL


def test_wide_spread_points_keep_one_table():
    """Few point components with indices far apart: the point rows fail the
    residual bound and the whole table runs in the chain form."""
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=26, ncomp=90, alpha=(-3.0, 2.0))
    p = SkyModelParams(op=OP_SUB)
    out, info = _run(uv, sky, p)
    assert info["mixed"] == 0
    assert _errors(out, uv, sky, p) < TOL_REL


@pytest.mark.parametrize("mod", GAUSS_TYPES)
def test_fp32_frequency_ratios_keep_one_table(mod):
    """With only the reference's FP32 freqScale the channel frequencies are not
    uniform to FP64 precision: short blocks, no factored form, so the whole
    table runs in the chain form."""
    uv, sky = _mixed(mod, seed=28, ncomp=900)
    p = SkyModelParams(op=OP_SUB)
    out, info = _run(uv, sky, p, exact=False)
    assert info["mixed"] == 0 and info["K"] == 2
    assert _errors(out, uv, sky, p, exact=False) < TOL_REL


def test_fp64_positions_keep_one_table():
    """FP64 positions with a Gaussian table: no split (the FP64-position
    instances read the caller's order)."""
    uv, sky = _mixed(U.MOD_GAUSS_SPEC, seed=27, ncomp=800, max_bl=3e5, radius_deg=3.0)
    p = SkyModelParams(op=OP_SUB)
    out, info = _run(uv, sky, p, xyz=sky.xyz)
    assert info["mixed"] == 0
    assert _errors(out, uv, sky, p, xyz=sky.xyz) < TOL_REL


def test_config3_layout_sampled_rows():
    """The config-3 layout (4 IF x 256 channels, 50,000 components, 70 %
    untapered, indices over [-1.5, 0.5]) on rows spread over the track."""
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    from bench import workload_geometry
    g = workload_geometry("config3", 0, None, None)
    idx = np.linspace(0, g.rows - 1, 12).astype(int)
    uv = U.make_uvdata(g.uvw[idx], g.nstok, g.nchan, g.nif, g.freq, g.fa, np.random.default_rng(7))
    p = SkyModelParams(op=OP_REPL)
    out, info = _run(uv, g.sky, p)
    assert info["mixed"] == 1 and info["K"] == 32
    e = _errors(out, uv, g.sky, p)
    print(f"MIXED config3: max {e:.3e}, {info['ncompPoint']} point components")
    assert e < TOL_REL
