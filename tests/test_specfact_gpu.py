"""GPU parity of the spectral-factored recurrence: point components with one
spectral index (PointSpec with one term, PointTSpec) evaluated as G_b H_a with
the linear part of the block's spectral exponent on a non-unit step and the
tile's common quadratic factor applied when the tile's sums are folded.  The
library orders its copy of the table by spectral index; the planner takes this
form only when every tile's residual bound holds, else the chain form.

Each case checks which form ran (plan info) and compares the model with the
FP64 oracle, |V_gpu - V_fp64| / sum_c |A_c| < 1e-5 per visibility."""
import numpy as np
import pytest

import oracle
from helpers import OP_DIV, OP_REPL, OP_SUB, TOL_REL, SkyModelParams, small
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import GPUSkyModel

pytestmark = pytest.mark.gpu

SPEC_TYPES = [U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC]


def _run(uv, sky, p, flavor=_lib.OBIT_DFT_RECUR, K=0, ct=0, xyz=None):
    """Apply the model; returns (records, plan info)."""
    out = uv.copy()
    q = SkyModelParams(**{**p.__dict__, "nVisPIO": max(1, uv.nvis)})
    gm = GPUSkyModel("specfact")
    try:
        gm.DFTInit(sky, out, q)
        gm.set_kernel(flavor, K, ct)
        gm.DFTSetMod(sky)
        if xyz is not None:
            gm.set_positions_fp64(xyz)
        info = gm.plan_info()
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    return out, info


def _model_err(uv, sky, p, **kw):
    """Max |model - FP64 oracle| / sum|A| of the first selected polarization,
    the model taken by the replace operation."""
    q = SkyModelParams(**{**p.__dict__, "op": OP_REPL, "doFlip": False, "stokFactor": 1.0})
    out, info = _run(uv, sky, q, **kw)
    v = out.vis_view()[..., 0, :]
    g = v[..., 0].astype(np.float64) + 1j * v[..., 1].astype(np.float64)
    m, l1 = oracle.model_fp64(uv, sky, q, xyz=kw.get("xyz"))
    sel = ~np.isnan(l1)
    rel = np.abs(g - m)[sel] / np.maximum(l1[sel], 1e-30)
    return float(rel.max()), info


def _dense(mod, seed=3, **kw):
    """Many components over a modest spectral-index range: sorted tiles are
    narrow enough for the spectral-factored form."""
    args = dict(nrow=48, nchan=64, nif=2, ncomp=2000, seed=seed, alpha=(-0.9, -0.3))
    args.update(kw)
    return small(mod, **args)


@pytest.mark.parametrize("mod", SPEC_TYPES)
@pytest.mark.parametrize("K", [32, 16, 8])
def test_factored_matches_the_oracle(mod, K):
    uv, sky = _dense(mod)
    mx, info = _model_err(uv, sky, SkyModelParams(), K=K)
    assert info["specFactored"] == 1 and info["K"] == K, info
    assert mx < TOL_REL, mx


@pytest.mark.parametrize("mod", SPEC_TYPES)
def test_chain_comparator_agrees(mod):
    """The chain form (OBIT_DFT_RECUR_CHAIN) on the same input: both within the
    bound of the oracle and of each other."""
    uv, sky = _dense(mod, seed=4)
    p = SkyModelParams()
    a, ia = _run(uv, sky, SkyModelParams(op=OP_REPL))
    b, ib = _run(uv, sky, SkyModelParams(op=OP_REPL), flavor=_lib.OBIT_DFT_RECUR_CHAIN)
    assert ia["specFactored"] == 1 and ib["specFactored"] == 0
    _, l1 = oracle.model_fp64(uv, sky, p)
    va, vb = a.vis_view()[..., 0, :], b.vis_view()[..., 0, :]
    d = np.abs((va[..., 0] - vb[..., 0]) + 1j * (va[..., 1] - vb[..., 1]))
    assert float(np.nanmax(d / l1)) < TOL_REL
    mx, _ = _model_err(uv, sky, p, flavor=_lib.OBIT_DFT_RECUR_CHAIN)
    assert mx < TOL_REL


def test_partial_blocks_and_selection():
    """40 channels (blocks of 32 and 8) with a channel and IF selection."""
    uv, sky = _dense(U.MOD_POINT_SPEC, nchan=40, nif=3, seed=5)
    p = SkyModelParams(startChannel=3, numberChannel=35, startIF=2, numberIF=2)
    mx, info = _model_err(uv, sky, p)
    assert info["specFactored"] == 1
    assert mx < TOL_REL


@pytest.mark.parametrize("op", [OP_SUB, OP_DIV, OP_REPL])
def test_operations_with_flags(op):
    uv, sky = _dense(U.MOD_POINT_SPEC, seed=6, flag_frac=0.1, ncomp=1500, alpha=(-0.9, -0.4))
    if op == OP_DIV:  # data 1 + 0i: the divided data is 1 / M
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    p = SkyModelParams(op=op)
    got, info = _run(uv, sky, p)
    assert info["specFactored"] == 1
    want = oracle.apply_fp64(uv, sky, p)
    _, l1 = oracle.model_fp64(uv, sky, p)
    a = got.vis_view()[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    if op == OP_DIV:
        sel = b[..., 2] > 0
        ga = 1.0 / (a[..., 0] + 1j * a[..., 1])
        wa = 1.0 / (b[..., 0] + 1j * b[..., 1])
        assert np.nanmax(np.where(sel, np.abs(ga - wa) / l1[..., None], 0)) < TOL_REL
        wrel = np.abs(a[..., 2] - b[..., 2]) / np.maximum(l1[..., None], 1e-30)
        assert np.nanmax(np.where(sel, wrel, 0)) < TOL_REL
        return
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert float(np.nanmax(d / l1[..., None])) < TOL_REL
    assert np.array_equal(a[..., 2], b[..., 2])


def test_wide_spread_keeps_the_chain_form():
    """A few components whose indices are far apart share one tile: the
    residual bound fails and the planner keeps the chain form."""
    uv, sky = small(U.MOD_POINT_SPEC, nrow=40, nchan=64, nif=2, ncomp=60, seed=7, alpha=(-3.0, 2.0))
    mx, info = _model_err(uv, sky, SkyModelParams())
    assert info["specFactored"] == 0
    assert mx < TOL_REL


def test_equal_indices_and_ties():
    """Every component with the same index (ties in the ordering)."""
    uv, sky = _dense(U.MOD_POINT_SPEC, seed=8, ncomp=700, alpha=(-0.7, -0.7))
    mx, info = _model_err(uv, sky, SkyModelParams())
    assert info["specFactored"] == 1
    assert mx < TOL_REL


def test_fp64_positions_follow_the_ordering():
    """FP64 positions (side table in the caller's order) with the ordered copy:
    300 km baselines, components within 3 deg."""
    uv, sky = _dense(U.MOD_POINT_SPEC, seed=9, nrow=40, nchan=40, max_bl=3e5, radius_deg=3.0,
                     alpha=(-0.8, -0.5), flag_frac=0.05)
    mx, info = _model_err(uv, sky, SkyModelParams(), xyz=sky.xyz)
    assert info["specFactored"] == 1
    assert mx < TOL_REL


def test_config2_layout_sampled_rows():
    """The config-2 layout (4 IF x 256 channels, 20,000 components with
    indices over [-1.5, 0.5], w-term) on rows spread over the track: the
    default plan is spectral-factored, and both forms meet the bound."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    from bench import workload_geometry
    g = workload_geometry("config2", 0, None, None)
    idx = np.linspace(0, g.rows - 1, 24).astype(int)
    uv = U.make_uvdata(g.uvw[idx], g.nstok, g.nchan, g.nif, g.freq, g.fa, np.random.default_rng(7))
    mx, info = _model_err(uv, g.sky, SkyModelParams())
    assert info["specFactored"] == 1 and info["K"] == 32
    assert mx < TOL_REL
    mc, ic = _model_err(uv, g.sky, SkyModelParams(), flavor=_lib.OBIT_DFT_RECUR_CHAIN)
    assert ic["specFactored"] == 0
    assert mc < TOL_REL
    print(f"SPECFACT config2: factored max {mx:.3e}, chain max {mc:.3e}")
