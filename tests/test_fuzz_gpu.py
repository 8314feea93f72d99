"""Seeded random layouts through the GPU path against the FP64 oracle: model
family and spectral terms, rows / channels / IFs / polarizations (1, 2 or 4
correlations), channel, IF and polarization selections, operation (subtract,
replace, divide), doFlip and stokFactor, flags, kernel flavor and channels per
thread, FP64 or FP32 frequency tables.  Inside the selection the records match
the oracle within the parity tolerance; outside it they are untouched."""
import numpy as np
import pytest

import oracle
from helpers import OBIT_DFT_PLAIN, OBIT_DFT_RECUR, TOL_REL, run_gpu, small
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

pytestmark = pytest.mark.gpu

FAMILIES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC,
            U.MOD_GAUSS_TSPEC]


def _draw(seed):
    r = np.random.default_rng(1000 + seed)
    mt = FAMILIES[seed % len(FAMILIES)]
    nterm = int(r.integers(1, 3)) if mt in (U.MOD_POINT_SPEC, U.MOD_GAUSS_SPEC) else 1
    nchan, nif = int(r.integers(1, 71)), int(r.integers(1, 5))
    nstok = int(r.choice([1, 2, 4]))
    uv, sky = small(mt, nrow=int(r.integers(1, 61)), nchan=nchan, nif=nif, nstok=nstok,
                    ncomp=int(r.integers(1, 401)), seed=2000 + seed, nterm=nterm,
                    flag_frac=float(r.uniform(0.0, 0.3)), radius_deg=float(r.uniform(0.05, 2.0)),
                    max_bl=float(r.uniform(1e3, 3e5)))
    sc = int(r.integers(1, nchan + 1))
    si = int(r.integers(1, nif + 1))
    npol = int(r.integers(1, min(2, nstok) + 1))
    sp = int(r.integers(1, nstok - npol + 2))
    op = [OP_SUB, OP_REPL, OP_DIV][int(r.integers(0, 3))]
    p = SkyModelParams(op=op, doFlip=bool(r.integers(0, 2)), stokFactor=float(r.choice([1.0, -1.0, 0.5])),
                       startChannel=sc, numberChannel=int(r.integers(1, nchan - sc + 2)),
                       startIF=si, numberIF=int(r.integers(1, nif - si + 2)), startPoln=sp, numberPoln=npol)
    flavor = OBIT_DFT_PLAIN if r.random() < 0.25 else OBIT_DFT_RECUR
    K = int(r.choice([0, 2, 4, 8, 16, 32])) if flavor == OBIT_DFT_RECUR else int(r.choice([0, 1, 4, 8, 16]))
    exact = bool(r.random() < 0.8)
    if op == OP_DIV:  # unit data: the quotient is 1/M, compared as the implied model
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    return uv, sky, p, flavor, K, exact


@pytest.mark.parametrize("seed", range(24))
def test_random_layout_matches_oracle(seed):
    uv, sky, p, flavor, K, exact = _draw(seed)
    got = run_gpu(uv, sky, p, flavor=flavor, K=K, exact=exact).vis
    want = oracle.apply_fp64(uv, sky, p, exact=exact)
    _, l1 = oracle.model_fp64(uv, sky, p, exact=exact)
    shape = uv.vis_view().shape  # (row, IF, chan, pol, 3)
    a = got[:, uv.nrparm:].reshape(shape)
    b = want[:, uv.nrparm:].reshape(shape)
    src = uv.vis_view()
    mask = np.zeros(shape[:-1], bool)
    c0, i0, p0 = p.startChannel - 1, p.startIF - 1, p.startPoln - 1
    mask[:, i0:i0 + p.numberIF, c0:c0 + p.numberChannel, p0:p0 + p.numberPoln] = True
    assert np.array_equal(a[~mask], src[~mask])  # outside the selection: untouched
    assert np.array_equal(got[:, :uv.nrparm], uv.vis[:, :uv.nrparm])
    if p.op != OP_DIV:
        assert np.array_equal(a[..., 2], b[..., 2])  # weights
    if sky.ncomp == 0 or not mask.any():
        return
    L = l1[:, :, :, None] * np.ones(shape[3])[None, None, None, :]
    if p.op == OP_DIV:
        sel = mask & (b[..., 2] > 0)
        ga = 1.0 / (a[..., 0] + 1j * a[..., 1])
        wa = 1.0 / (b[..., 0] + 1j * b[..., 1])
        # the implied models carry stokFactor^k (|stokFactor| <= 1 here), so
        # the L1 norm of the unscaled terms bounds them
        rel = np.abs(ga - wa) / np.maximum(L, 1e-30)
        assert np.nanmax(np.where(sel, rel, 0)) < 2 * TOL_REL
    else:
        d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
        rel = np.where(mask, d / np.maximum(L, 1e-30), 0)
        assert np.nanmax(rel) < TOL_REL + 1e-6
