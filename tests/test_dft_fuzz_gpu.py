"""Seeded random cases of the DFT path against the FP64 oracle: every model
family, channel and IF counts that leave partial blocks, polarization counts,
channel / IF / polarization selections, the three operations with flags, the
FP64 and FP32 frequency interfaces, and component counts from one to a few
thousand (spectral indices spread wide enough that some tables fail the
spectral-factored bound and others pass it).  Bound: the north-star
|V - V_fp64| / sum_c |A_c| < 1e-5 per visibility; weights exact except where
divided."""
import numpy as np
import pytest

import oracle
from helpers import OP_DIV, OP_REPL, OP_SUB, TOL_REL, SkyModelParams, run_gpu, small
from obit_b200 import uvdata as U

pytestmark = pytest.mark.gpu

TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC]


def _case(seed):
    r = np.random.default_rng(7000 + seed)
    mod = int(r.choice(TYPES))
    nchan = int(r.choice([1, 5, 17, 33, 64, 100]))
    nif = int(r.choice([1, 2, 3]))
    nstok = int(r.choice([1, 2, 4]))
    lo = float(r.uniform(-2.0, 0.0))
    kw = dict(nrow=int(r.integers(1, 60)), nchan=nchan, nif=nif, nstok=nstok, ncomp=int(r.integers(1, 3000)),
              seed=int(r.integers(0, 10 ** 6)), flag_frac=float(r.choice([0.0, 0.15])),
              alpha=(lo, lo + float(r.choice([0.05, 0.6, 2.5]))), gauss_frac=float(r.uniform(0, 1)),
              nterm=int(r.choice([1, 2])) if mod in (U.MOD_POINT_SPEC, U.MOD_GAUSS_SPEC) else 1,
              max_bl=float(r.choice([3e3, 36e3, 3e5])))
    c0 = int(r.integers(1, nchan + 1))
    i0 = int(r.integers(1, nif + 1))
    s0 = int(r.integers(1, min(2, nstok) + 1))
    p = SkyModelParams(op=int(r.choice([OP_SUB, OP_REPL, OP_DIV])), startChannel=c0,
                       numberChannel=int(r.integers(1, nchan - c0 + 2)), startIF=i0,
                       numberIF=int(r.integers(1, nif - i0 + 2)), startPoln=s0,
                       numberPoln=int(r.integers(1, min(2, nstok) - s0 + 2)))
    exact = bool(r.random() < 0.7)
    return mod, kw, p, exact


@pytest.mark.parametrize("seed", range(48))
def test_random_case(seed):
    mod, kw, p, exact = _case(seed)
    uv, sky = small(mod, **kw)
    if p.op == OP_DIV:  # data 1 + 0i: the divided data is 1 / M
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    got = run_gpu(uv, sky, p, exact=exact)
    want = oracle.apply_fp64(uv, sky, p, exact=exact)
    _, l1 = oracle.model_fp64(uv, sky, p, exact=exact)
    a = got.vis_view()
    b = want[:, uv.nrparm:].reshape(a.shape)
    # unselected correlations and random parameters untouched
    np.testing.assert_array_equal(got.vis[:, :uv.nrparm], uv.vis[:, :uv.nrparm])
    sel = ~np.isnan(l1)
    ps = slice(p.startPoln - 1, p.startPoln - 1 + p.numberPoln)
    pol = np.zeros(a.shape[3], bool)
    pol[ps] = True
    mask = sel[..., None] & pol
    np.testing.assert_array_equal(a[~mask], uv.vis_view()[~mask])
    if p.op == OP_DIV:
        ok = mask & (b[..., 2] > 0)
        ga = 1.0 / (a[..., 0] + 1j * a[..., 1])
        wa = 1.0 / (b[..., 0] + 1j * b[..., 1])
        rel = np.abs(ga - wa) / np.broadcast_to(l1[..., None], ga.shape)
        assert float(np.max(np.where(ok, rel, 0))) < TOL_REL, (mod, kw, p)
        return
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    # the records are FP32: a subtraction's result is rounded to the data's
    # precision, which a heavily tapered model's L1 norm may not reach
    d = np.maximum(d - 2.0 ** -22 * np.abs(b[..., 0] + 1j * b[..., 1]), 0.0)
    rel = d / np.broadcast_to(np.where(sel, l1, 1.0)[..., None], d.shape)
    assert float(np.max(np.where(mask, rel, 0))) < TOL_REL, (mod, kw, p, float(np.max(rel)))
    np.testing.assert_array_equal(a[..., 2], b[..., 2])
