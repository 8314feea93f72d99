"""Seeded random cases of the gridded model FT against the oracle's
restatement: image sizes (odd and even), component counts, baselines that reach
past the plane, channel counts that leave partial 32-pair chunks, 2-D and 3-D
fields, point and Gaussian models, both interpolation kernels, the three
operations with flags.  Bound: |dV| / sum|flux| < 1e-4 over every selected
correlation (edge windows of the reference kernel are ill-conditioned, so the
bound is looser than the interior cases' 1e-5); blanking and weights exact."""
import numpy as np
import pytest

import oracle_grid as G
from grid_helpers import field_case
from obit_b200 import grid as GR
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

pytestmark = pytest.mark.gpu


def _case(seed):
    r = np.random.default_rng(1000 + seed)
    kw = dict(N=int(r.choice([24, 31, 48, 64, 97])), ncomp=int(r.integers(1, 300)),
              seed=int(r.integers(0, 10 ** 6)), reach=float(r.uniform(0.3, 7.0)),
              nchan=int(r.choice([1, 3, 8, 33])), nif=int(r.choice([1, 2])), nint=int(r.integers(1, 4)),
              shift3d=bool(r.random() < 0.4), flag_frac=float(r.choice([0.0, 0.2])))
    if r.random() < 0.3:
        kw["gauss"] = (float(r.uniform(2, 8)), float(r.uniform(1, 2)), float(r.uniform(-90, 90)))
    kernel = int(r.choice([GR.KERNEL_REFERENCE, GR.KERNEL_EXACT]))
    op = int(r.choice([OP_SUB, OP_REPL, OP_DIV]))
    return kw, kernel, op


@pytest.mark.parametrize("seed", range(32))
def test_random_case(seed):
    kw, kernel, op = _case(seed)
    f, img, m, uv = field_case(**kw)
    if op == OP_DIV:
        uv.vis_view()[..., 0] += 3.0
    p = SkyModelParams(op=op, stokFactor=-0.5, doFlip=bool(seed % 2))
    gm = G.build(f, img, m)
    want = G.apply(gm, uv, p, exact=(kernel == GR.KERNEL_EXACT))
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m, kernel=kernel) as gf:
        got = gf.FTGrid(uv, p).vis
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)
    np.testing.assert_array_equal(a[..., 2] == 0, b[..., 2] == 0)
    if op == OP_DIV:  # compare the models: data / result
        sel = b[..., 2] > 0
        v0 = uv.vis_view()
        d0 = (v0[..., 0] + 1j * v0[..., 1])[sel].astype(np.complex128)
        ma = d0 / (a[..., 0] + 1j * a[..., 1])[sel]
        mb = d0 / (b[..., 0] + 1j * b[..., 1])[sel]
        assert float(np.max(np.abs(ma - mb))) / gm.l1 < 1e-4, (kw, kernel)
        return
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    np.testing.assert_array_equal(a[..., 2], b[..., 2])
    assert float(d.max()) / gm.l1 < 1e-4, (kw, kernel, float(d.max()) / gm.l1)
