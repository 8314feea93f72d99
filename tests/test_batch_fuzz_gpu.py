"""Seeded random multi-facet batches against the FP64 oracle, facet by
facet: 2 to 9 facets of random model families (so several persistent kernels
share one graph), layouts, row and component counts (an empty model at
times) and operations; half the batches autotuned first."""
import numpy as np
import pytest

from obit_b200 import uvdata as U
from obit_b200.batch import DFTBatch
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB
from test_batch_gpu import _check_facet, _facets

pytestmark = pytest.mark.gpu

TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC]


@pytest.mark.parametrize("seed", range(8))
def test_random_batch(seed):
    torch = pytest.importorskip("torch")
    r = np.random.default_rng(11000 + seed)
    specs = []
    for i in range(int(r.integers(2, 10))):
        ncomp = 0 if r.random() < 0.1 else int(r.integers(1, 1500))
        specs.append((int(r.choice(TYPES)), int(r.integers(1, 120)), int(r.choice([8, 17, 32, 64])),
                      int(r.choice([1, 2, 3])), int(r.choice([1, 2, 4])), ncomp, int(r.integers(0, 10 ** 6)),
                      int(r.choice([OP_SUB, OP_REPL, OP_DIV]))))
    fs, keep = _facets(specs, torch)
    for f in fs:  # division on data 1 + 0i
        if f[2].op == OP_DIV:
            v = f[0].vis_view()
            v[..., 0] = 1.0
            v[..., 1] = 0.0
            f[3].copy_(torch.from_numpy(f[0].vis))
    b = DFTBatch([f[4] for f in fs])
    try:
        if seed % 2:
            b.autotune()
        b.run()
        torch.cuda.synchronize()
        for uv, sky, p, d_vis, _ in fs:
            _check_facet(uv, sky, p, d_vis.cpu().numpy())
    finally:
        b.close()
