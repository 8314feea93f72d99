"""Seeded random cases of the beam-corrected DFT against the FP64 beam
oracle: model family, Stokes of the sky, linear or circular feeds, 2 or 4
correlations, antenna types, Jones planes, channel and IF counts, component
counts, parallactic angle, the three operations with flags; channel runs
long enough for several 16-channel tiles of the tensor-core form, which the
point families take by default, and the FP32 block form drawn for some."""
import numpy as np
import pytest

import oracle
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams
from test_beam_gpu import _check, _run_beam
from test_beam_oracle_cpu import beam_case

pytestmark = pytest.mark.gpu

TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC]


@pytest.mark.parametrize("seed", range(24))
def test_random_case(seed):
    torch = pytest.importorskip("torch")
    r = np.random.default_rng(9000 + seed)
    kw = dict(mt=int(r.choice(TYPES)), nstok=int(r.choice([2, 4])), nrow=int(r.integers(1, 50)),
              nchan=int(r.choice([1, 7, 8, 13, 24, 40, 130, 300])), nif=int(r.choice([1, 2, 3])),
              ncomp=int(r.integers(1, 200)), seed=int(r.integers(0, 10 ** 6)), ntype=int(r.choice([1, 2, 3])),
              njc=int(r.choice([1, 2, 5])), flag_frac=float(r.choice([0.0, 0.1])),
              stok=int(r.choice([1, 2, 3, 4])), par_ang=float(r.uniform(-1.5, 1.5)),
              circular=bool(r.random() < 0.4))
    op = int(r.choice([OP_SUB, OP_REPL, OP_DIV]))
    flavor = _lib.OBIT_DFT_RECUR_CHAIN if r.random() < 0.25 else _lib.OBIT_DFT_RECUR
    uv, sky, beam = beam_case(**kw)
    if op == OP_DIV:
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    p = SkyModelParams(op=op)
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, op)
