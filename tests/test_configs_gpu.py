"""Accuracy on the measured configurations: for configs 1-4 (the bench's seeded
geometry, a sample of rows spread over the track), the split-FP32 recurrence
kernel and the FP64-phase plain kernel against the FP64 oracle, with the
reference-faithful CPU restatement (FP32 phase, the reference's vector sin/cos)
beside them.  Error = |V - V_fp64| / sum_c |A_c| per visibility, over the
selected polarizations.  Each case prints one "CONFIGSTAT {json}" line."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import OBIT_DFT_PLAIN, OBIT_DFT_RECUR, TOL_REL, run_gpu
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_REPL, SkyModelParams

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
from bench import workload_geometry  # noqa: E402

SAMPLE = {"config1": 400, "config2": 48, "config3": 24, "config4": 160}


def _errors(out, want, l1, uv):
    shape = uv.vis_view().shape
    a = out[:, uv.nrparm:].reshape(shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1])) / l1[..., None]
    return float(d.max()), float(np.sqrt(np.mean(d ** 2)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config1", "config2", "config3", "config4"])
def test_config_accuracy(name):
    g = workload_geometry(name, 0, None, None)
    idx = np.linspace(0, g.rows - 1, SAMPLE[name]).astype(int)
    uv = U.make_uvdata(g.uvw[idx], g.nstok, g.nchan, g.nif, g.freq, g.fa, np.random.default_rng(7))
    p = SkyModelParams(op=OP_REPL)
    _, l1 = oracle.model_fp64(uv, g.sky, p)
    want = oracle.apply_fp64(uv, g.sky, p)
    stats = {"config": name, "rows": len(idx), "components": g.sky.ncomp,
             "evals": int(len(idx) * g.channels * g.sky.ncomp)}
    for label, flavor in (("recur", OBIT_DFT_RECUR), ("plain", OBIT_DFT_PLAIN)):
        out = run_gpu(uv, g.sky, p, flavor=flavor).vis
        stats[f"{label}_max"], stats[f"{label}_rms"] = _errors(out, want, l1, uv)
    if oracle.have_refcpu():
        stats["refcpu_max"], stats["refcpu_rms"] = _errors(oracle.apply_refcpu(uv, g.sky, p), want, l1, uv)
    print("CONFIGSTAT " + json.dumps(stats))
    assert stats["recur_max"] < TOL_REL
    assert stats["plain_max"] < TOL_REL
