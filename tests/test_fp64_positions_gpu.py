"""FP64 component positions (obit_dft_set_mod_d): on a 22 GHz, 8000 km array
with the components 0.3 deg from the phase centre, phases reach ~1e7 rad, so the
FP32 X, Y, Z of the reference's component table already move the phase by up to
about a radian.  With the FP64 side table both kernels must match the FP64
oracle evaluated at the FP64 positions within the parity tolerance; without it
they match the oracle at the table's FP32 positions, and dropping the side table
restores that result bit for bit."""
import numpy as np
import pytest

import oracle
from helpers import OBIT_DFT_PLAIN, OBIT_DFT_RECUR, TOL_REL
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_REPL, OP_SUB, GPUSkyModel, SkyModelParams

pytestmark = pytest.mark.gpu


def _vlbi_sample(nrow=48, ncomp=1500):
    """Rows spread over the track of the 22 GHz / 8000 km workload (32
    antennas, 8 IFs x 64 channels) and points within 2 arcmin of a position
    0.3 deg from the phase centre."""
    w = U.config4(nint=6, ncomp=ncomp)
    idx = np.linspace(0, w.uv.nvis - 1, nrow).astype(int)
    uv = U.make_uvdata(w.uv.vis[idx, :3].astype(np.float64), 2, 64, 8, w.uv.freq, w.uv.freqArr,
                       np.random.default_rng(9), flag_frac=0.05)
    return uv, w.sky


def _run(uv, sky, p, flavor, xyz=None, drop=False):
    out = uv.copy()
    q = SkyModelParams(**{**p.__dict__, "nVisPIO": uv.nvis})
    gm = GPUSkyModel("fp64pos")
    try:
        gm.DFTInit(sky, out, q)
        gm.set_kernel(flavor)
        gm.DFTSetMod(sky)
        if xyz is not None:
            gm.set_positions_fp64(xyz)
        if drop:
            gm.set_positions_fp64(None)
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    return out.vis


def _err(got, want, l1, uv):
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    return float(np.nanmax(d / l1[..., None]))


@pytest.mark.parametrize("flavor", [OBIT_DFT_RECUR, OBIT_DFT_PLAIN])
def test_fp64_positions_match_the_fp64_oracle(flavor):
    uv, sky = _vlbi_sample()
    p = SkyModelParams(op=OP_REPL)
    _, l1 = oracle.model_fp64(uv, sky, p, xyz=sky.xyz)
    want64 = oracle.apply_fp64(uv, sky, p, xyz=sky.xyz)
    want32 = oracle.apply_fp64(uv, sky, p)
    # the FP32 table alone is far from the FP64-position sky at these phases
    assert _err(want32, want64, l1, uv) > 1e-2
    got = _run(uv, sky, p, flavor, xyz=sky.xyz)
    assert _err(got, want64, l1, uv) < TOL_REL
    got32 = _run(uv, sky, p, flavor)
    assert _err(got32, want32, l1, uv) < TOL_REL


def test_dropping_the_side_table_restores_the_fp32_result():
    uv, sky = _vlbi_sample(nrow=24, ncomp=400)
    p = SkyModelParams(op=OP_SUB)
    a = _run(uv, sky, p, OBIT_DFT_RECUR)
    b = _run(uv, sky, p, OBIT_DFT_RECUR, xyz=sky.xyz, drop=True)
    assert np.array_equal(a, b)


def test_side_table_must_cover_the_model():
    uv, sky = _vlbi_sample(nrow=8, ncomp=50)
    out = uv.copy()
    gm = GPUSkyModel("fp64pos-short")
    try:
        gm.DFTInit(sky, out, SkyModelParams(op=OP_SUB, nVisPIO=uv.nvis))
        gm.DFTSetMod(sky)
        with pytest.raises(_lib.DFTError) as e:
            gm.set_positions_fp64(sky.xyz[:10])
        assert e.value.code == 1 and "FP64 positions" in str(e.value)
        gm.DFTShutdown()
    finally:
        gm.close()


ALL_TYPES = [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS, U.MOD_GAUSS_SPEC,
             U.MOD_GAUSS_TSPEC]


@pytest.mark.parametrize("flavor", [OBIT_DFT_RECUR, OBIT_DFT_PLAIN])
@pytest.mark.parametrize("mt,nterm", [(m, 1) for m in ALL_TYPES] + [(U.MOD_POINT_SPEC, 2)])
def test_fp64_position_instances_of_every_family(mt, nterm, flavor):
    """Every model family (and the 16-channel blocks of two spectral terms)
    through the FP64-position kernel instances: 300 km baselines at 1.4 GHz,
    components within 3 deg, subtract with flags."""
    from helpers import small
    uv, sky = small(mt, nrow=40, nchan=40, nif=2, nstok=2, ncomp=160, seed=31 + mt, max_bl=3e5,
                    radius_deg=3.0, nterm=nterm, flag_frac=0.05)
    p = SkyModelParams(op=OP_SUB)
    _, l1 = oracle.model_fp64(uv, sky, p, xyz=sky.xyz)
    want = oracle.apply_fp64(uv, sky, p, xyz=sky.xyz)
    got = _run(uv, sky, p, flavor, xyz=sky.xyz)
    assert _err(got, want, l1, uv) < TOL_REL
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    assert np.array_equal(a[..., 2], uv.vis_view()[..., 2])  # weights untouched by subtract
