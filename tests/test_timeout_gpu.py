"""The kernels' timeout path on a B200, without a GPU fault: with the
component-copy wait limited to zero polls (obit_dft_set_wait_limit) every CTA
gives up at its first tile -- after letting the copy in flight land -- sets the
device error flag and leaves its records untouched; the host reads the status
(OBIT_DFT_EKERNEL), and the same context then runs the normal path correctly."""
import numpy as np
import pytest

import oracle
from helpers import TOL_REL, small
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_SUB, GPUSkyModel, SkyModelParams

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flag_path", ["calc_device", "calc"])
def test_wait_that_gives_up_reports_and_context_survives(flag_path):
    torch = pytest.importorskip("torch")
    uv, sky = small(U.MOD_POINT_SPEC, nrow=120, nchan=64, nif=2, nstok=2, ncomp=500, seed=61)
    p = SkyModelParams(op=OP_SUB, nVisPIO=uv.nvis)
    lib = _lib.load()
    gm = GPUSkyModel("timeout")
    try:
        gm.DFTInit(sky, uv, p)
        gm.DFTSetMod(sky)
        _lib.check(lib.obit_dft_set_wait_limit(gm.gpuinfo, 0))
        if flag_path == "calc_device":
            d_vis = torch.from_numpy(uv.vis.copy()).cuda()
            gm.calc_device(d_vis.data_ptr(), uv.nvis, 0)
            with pytest.raises(_lib.DFTError) as e:
                gm.check()
            assert e.value.code == 4
            assert np.array_equal(d_vis.cpu().numpy(), uv.vis)  # nothing applied
        else:
            work = uv.copy()
            with pytest.raises(_lib.DFTError) as e:
                gm.DFTCalc(work)
            assert e.value.code == 4 or "error" in str(e.value).lower()
        # the default limit restored: the same context computes the model
        _lib.check(lib.obit_dft_set_wait_limit(gm.gpuinfo, -1))
        d_vis = torch.from_numpy(uv.vis.copy()).cuda()
        gm.calc_device(d_vis.data_ptr(), uv.nvis, 0)
        gm.check()
        got = d_vis.cpu().numpy()
        gm.DFTShutdown()
    finally:
        gm.close()
    want = oracle.apply_fp64(uv, sky, p)
    _, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert float(np.max(d / l1[..., None])) < TOL_REL
