"""Records resident across CLEAN major cycles (obit_dft_resident_*): two
cycles on one upload, the first subtracting a DFT model, the second a
different DFT model and a gridded one; each residual against the oracle, and
the uploaded records unchanged by the cycles."""
import numpy as np
import pytest

import oracle
import oracle_grid as G
from grid_helpers import dft_sky, field_case
from obit_b200 import grid as GR
from obit_b200.resident import ResidentUV
from obit_b200.skymodel import OP_SUB, GPUSkyModel, SkyModelParams

pytestmark = pytest.mark.gpu


def _dft_device(sky, uv, d_ptr, p):
    gm = GPUSkyModel("resident")
    try:
        gm.DFTInit(sky, uv, SkyModelParams(**{**p.__dict__, "nVisPIO": uv.nvis}), exact_freq=False)
        gm.DFTSetMod(sky)
        gm.calc_device(d_ptr, uv.nvis, 0)
        gm.check()
        gm.DFTShutdown()
    finally:
        gm.close()


def _rel(got, want, uv, l1):
    a = got.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    return float(np.max(d / l1[..., None]))


def test_two_major_cycles_on_one_upload():
    f, img, m, uv = field_case(N=96, seed=40, ncomp=200, nint=6)
    skyA = dft_sky(f, m)
    half = len(f.flux) // 2
    from obit_b200.comps import CCField
    fB = CCField(**{**f.__dict__, "flux": f.flux[:half], "deltaX": f.deltaX[:half], "deltaY": f.deltaY[:half]})
    fC = CCField(**{**f.__dict__, "flux": f.flux[half:], "deltaX": f.deltaX[half:], "deltaY": f.deltaY[half:]})
    p = SkyModelParams(op=OP_SUB)
    _, l1 = oracle.model_fp64(uv, skyA, p, exact=False)
    with ResidentUV(uv) as r:
        # cycle 1: the whole field by the DFT
        r.reset()
        _dft_device(skyA, uv, r.d_records, p)
        res1 = r.download()
        want1 = oracle.apply_fp64(uv, skyA, p, exact=False)
        assert _rel(res1, want1, uv, l1) < 1e-5
        # cycle 2: half by the DFT, half gridded (exact kernel), from the same upload
        r.reset()
        _dft_device(dft_sky(fB, m), uv, r.d_records, p)
        with GR.GridField(fC, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m,
                          kernel=GR.KERNEL_EXACT) as gf:
            gf.FTGrid_device(uv, r.d_records, uv.nvis, p)
        res2 = r.download()
        assert _rel(res2, want1, uv, l1) < 1e-5
        # a reset alone gives back the uploaded records
        r.reset()
        np.testing.assert_array_equal(r.download().vis, uv.vis)
