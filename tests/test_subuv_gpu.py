"""The SubUV pass structure over the GPU paths (obit_b200.subuv.sub_uv): a
two-field model (one 2-D field at the phase centre, one 3-D field off it)
applied by the DFT (all fields in one pass) and by the gridded model (a pass
per field, exact kernel) gives the oracle's result; the chosen mode follows
ObitSkyModelChose."""
import numpy as np
import pytest

import oracle
from grid_helpers import dft_sky, field_case
from obit_b200 import grid as GR
from obit_b200.comps import load_comps
from obit_b200.skymodel import OP_SUB, SkyModelParams
from obit_b200.subuv import sub_uv

pytestmark = pytest.mark.gpu


def test_two_fields_by_dft_and_by_grid():
    f1, img1, m, uv = field_case(N=96, seed=50, ncomp=120, nint=5)
    f2, img2, m3, _ = field_case(N=96, seed=51, ncomp=80, nint=5, shift3d=True)
    m.do3D = True  # the model's flag: 3-D re-projection for the shifted field
    fields, images = [f1, f2], [img1, img2]
    gimages = [GR.GridImage(i.nx, i.ny, i.crpixX, i.crpixY) for i in images]
    p = SkyModelParams(op=OP_SUB)
    sky, _ = load_comps(fields, m)
    want = oracle.apply_fp64(uv, sky, p, exact=False)
    _, l1 = oracle.model_fp64(uv, sky, p, exact=False)
    for mode, kernel in ((GR.MODE_DFT, GR.KERNEL_REFERENCE), (GR.MODE_GRID, GR.KERNEL_EXACT)):
        r = sub_uv(uv, fields, gimages, m, p, mode=mode, kernel=kernel)
        assert r.mode == mode
        a = r.uv.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
        b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
        d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1])) / l1[..., None]
        assert float(d.max()) < 1e-5, (mode, float(d.max()))
    np.testing.assert_array_equal(uv.vis, field_case(N=96, seed=50, ncomp=120, nint=5)[3].vis)


def test_fastest_follows_the_reference_choice():
    f1, img1, m, uv = field_case(N=64, seed=52, ncomp=200, nint=3)
    gim = [GR.GridImage(img1.nx, img1.ny, img1.crpixX, img1.crpixY)]
    want = GR.choose_mode(GR.MODE_FASTEST, GR.TYPE_COMPS, [200], [64], [64], uv.nvis, uv.nchan * uv.nif)
    r = sub_uv(uv, [f1], gim, m, SkyModelParams(op=OP_SUB))
    assert r.mode == want
    r2 = sub_uv(uv, [f1], gim, m, SkyModelParams(op=OP_SUB), measured=True)
    assert r2.mode == GR.MODE_DFT  # 200 components: the DFT on the B200


def test_mixed_dft_above_min_then_grid():
    """OBIT_SkyModel_Mixed: per field, the DFT of the components above minDFT,
    then the gridded model of those of at most maxGrid (the same threshold),
    exact kernel: the whole model is subtracted as the DFT oracle has it.  One
    component per cell, so the split by flux is the same for the DFT's merged
    table and the grid's rows."""
    from obit_b200.comps import CCModel
    fields, images = [], []
    f0, img0, m, uv = field_case(N=96, seed=60, ncomp=200, nint=5)
    for s_, f in ((60, f0), (61, field_case(N=96, seed=61, ncomp=150, nint=5, shift3d=True)[0])):
        cells = {}
        keep = [i for i, (x, y) in enumerate(zip(f.deltaX, f.deltaY)) if cells.setdefault((x, y), i) == i]
        f.flux, f.deltaX, f.deltaY = f.flux[keep], f.deltaX[keep], f.deltaY[keep]
        fields.append(f)
        images.append(GR.GridImage(img0.nx, img0.ny, img0.crpixX, img0.crpixY))
    m.do3D = True
    T = 0.4
    mm = CCModel(**{**m.__dict__, "minDFT": T})
    p = SkyModelParams(op=OP_SUB)
    r = sub_uv(uv, fields, images, mm, p, mode=GR.MODE_MIXED, maxGrid=T, kernel=GR.KERNEL_EXACT)
    assert r.mode == GR.MODE_MIXED
    sky, _ = load_comps(fields, m)
    assert r.ncomp >= sky.ncomp
    want = oracle.apply_fp64(uv, sky, p, exact=False)
    _, l1 = oracle.model_fp64(uv, sky, p, exact=False)
    a = r.uv.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1])) / l1[..., None]
    assert float(d.max()) < 1e-5, float(d.max())


def test_image_models_one_pass_per_field():
    """OBIT_SkyModel_Image through the pass structure (obit_dft_sub_uv_image):
    two fields' model images (clipped, blanked, scaled by factor) applied in
    field order give the oracle's image model of each, subtracted in turn."""
    import oracle_grid as G
    from obit_b200.comps import CCModel
    from obit_b200.subuv import sub_uv_image
    from test_grid_gpu import _image_of
    f1, img1, m, uv = field_case(N=96, seed=70, nint=5)
    f2, img2, _, _ = field_case(N=96, seed=71, nint=5, shift3d=True)
    m.do3D = True
    pix = [_image_of(f1, img1), _image_of(f2, img2)]
    pix[0][10, 12] = -999.0
    pix[1][40:44, 50:52] = 0.7
    m2 = CCModel(**{**m.__dict__, "factor": 0.5})
    p = SkyModelParams(op=OP_SUB)
    gims = [GR.GridImage(i.nx, i.ny, i.crpixX, i.crpixY) for i in (img1, img2)]
    r = sub_uv_image(uv, pix, -999.0, [f1, f2], gims, m2, p)
    assert r.ncomp == 2 * 96 * 96
    want = uv
    l1 = 0.0
    for px, f, img in zip(pix, (f1, f2), (img1, img2)):
        gm = G.build_image(px, -999.0, f, img, m2)
        l1 += gm.l1
        nxt = want.copy()
        nxt.vis = G.apply(gm, want, p)
        want = nxt
    a = r.uv.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert float(d.max()) / l1 < 1e-5, float(d.max()) / l1
