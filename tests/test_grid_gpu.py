"""GPU parity of the gridded model FT (obit_dft_grid_* through the C ABI)
against the oracle's restatement of the reference's gridded path and, with
exact Lagrange weights, against the DFT oracle.

Bounds (per (record, IF, channel), relative to sum |flux| of the field, the
bound of every plane value): the plane within 1e-5 of the oracle's FP64 FFT
plane; the reference-kernel model within 1e-5 of the oracle's (the GPU picks
the same windows and table rows: single-precision steps in the reference's
order); the exact-kernel model within 1e-5 of the DFT oracle."""
import numpy as np
import pytest

import oracle
import oracle_grid as G
from grid_helpers import dft_sky, field_case, with_pa
from obit_b200 import _lib
from obit_b200 import grid as GR
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _l1(field):
    return float(np.abs(np.asarray(field.flux, np.float64)).sum())


def _gpu_model(field, image, model, uv, kernel=GR.KERNEL_REFERENCE, params=None):
    """Model per (record, IF, channel) of the first selected polarization,
    taken with the replace operation: complex128 (nvis, nif, nchan)."""
    p = params or SkyModelParams()
    q = SkyModelParams(**{**p.__dict__, "op": OP_REPL, "stokFactor": 1.0})
    with GR.GridField(field, GR.GridImage(image.nx, image.ny, image.crpixX, image.crpixY), model,
                      kernel=kernel) as gf:
        out = gf.FTGrid(uv, q)
        info = gf.info()
    pol0 = (q.startPoln if q.startPoln > 0 else 1) - 1
    v = out.vis_view()[..., pol0, :]
    return v[..., 0].astype(np.float64) + 1j * v[..., 1].astype(np.float64), info, out


@pytest.mark.parametrize("gauss", [None, (6.0, 3.0, 30.0)])
def test_plane_matches_the_oracle(gauss):
    f, img, m, uv = field_case(N=96, seed=21, gauss=gauss)
    grid, n, gparm, _ = G.grid_comps(f, img)
    want = G.ft_plane(grid, gparm, f, img)
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m) as gf:
        got = gf.plane()
        info = gf.info()
    assert info["ncomp"] == n and info["gauss"] == int(gauss is not None)
    assert got.shape == want.shape
    err = np.abs(got.astype(np.complex128) - want).max() / _l1(f)
    assert err < TOL, err


REF_CASES = {"point": {}, "gauss": {"gauss": (6.0, 3.0, 30.0)}, "shift3d": {"shift3d": True},
             "rot3d": {"shift3d": True, "rotation": 12.0, "uv_rotation": -5.0},
             "nonsquare_gauss": {"Ny": 64, "gauss": (5.0, 4.0, -40.0)}}


@pytest.mark.parametrize("case", list(REF_CASES))
def test_reference_kernel_matches_the_oracle(case):
    f, img, m, uv = field_case(N=96, seed=22, nint=6, **REF_CASES[case])
    got, info, _ = _gpu_model(f, img, m, uv)
    want = G.model_values(G.build(f, img, m), uv, SkyModelParams())
    assert not np.isnan(want).any()
    err = np.abs(got - want).max() / _l1(f)
    assert err < TOL, err
    off = case in ("shift3d", "rot3d")
    assert info["doPC"] == int(off) and info["do3Dmul"] == int(off)


@pytest.mark.parametrize("case", ["point", "shift3d", "gauss"])
def test_exact_kernel_matches_the_dft(case):
    kw = {"point": {}, "gauss": {"gauss": (6.0, 3.0, 25.0)}, "shift3d": {"shift3d": True}}[case]
    f, img, m, uv = field_case(N=96, seed=23, nint=6, **kw)
    got, info, _ = _gpu_model(f, img, m, uv, kernel=GR.KERNEL_EXACT)
    assert info["kernel"] == GR.KERNEL_EXACT
    dft_field = with_pa(f, 90.0 - 25.0) if case == "gauss" else f
    mod, l1 = oracle.model_fp64(uv, dft_sky(dft_field, m), SkyModelParams(op=OP_REPL), exact=False)
    err = float(np.max(np.abs(got - mod) / l1))
    assert err < TOL, err


@pytest.mark.parametrize("op", [OP_SUB, OP_DIV, OP_REPL])
def test_operations_with_flags_and_polarization_rules(op):
    f, img, m, uv = field_case(N=64, seed=24, nstok=4, flag_frac=0.15)
    if op == OP_DIV:
        c = uv.vis_view()
        c[..., 0] += 2.0  # keep the divided data away from zero
    p = SkyModelParams(op=op, stokFactor=-1.0, doFlip=True, numberPoln=4)
    gm = G.build(f, img, m)
    want = G.apply(gm, uv, p)
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m) as gf:
        got = gf.FTGrid(uv, p).vis
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)
    np.testing.assert_array_equal(a[..., 2] > 0, b[..., 2] > 0)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    scale = _l1(f) if op != OP_DIV else 1.0
    assert float(d.max()) / scale < (TOL if op != OP_DIV else 1e-4), float(d.max())
    np.testing.assert_allclose(a[..., 2], b[..., 2], rtol=1e-5, atol=1e-6)


def test_selection_leaves_the_rest_untouched():
    f, img, m, uv = field_case(N=64, seed=25, nchan=40, nif=3)
    p = SkyModelParams(op=OP_SUB, startChannel=3, numberChannel=30, startIF=2, numberIF=2, startPoln=2,
                       numberPoln=1)
    want = G.apply(G.build(f, img, m), uv, p)
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m) as gf:
        got = gf.FTGrid(uv, p).vis
    sel = np.zeros(uv.vis_view().shape[:-1], bool)
    sel[:, 1:3, 2:32, 1] = True
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)
    o = uv.vis_view()
    np.testing.assert_array_equal(a[~sel], o[~sel])
    assert np.abs(a[sel] - b[sel]).max() / _l1(f) < TOL
    np.testing.assert_array_equal(got[:, :uv.nrparm], uv.vis[:, :uv.nrparm])


@pytest.mark.parametrize("kernel", [GR.KERNEL_REFERENCE, GR.KERNEL_EXACT])
def test_points_off_the_plane_are_blanked(kernel):
    """Baselines beyond the plane: the reference zeroes data and weight; near
    its edge, the reference's clamped windows (or the exact kernel's clamped,
    centred ones) are followed."""
    f, img, m, uv = field_case(N=48, seed=26, reach=6.0, nint=8)
    p = SkyModelParams(op=OP_SUB)
    want = G.apply(G.build(f, img, m), uv, p, exact=(kernel == GR.KERNEL_EXACT))
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m, kernel=kernel) as gf:
        got = gf.FTGrid(uv, p).vis
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)
    blank = b[..., 2] == 0
    assert blank.any() and (~blank).any()
    np.testing.assert_array_equal(a[..., 2] == 0, blank)
    np.testing.assert_array_equal(a[blank][..., :2], 0.0)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert float(d.max()) / _l1(f) < 1e-4


def test_device_records_equal_host_records():
    import torch
    f, img, m, uv = field_case(N=64, seed=27)
    p = SkyModelParams(op=OP_SUB)
    gimg = GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY)
    with GR.GridField(f, gimg, m) as gf:
        host = gf.FTGrid(uv, p).vis
        d = torch.from_numpy(uv.vis.copy()).cuda()
        fs = torch.from_numpy(np.ascontiguousarray(uv.fscale)).cuda()
        gf.FTGrid_device(uv, d.data_ptr(), uv.nvis, p, d_fscale=fs.data_ptr(),
                         stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        dev = d.cpu().numpy()
    np.testing.assert_array_equal(host, dev)


def test_grid_info_and_empty_field():
    f, img, m, uv = field_case(N=64, seed=28, ncomp=40)
    f.deltaX = f.deltaX + np.float32(0.3 * f.cdeltX)  # off the cells
    grid, n, gparm, bad = G.grid_comps(f, img)
    gimg = GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY)
    with GR.GridField(f, gimg, m) as gf:
        info = gf.info()
    assert info["ncomp"] == n == 40 and info["bad"] == bad
    assert info["nx"] == 128 and info["ny"] == 128 and info["nxp"] == 64 + 1 + 12
    f.startComp, f.endComp = 10, 5  # nothing selected: records untouched
    with GR.GridField(f, gimg, m) as gf:
        assert gf.info()["ncomp"] == 0
        out = gf.FTGrid(uv, SkyModelParams(op=OP_SUB))
    np.testing.assert_array_equal(out.vis, uv.vis)


def test_larger_field_exact_kernel_against_the_dft():
    """A 512 x 512 image (1024 x 1024 grid), 2000 components, 64 channels:
    sampled records against the DFT oracle."""
    f, img, m, uv = field_case(N=512, ncomp=2000, seed=29, nchan=64, nif=1, nint=3)
    got, _, _ = _gpu_model(f, img, m, uv, kernel=GR.KERNEL_EXACT)
    idx = np.arange(0, uv.nvis, 7)
    sub = uv.rows(0, uv.nvis)
    sub.vis = uv.vis[idx]
    mod, l1 = oracle.model_fp64(sub, dft_sky(f, m), SkyModelParams(op=OP_REPL), exact=False)
    err = float(np.max(np.abs(got[idx] - mod) / l1))
    assert err < TOL, err


def test_mixed_mode_dft_then_grid():
    """OBIT_SkyModel_Mixed through both GPU paths: the DFT of the components
    above minDFT subtracted, then the gridded model of the rest (maxGrid, exact
    kernel); equals subtracting the DFT of the whole field."""
    from helpers import run_gpu
    from obit_b200.comps import CCModel
    f, img, m, uv = field_case(N=96, seed=30, ncomp=200, nint=6)
    cells = {}
    keep = [i for i, (x, y) in enumerate(zip(f.deltaX, f.deltaY)) if cells.setdefault((x, y), i) == i]
    f.flux, f.deltaX, f.deltaY = f.flux[keep], f.deltaX[keep], f.deltaY[keep]
    T = 0.4
    p = SkyModelParams(op=OP_SUB)
    after_dft = run_gpu(uv, dft_sky(f, CCModel(**{**m.__dict__, "minDFT": T})), p, exact=False)
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m, maxGrid=T,
                      kernel=GR.KERNEL_EXACT) as gf:
        assert 0 < gf.info()["ncomp"] < len(f.flux)
        got = gf.FTGrid(after_dft, p).vis
    want = oracle.apply_fp64(uv, dft_sky(f, m), p, exact=False)
    _, l1 = oracle.model_fp64(uv, dft_sky(f, m), p, exact=False)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1])) / l1[..., None]
    assert float(d.max()) < TOL


def _image_of(field, image):
    n = image.nx
    pix = np.zeros((n, n), np.float32)
    ix = np.rint(np.asarray(field.deltaX, np.float64) / field.cdeltX).astype(int) + n // 2
    iy = np.rint(np.asarray(field.deltaY, np.float64) / field.cdeltY).astype(int) + n // 2
    for x, y, fl in zip(ix, iy, np.asarray(field.flux, np.float32)):
        pix[y, x] = np.float32(pix[y, x] + fl)
    return pix


def test_image_model_matches_the_oracle_and_the_components():
    """obit_dft_grid_create_image (ObitSkyModelLoadImage): an image holding the
    components gives the component model's plane; a clipped, blanked, scaled
    image matches the oracle's image model."""
    f, img, m, uv = field_case(N=96, seed=31, nint=6, shift3d=True)
    gimg = GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY)
    pix = _image_of(f, img)
    with GR.GridField(f, gimg, m) as gc, GR.GridField.from_image(pix, -999.0, f, gimg, m) as gi:
        np.testing.assert_array_equal(gi.plane(), gc.plane())
        assert gi.info()["ncomp"] == 96 * 96
    pix[3, 4] = -0.5
    pix[10, 12] = -999.0
    pix[40:44, 50:52] = 0.7
    from obit_b200.comps import CCModel
    m2 = CCModel(**{**m.__dict__, "factor": 0.5, "minFlux": 0.0})
    want_gm = G.build_image(pix, -999.0, f, img, m2)
    p = SkyModelParams(op=OP_SUB)
    want = G.apply(want_gm, uv, p)
    with GR.GridField.from_image(pix, -999.0, f, gimg, m2) as gi:
        got = gi.FTGrid(uv, p).vis
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(uv.vis_view().shape)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert float(d.max()) / want_gm.l1 < TOL


def test_host_records_in_many_chunks():
    """More records than the host path's three 64 MB staging slots hold
    (4,500 records of 2 x 2,048 channels, 221 MB): the chunked pipeline
    reuses its slots and gives the device path's result bit for bit."""
    import torch
    from obit_b200 import uvdata as U
    f, img, m, uv0 = field_case(N=64, seed=32, nchan=1024, nif=2, nint=1)
    rng = np.random.default_rng(5)
    uvw = np.repeat(uv0.vis[:, :3].astype(np.float64), 70, axis=0)[:4500]
    uvw *= rng.uniform(0.5, 1.0, (len(uvw), 1))
    uv = U.make_uvdata(uvw, 2, 1024, 2, uv0.freq, uv0.freqArr, rng)
    p = SkyModelParams(op=OP_SUB)
    gimg = GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY)
    with GR.GridField(f, gimg, m) as gf:
        host = gf.FTGrid(uv, p).vis
        d = torch.from_numpy(uv.vis.copy()).cuda()
        fs = torch.from_numpy(np.ascontiguousarray(uv.fscale)).cuda()
        gf.FTGrid_device(uv, d.data_ptr(), uv.nvis, p, d_fscale=fs.data_ptr(),
                         stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        dev = d.cpu().numpy()
    assert uv.vis.nbytes > 3 * (64 << 20)
    np.testing.assert_array_equal(host, dev)
    assert not np.array_equal(host, uv.vis)


def test_many_rows_per_cell():
    """A CLEAN-like table: 60,000 rows on 1,500 cells (each cell's rows spread
    over the table), a negative row late in the table with noNeg, factor and
    minFlux: the device pass (cells per row, stable sort by cell, row-order
    sums) gives the oracle's grid, so the planes agree."""
    from obit_b200.comps import CCModel
    f, img, m, uv = field_case(N=96, seed=33, ncomp=1500, nint=2)
    rng = np.random.default_rng(9)
    pick = rng.integers(0, 1500, 60000)
    f.flux = rng.uniform(-0.01, 0.2, 60000).astype(np.float32)
    f.flux[:50000] = np.abs(f.flux[:50000])
    f.deltaX, f.deltaY = f.deltaX[pick], f.deltaY[pick]
    m2 = CCModel(**{**m.__dict__, "factor": 0.8, "minFlux": 0.001, "noNeg": True})
    grid, n, gparm, bad = G.grid_comps(f, img, factor=0.8, minFlux=0.001, noNeg=True)
    want = G.ft_plane(grid, gparm, f, img)
    with GR.GridField(f, GR.GridImage(img.nx, img.ny, img.crpixX, img.crpixY), m2) as gf:
        info = gf.info()
        got = gf.plane()
    assert info["ncomp"] == n and info["bad"] == bad and 40000 < n < 60000
    err = np.abs(got.astype(np.complex128) - want).max() / float(np.abs(grid.astype(np.float64)).sum())
    assert err < TOL, err
