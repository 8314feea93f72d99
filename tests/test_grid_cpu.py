"""CPU checks of the gridded model FT: the oracle's restatement of the
reference's gridded path (ObitSkyModelGridFTComps / ThreadSkyModelFTGrid)
pinned against the DFT oracle on fields where both apply, the reference's
interpolation-kernel table, the mode choice of ObitSkyModelChose, and the
host-side argument checks of obit_dft_grid_create (no GPU call is reached).

Pins.  With Lagrange weights at the requested point the gridded model equals
the DFT to |dV| / sum|A| < 1e-5 (2-D field, 3-D field off the phase centre with
re-projection and field-offset phase, circular Gaussians); the reference's own
table puts the point 0.005 cell low (plus 0.0025 tabulation), bounded by
cell_bound; and the reference's taper of an elliptical Gaussian of position
angle t is the DFT's Gaussian of position angle 90 - t (the two paths of the
reference differ by that reflection)."""
import ctypes as C

import numpy as np
import pytest

import oracle
import oracle_grid as G
from grid_helpers import cell_bound, dft_sky, field_case, with_pa
from obit_b200 import _lib
from obit_b200 import grid as GR
from obit_b200.skymodel import OP_REPL, SkyModelParams

TOL = 1e-5


def _dft_err(field, image, model, uv, exact, dft_field=None):
    sky = dft_sky(dft_field or field, model)
    gm = G.build(field, image, model)
    val = G.model_values(gm, uv, SkyModelParams(), exact=exact)
    mod, l1 = oracle.model_fp64(uv, sky, SkyModelParams(op=OP_REPL), exact=False)
    assert not np.isnan(val).any()
    return float(np.nanmax(np.abs(val - mod) / l1)), gm


def test_exact_kernel_equals_the_dft():
    f, img, m, uv = field_case()
    e, gm = _dft_err(f, img, m, uv, exact=True)
    assert not gm.geom.doPC and not gm.geom.do3Dmul
    assert e < TOL, e


def test_reference_kernel_within_its_bound():
    f, img, m, uv = field_case(seed=4)
    e, _ = _dft_err(f, img, m, uv, exact=False)
    b = cell_bound(f, img)
    assert 1e-4 < e < b + TOL, (e, b)


def test_shifted_3d_field_equals_the_dft():
    f, img, m, uv = field_case(seed=5, shift3d=True)
    e, gm = _dft_err(f, img, m, uv, exact=True)
    assert gm.geom.doPC and gm.geom.do3Dmul
    assert e < TOL, e


def test_circular_gaussian_equals_the_dft():
    f, img, m, uv = field_case(seed=6, gauss=(6.0, 6.0, 30.0))
    e, _ = _dft_err(f, img, m, uv, exact=True)
    assert e < TOL, e


@pytest.mark.parametrize("pa", [30.0, 70.0, -20.0])
def test_elliptical_gaussian_is_the_dfts_at_90_minus_pa(pa):
    f, img, m, uv = field_case(seed=7, gauss=(6.0, 3.0, pa))
    e, _ = _dft_err(f, img, m, uv, exact=True, dft_field=with_pa(f, 90.0 - pa))
    assert e < TOL, e
    e_same, _ = _dft_err(f, img, m, uv, exact=True)
    assert e_same > 100 * TOL  # the same angle in both paths does not agree


def test_kernel_table_rows():
    """Rows sum to one; row 100 (offset 0 in SetConvKernal) interpolates a
    linear ramp at 0.995 past the centre tap, the reference's offset."""
    t = G.kernel_table()
    assert t.shape == (201, 25)
    assert np.allclose(t.astype(np.float64).sum(1), 1.0, atol=2e-6)
    ramp = np.arange(25, dtype=np.float64)
    assert abs(t[100].astype(np.float64) @ ramp - 12.995) < 1e-5
    assert abs(t[0].astype(np.float64) @ ramp - 12.495) < 1e-5
    assert abs(t[200].astype(np.float64) @ ramp - 13.495) < 1e-5


def test_conjugate_columns():
    f, img, m, uv = field_case(N=48, seed=8)
    grid, n, gparm, _ = G.grid_comps(f, img)
    P = G.ft_plane(grid, gparm, f, img)
    ny = P.shape[0]
    H = G.HWIDTH
    for r in (1, 5, ny // 2, ny - 1):
        for c in range(H):
            assert P[r, c] == np.conj(P[ny - r, H + (H - c)])
    for c in range(H):
        assert P[0, c] == np.conj(P[0, H + (2 * H - c)])


def test_grid_comps_selection():
    """factor, minFlux, maxGrid, noNeg and the row range, as ObitTableCCUtilGrid."""
    f, img, m, uv = field_case(N=48, ncomp=60, seed=9, neg_frac=0.3)
    g0, n0, _, _ = G.grid_comps(f, img)
    assert n0 == 60
    f.startComp, f.endComp = 5, 40
    g1, n1, _, _ = G.grid_comps(f, img, factor=2.0, minFlux=0.05, maxGrid=1.5)
    fl = np.asarray(f.flux[4:40], np.float64) * 2.0
    assert n1 == int(np.sum((np.abs(fl) >= 0.05) & (np.abs(fl) <= 1.5)))
    g2, n2, _, _ = G.grid_comps(f, img, noNeg=True)
    first_neg = int(np.argmax(np.asarray(f.flux[4:40]) < 0))
    assert n2 == first_neg
    assert abs(float(g1.astype(np.float64).sum()) - float(fl[(np.abs(fl) >= 0.05) & (np.abs(fl) <= 1.5)].sum())) < 1e-4


@pytest.mark.parametrize("nvis", [1000, 100000])
def test_choose_mode_matches_the_oracle(nvis):
    _lib.load()
    for ncc in (1, 30, 300, 3000, 30000):
        for n in (512, 2048, 4096):
            for nchan in (1, 64):
                for mtype in (0, 1, 2):
                    a = GR.choose_mode(0, mtype, [ncc, ncc // 2], [n, n], [n, n], nvis, nchan)
                    b = G.choose_mode(0, mtype, [ncc, ncc // 2], [n, n], [n, n], nvis, nchan)
                    assert a == b, (ncc, n, nchan, mtype)
    assert GR.choose_mode(2, 0, [5], [64], [64], 10, 1) == 2
    assert GR.choose_mode(1, 1, [5], [64], [64], 10, 1) == 1


def _create_rc(field, image, model):
    from obit_b200.comps import _field_array, _model
    lib = _lib.load()
    keep = []
    arr = _field_array([field], keep)
    im = _lib.ObitDFTGridImage(image.nx, image.ny, image.crpixX, image.crpixY)
    h = C.c_void_p()
    rc = lib.obit_dft_grid_create(arr, C.byref(im), C.byref(_model(model)), 1e20, 0, None, C.byref(h))
    return rc, lib.obit_dft_last_error().decode()


def test_create_rejects_unsupported_fields_on_the_host():
    f, img, m, uv = field_case(N=48, ncomp=20, seed=10, gauss=(6.0, 3.0, 10.0))
    f.parms[3, 0] = 7.0 / 3600
    rc, msg = _create_rc(f, img, m)
    assert rc == 1 and "same size" in msg
    f.parms[:, 0] = 6.0 / 3600
    f.parms[:, 3] = 4.0  # exponential disk
    rc, msg = _create_rc(f, img, m)
    assert rc == 3 and "disk" in msg
    f2, img2, m2, _ = field_case(N=48, ncomp=20, seed=11)
    f2.xShift = 0.01
    rc, msg = _create_rc(f2, img2, m2)
    assert rc == 3 and "2-D" in msg
    f2.xShift = 0.0
    f2.ncp = True
    rc, msg = _create_rc(f2, img2, m2)
    assert rc == 3 and "NCP" in msg
    rc, msg = _create_rc(f2, G.GridImage(16, 16, 9, 9), m2)
    assert rc == 1 and "smaller" in msg


@pytest.mark.parametrize("op", [0, 1, 2])
def test_c_restatement_matches_the_numpy_oracle(op):
    """refcpu_grid.c (single precision, the CPU baseline) against the numpy
    oracle on the same plane: windows and table rows agree, sums within FP32."""
    f, img, m, uv = field_case(N=48, seed=12, shift3d=(op == 1), nstok=4, flag_frac=0.1)
    if op == 1:
        uv.vis_view()[..., 0] += 2.0
    p = SkyModelParams(op=op, stokFactor=-1.0, doFlip=(op == 2), numberPoln=4)
    gm = G.build(f, img, m)
    a = G.apply_c(gm, uv, p, nthreads=3)
    b = G.apply(gm, uv, p)
    va = a[:, uv.nrparm:].reshape(uv.vis_view().shape)
    vb = b[:, uv.nrparm:].reshape(uv.vis_view().shape)
    np.testing.assert_array_equal(va[..., 2] == 0, vb[..., 2] == 0)
    scale = 1.0 if op == 1 else _l1(f)
    assert np.abs(va[..., :2] - vb[..., :2]).max() / scale < (1e-4 if op == 1 else 2e-6)


def _l1(field):
    return float(np.abs(np.asarray(field.flux, np.float64)).sum())


def test_vis_info_of_a_selection():
    f, img, m, uv = field_case(N=48, ncomp=10, seed=13, nchan=40, nif=3, nstok=4)
    p = SkyModelParams(startChannel=3, numberChannel=30, startIF=2, numberIF=2, startPoln=2, numberPoln=3)
    vi, fs = GR.vis_info(uv, p)
    assert (vi.chanb, vi.chane, vi.IFb, vi.IFe, vi.stokb, vi.stoke) == (2, 31, 1, 2, 1, 3)
    assert (vi.incs, vi.incf, vi.incif) == (1, 4, 160) and vi.lenvis == uv.lrec
    assert vi.freqScale == fs.ctypes.data and fs.dtype == np.float32


def test_rotated_3d_field_equals_the_dft():
    """A 3-D field off the phase centre with an image rotation and a uv
    rotation: re-projection, rotated field offset and phase."""
    f, img, m, uv = field_case(seed=14, shift3d=True, rotation=12.0, uv_rotation=-5.0)
    e, gm = _dft_err(f, img, m, uv, exact=True)
    assert gm.geom.do3Dmul and gm.geom.doPC
    assert e < TOL, e


def test_rotation_without_reprojection_equals_the_dft():
    """A 3-D field image with a rotation while the sky model is 2-D (no
    re-projection): u, v rotated by uv minus map rotation."""
    f, img, m, uv = field_case(seed=15, shift3d=True, rotation=10.0)
    m.do3D = False
    gm = G.build(f, img, m)
    assert gm.geom.doRot and not gm.geom.do3Dmul and gm.geom.doPC
    # the DFT loader re-projects 3-D fields regardless of the model's flag, so
    # compare with the oracle's own C restatement instead
    a = G.apply_c(gm, uv, SkyModelParams(op=2))
    b = G.apply(gm, uv, SkyModelParams(op=2))
    va = a[:, uv.nrparm:].reshape(uv.vis_view().shape)
    vb = b[:, uv.nrparm:].reshape(uv.vis_view().shape)
    assert np.abs(va[..., :2] - vb[..., :2]).max() / _l1(f) < 2e-6


def test_non_square_image():
    """nx != ny: the taper's rows use nx / 2 as the reference's loop does;
    point fields equal the DFT."""
    f, img, m, uv = field_case(N=64, Ny=48, seed=16)
    e, _ = _dft_err(f, img, m, uv, exact=True)
    assert e < TOL, e


def test_mixed_mode_partition():
    """OBIT_SkyModel_Mixed: the DFT takes the merged components above minDFT
    (ObitSkyModel.c:1861, 1959) and the grid the rows at or below maxGrid
    (:4421); with both at one threshold and distinct positions the two models
    partition the field, and together equal the DFT of all (exact kernel)."""
    from obit_b200.comps import CCModel
    f, img, m, uv = field_case(seed=17, ncomp=120)
    # distinct cells, so that merging cannot move flux across the threshold
    cells = {}
    keep = [i for i, (x, y) in enumerate(zip(f.deltaX, f.deltaY)) if cells.setdefault((x, y), i) == i]
    f.flux, f.deltaX, f.deltaY = f.flux[keep], f.deltaX[keep], f.deltaY[keep]
    T = 0.4
    mdft = CCModel(**{**m.__dict__, "minDFT": T})
    part_dft, _ = oracle.model_fp64(uv, dft_sky(f, mdft), SkyModelParams(op=OP_REPL), exact=False)
    gm = G.build(f, img, m, maxGrid=T)
    part_grid = G.model_values(gm, uv, SkyModelParams(), exact=True)
    full, l1 = oracle.model_fp64(uv, dft_sky(f, m), SkyModelParams(op=OP_REPL), exact=False)
    n_dft = int(np.sum(np.abs(f.flux) > T))
    assert 0 < n_dft < len(f.flux) and gm.ncomp == len(f.flux) - n_dft
    assert float(np.max(np.abs(part_dft + part_grid - full) / l1)) < TOL


def _image_of(field, image):
    """The image whose pixels hold the field's components (row-order sums)."""
    n = image.nx
    pix = np.zeros((n, n), np.float32)
    ix = np.rint(np.asarray(field.deltaX, np.float64) / field.cdeltX).astype(int) + n // 2
    iy = np.rint(np.asarray(field.deltaY, np.float64) / field.cdeltY).astype(int) + n // 2
    for x, y, fl in zip(ix, iy, np.asarray(field.flux, np.float32)):
        pix[y, x] = np.float32(pix[y, x] + fl)
    return pix


def test_image_model_grid_equals_the_component_grid():
    """An image holding the components on their pixels grids to the same
    cells as the components (ObitSkyModelLoadImage vs ObitTableCCUtilGrid)."""
    f, img, m, uv = field_case(seed=18)
    pix = _image_of(f, img)
    gi = G.grid_image(pix, -12345.0)
    gc, _, _, _ = G.grid_comps(f, img)
    np.testing.assert_array_equal(gi, gc)


def test_image_model_clip_blank_and_factor():
    f, img, m, uv = field_case(N=48, seed=19)
    pix = _image_of(f, img)
    pix[5, 7] = -0.3   # below minFlux: zero
    pix[9, 11] = -999.0  # blank
    g = G.grid_image(pix, -999.0, factor=2.0, minFlux=0.0)
    n = 48
    off = n - n // 2
    assert g[off + 5, off + 7] == 0.0 and g[off + 9, off + 11] == 0.0
    keep = (pix >= 0.0) & (pix != -999.0)
    np.testing.assert_array_equal(g[off:off + n, off:off + n][keep], (np.float32(2.0) * pix)[keep])


def test_choose_mode_measured_crossover():
    """With the B200 rates the DFT stays the cheaper mode up to about
    dftRate / gridRate components (1,300), far above the reference's
    time model's crossover (a few components for such data)."""
    _lib.load()
    nvis, nchan = 2_000_000, 1024
    assert GR.choose_mode(0, 0, [50], [4096], [4096], nvis, nchan) == 2
    assert GR.choose_mode_measured(0, [50], [4096], [4096], nvis, nchan) == 1
    assert GR.choose_mode_measured(0, [1000], [4096], [4096], nvis, nchan) == 1
    assert GR.choose_mode_measured(0, [2000], [4096], [4096], nvis, nchan) == 2
    # little data: the grid's set-up dominates and the DFT is cheaper even for many components
    assert GR.choose_mode_measured(0, [20000], [4096], [4096], 1000, 1) == 1
    assert GR.choose_mode_measured(1, [5], [64], [64], 10, 1) == 2
    assert GR.choose_mode_measured(2, [5000], [64], [64], 10 ** 6, 64) == 1
    assert GR.choose_mode_measured(0, [2000], [4096], [4096], nvis, nchan, dft_rate=1e14) == 1
