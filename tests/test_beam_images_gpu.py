"""Jones matrices interpolated from beam images on the GPU
(obit_dft_beam_jones) against the FP64 oracle of the same interpolation, then
the beam-corrected DFT fed with them against the FP64 beam oracle fed with the
oracle's table: smooth beams with blanked patches, components on and off the
grid, a parallactic angle, linear grids and the eight projections, linear and
circular feeds."""
import numpy as np
import pytest

import oracle
from helpers import TOL_REL
from obit_b200 import uvdata as U
from obit_b200.beam import Beam, BeamImages, jones_from_images
from obit_b200.skymodel import OP_SUB, GPUSkyModel, SkyModelParams
from test_beam_oracle_cpu import beam_case

pytestmark = pytest.mark.gpu
FBLANK = -3.0e38


def _images(ntype, nplane, n=61, projection=0, seed=3):
    """Smooth parallel hands near 1 tapering outwards, small smooth cross
    terms and imaginary parts, a blanked patch per type."""
    r = np.random.default_rng(seed)
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    x = (x - n // 2) / (n // 2)
    y = (y - n // 2) / (n // 2)
    px = np.zeros((ntype, 8, nplane, n, n), np.float32)
    for t in range(ntype):
        for k in range(nplane):
            for q in range(8):
                a, b, c = r.uniform(-1, 1, 3)
                base = 0.95 * np.exp(-0.3 * (x * x + y * y)) if q in (0, 2) else 0.05
                px[t, q, k] = base + 0.02 * (a * x + b * y + c * x * y)
        i0, j0 = r.integers(5, n - 12, 2)
        px[t, :, :, i0:i0 + 6, j0:j0 + 6] = FBLANK
    return BeamImages(px, np.linspace(1.2e9, 1.6e9, nplane), crval=(0.0, 0.0), crpix=(n // 2 + 1, n // 2 + 1),
                      cdelt=(0.05, 0.05), projection=projection, hwidth=2, fblank=FBLANK, refSizeFact=3.0e-10)


@pytest.mark.parametrize("projection", range(9))
@pytest.mark.parametrize("crval", [(0.0, 0.0), (30.0, 40.0)])
def test_jones_from_images_match_the_oracle(projection, crval):
    torch = pytest.importorskip("torch")
    im = _images(2, 3, projection=projection)
    im.crval = crval
    im.crota = 10.0  # enters the -MER and -AIT scales
    if crval != (0.0, 0.0):
        im.refSizeFact = 0.0  # positions far from the pointing centre: no primary-beam factor
    r = np.random.default_rng(7)
    # some off the +-1.5 deg grid
    pos = (r.uniform(-1.8, 1.8, (500, 2)) + np.array(crval)).astype(np.float32)
    par = 0.37
    d_px = torch.from_numpy(im.pixels).cuda()
    d_pos = torch.from_numpy(pos).cuda()
    d_j = torch.zeros((2, 500, 3, 8), dtype=torch.float32, device="cuda")
    jones_from_images(im, d_px.data_ptr(), d_pos.data_ptr(), 500, par, d_j.data_ptr())
    torch.cuda.synchronize()
    got = d_j.cpu().numpy()
    want = oracle.beam_jones_fp64(im, pos, par)
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    is_unit = np.all(want == unit, axis=-1)
    if projection == 4 and crval[1] == 0.0:  # -NCP cannot place anything about the equator
        assert is_unit.all()
    else:
        assert is_unit.any() and (~is_unit).sum() > 1000
    assert np.array_equal(np.all(got == unit, axis=-1), is_unit)
    assert np.max(np.abs(got - want)) < 2e-5


@pytest.mark.parametrize("circular", [False, True])
def test_beam_dft_from_images(circular):
    """The whole path: images -> Jones (GPU) -> beam-corrected DFT (GPU); the
    Jones table against the interpolation oracle, the records against the
    beam oracle."""
    torch = pytest.importorskip("torch")
    uv, sky, beam0 = beam_case(nstok=4, nrow=40, nchan=24, nif=2, ncomp=140, seed=61, njc=3, flag_frac=0.1,
                               circular=circular)
    im = _images(2, 3, seed=5)
    # beam-image offsets of the components (deg), from their direction cosines
    xyz = sky.xyz
    l = xyz[:, 0] / (2 * np.pi)
    m = xyz[:, 1] / (2 * np.pi)
    pos = np.stack([np.degrees(l), np.degrees(m)], axis=1).astype(np.float32)
    d_px = torch.from_numpy(im.pixels).cuda()
    d_pos = torch.from_numpy(pos).cuda()
    d_j = torch.zeros((2, sky.ncomp, 3, 8), dtype=torch.float32, device="cuda")
    jones_from_images(im, d_px.data_ptr(), d_pos.data_ptr(), sky.ncomp, 0.21, d_j.data_ptr())
    torch.cuda.synchronize()
    got_j = d_j.cpu().numpy()
    want_j = oracle.beam_jones_fp64(im, pos, 0.21)
    assert np.max(np.abs(got_j - want_j)) < 2e-5
    # the DFT stage against the beam oracle on the same table (the tables
    # themselves were compared just above)
    beam = Beam(beam0.antType, beam0.jchan, got_j, circular=circular)
    out = uv.copy()
    gm = GPUSkyModel("beam-images")
    try:
        gm.DFTInit(sky, out, SkyModelParams(op=OP_SUB, nVisPIO=uv.nvis))
        gm.set_beam(beam, d_j.data_ptr())
        gm.DFTSetMod(sky)
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    want, l1 = oracle.apply_beam_fp64(uv, sky, SkyModelParams(op=OP_SUB), beam)
    a = out.vis[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(a.shape)
    model_of = [0, 3, 1, 2]
    for p_ in range(4):
        d = np.abs((a[..., p_, 0] - b[..., p_, 0]) + 1j * (a[..., p_, 1] - b[..., p_, 1]))
        assert np.nanmax(d / np.maximum(l1[..., model_of[p_]], 1e-30)) < TOL_REL + 1e-6


@pytest.mark.parametrize("seed", range(12))
def test_random_images(seed):
    """Seeded random grids: antenna types, planes, image size, projection,
    interpolation half-width, cell, parallactic angle and component positions
    (some off the grid)."""
    torch = pytest.importorskip("torch")
    r = np.random.default_rng(13000 + seed)
    ntype, nplane = int(r.integers(1, 4)), int(r.integers(1, 5))
    n = int(r.choice([21, 40, 61]))
    im = _images(ntype, nplane, n=n, projection=int(r.integers(0, 9)), seed=int(r.integers(0, 10 ** 6)))
    if seed % 2:  # a grid about a sky position, no primary-beam factor
        im.crval = (float(r.uniform(0, 360)), float(r.uniform(-80, 80)))
        im.refSizeFact = 0.0
    im.crota = float(r.uniform(-30, 30))
    im.hwidth = int(r.integers(1, 5))
    im.cdelt = (float(r.uniform(0.02, 0.08)), float(r.uniform(0.02, 0.08)))
    ncomp = int(r.integers(1, 400))
    half = 0.5 * n * max(im.cdelt)
    pos = (r.uniform(-1.2 * half, 1.2 * half, (ncomp, 2)) + np.array(im.crval)).astype(np.float32)
    par = float(r.uniform(-1.5, 1.5))
    d_px = torch.from_numpy(im.pixels).cuda()
    d_pos = torch.from_numpy(pos).cuda()
    d_j = torch.zeros((ntype, ncomp, nplane, 8), dtype=torch.float32, device="cuda")
    jones_from_images(im, d_px.data_ptr(), d_pos.data_ptr(), ncomp, par, d_j.data_ptr())
    torch.cuda.synchronize()
    got = d_j.cpu().numpy()
    want = oracle.beam_jones_fp64(im, pos, par)
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    np.testing.assert_array_equal(np.all(got == unit, axis=-1), np.all(want == unit, axis=-1))
    assert np.max(np.abs(got - want)) < 2e-5


def test_types_on_different_grids_one_call_per_type():
    """Antenna types whose beam images lie on different grids: one call per
    type into its slice of the table equals the oracle per type, and on a
    shared grid equals the single call over all types."""
    torch = pytest.importorskip("torch")
    ntype, nplane, ncomp = 3, 2, 257
    im = _images(ntype, nplane, projection=1)
    r = np.random.default_rng(21)
    pos = r.uniform(-1.6, 1.6, (ncomp, 2)).astype(np.float32)
    par = -0.41
    d_pos = torch.from_numpy(pos).cuda()
    d_all = torch.zeros((ntype, ncomp, nplane, 8), dtype=torch.float32, device="cuda")
    jones_from_images(im, torch.from_numpy(im.pixels).cuda().data_ptr(), d_pos.data_ptr(), ncomp, par,
                      d_all.data_ptr())
    d_per = torch.zeros_like(d_all)
    keep = []
    for t in range(ntype):
        sub = BeamImages(np.ascontiguousarray(im.pixels[t:t + 1]), im.planeFreq, crval=im.crval, crpix=im.crpix,
                         cdelt=(0.05 + 0.01 * t, 0.05 - 0.005 * t), projection=t, hwidth=t + 1, fblank=FBLANK,
                         refSizeFact=im.refSizeFact)
        d_px = torch.from_numpy(sub.pixels).cuda()
        keep.append((sub, d_px))
        jones_from_images(sub, d_px.data_ptr(), d_pos.data_ptr(), ncomp, par, d_per[t].data_ptr())
    d_same = torch.zeros_like(d_all)
    for t in range(ntype):
        sub = BeamImages(np.ascontiguousarray(im.pixels[t:t + 1]), im.planeFreq, crval=im.crval, crpix=im.crpix,
                         cdelt=im.cdelt, projection=im.projection, hwidth=im.hwidth, fblank=FBLANK,
                         refSizeFact=im.refSizeFact)
        d_px = torch.from_numpy(sub.pixels).cuda()
        keep.append((sub, d_px))
        jones_from_images(sub, d_px.data_ptr(), d_pos.data_ptr(), ncomp, par, d_same[t].data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_same.cpu().numpy(), d_all.cpu().numpy())
    got = d_per.cpu().numpy()
    for t, (sub, _) in enumerate(keep[:ntype]):
        want = oracle.beam_jones_fp64(sub, pos, par)[0]
        assert np.max(np.abs(got[t] - want)) < 2e-5
