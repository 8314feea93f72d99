"""CPU checks of the oracle's Jones interpolation from beam images
(oracle_beam_jones): the Lagrange interpolator reproduces pixel values at
pixel centres and polynomials of its degree anywhere; off-grid positions,
blanked windows and gains past the limits give the unit matrix; the parallactic
angle rotates the lookup position."""
import numpy as np
import pytest

import oracle
from obit_b200.beam import BeamImages

FBLANK = -3.0e38


def images(ntype=2, n=21, nplane=2, projection=0, refsize=0.0, fn=None):
    y, x = np.mgrid[1:n + 1, 1:n + 1].astype(np.float64)
    px = np.zeros((ntype, 8, nplane, n, n), np.float32)
    for t in range(ntype):
        for q in range(8):
            for k in range(nplane):
                px[t, q, k] = fn(x, y, t, q, k) if fn else (0.9 if q in (0, 2) else 0.05) + 0.001 * (q + t + k)
    return BeamImages(px, np.array([1.4e9, 1.5e9][:nplane]), crval=(0.0, 0.0), crpix=((n + 1) / 2, (n + 1) / 2),
                      cdelt=(0.1, 0.1), projection=projection, hwidth=2, fblank=FBLANK, refSizeFact=refsize)


def test_pixel_centres_and_polynomials():
    # a cubic in x and y is reproduced exactly by 5-tap Lagrange interpolation
    f = lambda x, y, t, q, k: (0.5 + 0.01 * x - 0.0003 * x * x + 0.00001 * y ** 3 + 0.001 * q)  # noqa: E731
    im = images(fn=f)
    pos = np.array([[0.0, 0.0], [0.1, -0.2], [0.237, 0.311], [-0.55, 0.42]], np.float32)
    J = oracle.beam_jones_fp64(im, pos, 0.0)
    for c, (x, y) in enumerate(pos.astype(np.float64)):
        pxl, pyl = x / 0.1 + 11.0, y / 0.1 + 11.0
        want = {q: f(pxl, pyl, 0, q, 0) for q in range(8)}
        assert abs(J[0, c, 0, 0] - want[0]) < 1e-5 and abs(J[0, c, 0, 6] - want[2]) < 1e-5
        assert abs(J[0, c, 0, 2] - want[4]) < 1e-5 and abs(J[0, c, 0, 5] - want[7]) < 1e-5


def test_off_grid_blank_and_limits_give_unit():
    im = images()
    im.pixels[1, 3, 0, 8:14, 8:14] = FBLANK  # blank P2 im of type 1 about the centre
    pos = np.array([[5.0, 0.0], [0.0, 0.0]], np.float32)  # off the grid; on the blank
    J = oracle.beam_jones_fp64(im, pos, 0.0)
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    assert np.array_equal(J[0, 0, 0], unit) and np.array_equal(J[1, 0, 1], unit)
    assert np.array_equal(J[1, 1, 0], unit)      # blanked window
    assert not np.array_equal(J[0, 1, 0], unit)  # the other type is fine
    # a parallel hand above 1.3 after the gain factor
    big = images(fn=lambda x, y, t, q, k: 1.5 if q == 0 else 0.1)
    assert np.array_equal(oracle.beam_jones_fp64(big, pos[1:], 0.0)[0, 0, 0], unit)


def test_parallactic_angle_rotates_the_lookup():
    f = lambda x, y, t, q, k: 0.5 + 0.02 * x + 0.0 * y  # noqa: E731
    im = images(fn=f)
    pos = np.array([[0.3, 0.0]], np.float32)
    a = oracle.beam_jones_fp64(im, pos, 0.0)[0, 0, 0, 0]
    b = oracle.beam_jones_fp64(im, pos, np.pi / 2)[0, 0, 0, 0]
    # rotated by 90 deg the offset lies along the grid's y axis: x pixel at the centre
    assert abs(a - f(14.0, 11.0, 0, 0, 0)) < 1e-6 and abs(b - f(11.0, 11.0, 0, 0, 0)) < 1e-6


def test_primary_beam_factor():
    im = images(refsize=2.0e-10)  # arg = 2e-10 x freq x offset
    pos = np.array([[0.3, 0.4]], np.float32)  # 0.5 deg
    J = oracle.beam_jones_fp64(im, pos, 0.0)
    arg = 2.0e-10 * 1.4e9 * 0.5
    g = (1 - 4 * arg * arg) / np.cos(np.pi * arg)
    assert abs(J[0, 0, 0, 0] - g * 0.9) < 1e-5


def _lookup_pixel(im, pos, par=0.0):
    """Pixel (1-relative) the oracle looks up for each position: P1 re and im
    of the images are 0.001 x and 0.001 y, which the interpolator reproduces."""
    J = oracle.beam_jones_fp64(im, np.asarray(pos, np.float32), par)
    return J[0, :, 0, 0] / 0.001, J[0, :, 0, 1] / 0.001


def _ramp_images(projection, crval, cdelt=(0.01, 0.01), n=201, crota=0.0):
    f = lambda x, y, t, q, k: 0.001 * x if q == 0 else (0.001 * y if q == 1 else 0.0)  # noqa: E731
    im = images(ntype=1, n=n, nplane=1, projection=projection, fn=f)
    im.crval, im.cdelt, im.crota = crval, cdelt, crota
    return im


def test_projections_known_answers():
    """Known answers of each projection (CUDASkyGeom.h:91-250) for a position
    theta north of the reference and one east of it: -SIN sin(theta),
    -TAN tan(theta), -ARC theta, -STG 2 tan(theta / 2), -NCP and -GLS their
    defining formulas; -MER and -AIT are scaled so that one increment of
    declination (and of right ascension, -AIT) at the reference is one pixel."""
    d2r = 1.745329252e-2
    ra0, dec0, th = 30.0, 40.0, 0.6  # theta in deg
    cen = 101.0
    radial = {1: np.sin, 2: np.tan, 3: lambda a: a, 8: lambda a: 2 * np.tan(a / 2)}
    for proj, R in radial.items():
        im = _ramp_images(proj, (ra0, dec0))
        px, py = _lookup_pixel(im, [[ra0, dec0 + th]])
        assert abs(px[0] - cen) < 2e-3
        assert abs(py[0] - (cen + R(th * d2r) / d2r / 0.01)) < 2e-3, proj
    # -NCP: (cos d0 - cos d cos da) / sin d0 north, sin(da) cos d east
    im = _ramp_images(4, (ra0, dec0))
    da, dec = 0.5, 40.3
    px, py = _lookup_pixel(im, [[ra0 + da, dec]])
    d, d0, a = dec * d2r, dec0 * d2r, da * d2r
    assert abs(px[0] - (cen + np.sin(a) * np.cos(d) / d2r / 0.01)) < 2e-3
    assert abs(py[0] - (cen + (np.cos(d0) - np.cos(d) * np.cos(a)) / np.sin(d0) / d2r / 0.01)) < 2e-3
    # -GLS: da cos(dec) east, dec - dec0 north
    im = _ramp_images(5, (ra0, dec0))
    px, py = _lookup_pixel(im, [[ra0 + da, dec]])
    assert abs(px[0] - (cen + da * np.cos(d) / 0.01)) < 2e-3
    assert abs(py[0] - (cen + 0.3 / 0.01)) < 2e-3
    # -MER and -AIT: one increment north (and east for -AIT) is one pixel
    for proj in (6, 7):
        im = _ramp_images(proj, (ra0, dec0), cdelt=(0.02, 0.02))
        px, py = _lookup_pixel(im, [[ra0, dec0], [ra0, dec0 + 0.02], [ra0, dec0 + 0.2]])
        assert abs(px[0] - cen) < 2e-3 and abs(py[0] - cen) < 2e-3
        assert abs(py[1] - (cen + 1)) < 2e-3, proj
        assert 9.5 < py[2] - cen < 10.5
    im = _ramp_images(7, (ra0, dec0), cdelt=(0.02, 0.02))
    px, py = _lookup_pixel(im, [[ra0 + 0.02, dec0]])
    assert abs(px[0] - (cen + 1)) < 2e-3


def test_projections_limits_give_unit():
    """Positions a projection cannot place give the unit matrix: -SIN past 90
    degrees from the reference, -TAN at 90 degrees, -NCP about an equatorial
    reference; all projections agree with the linear offsets near the
    reference on the equator."""
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    for proj, crval, pos in ((1, (0.0, 0.0), [0.0, 91.0]), (2, (0.0, 0.0), [90.0, 0.0]), (4, (10.0, 0.0), [10.0, 0.1])):
        im = _ramp_images(proj, crval, cdelt=(1.0, 1.0))
        J = oracle.beam_jones_fp64(im, np.array([pos], np.float32), 0.0)
        np.testing.assert_array_equal(J[0, 0, 0], unit)
    for proj in range(9):
        if proj == 4:
            continue
        im = _ramp_images(proj, (0.0, 0.0))
        px, py = _lookup_pixel(im, [[0.05, -0.03]])
        assert abs(px[0] - 106.0) < 2e-3 and abs(py[0] - 98.0) < 2e-3, proj


CTYPES = ["RA---LIN", "RA---SIN", "RA---TAN", "RA---ARC", "RA---NCP", "RA---GLS", "RA---MER", "RA---AIT",
          "RA---STG"]


@pytest.mark.skipif(not oracle.have_refgeom(), reason="oracle/_ref not built")
@pytest.mark.parametrize("projection", range(9))
def test_projections_match_the_reference_geometry(projection):
    """The oracle's lookup pixel against the reference's own CUDAPositionXYpix
    (CUDASkyGeom.h, compiled for the host by oracle/refgeom.cpp) at random
    positions about three reference positions, with a parallactic angle and a
    rotated grid; positions the reference cannot project give the unit
    matrix."""
    r = np.random.default_rng(600 + projection)
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    for crval in ((0.0, 0.0), (123.0, -35.0), (300.0, 71.0)):
        im = _ramp_images(projection, crval, cdelt=(0.02, 0.025), crota=12.0)
        crpix = tuple(float(c) for c in im.crpix)
        pos = (r.uniform(-1.5, 1.5, (64, 2)) + np.array(crval)).astype(np.float32)
        par = float(r.uniform(-1, 1))
        J = oracle.beam_jones_fp64(im, pos, par)
        for c in range(pos.shape[0]):
            (rx, ry), rc = oracle.ref_position_xypix(pos[c].astype(np.float64), CTYPES[projection], crval, crpix,
                                                   im.cdelt, (0.0, im.crota), par)
            if rc != 0 or not (1.0 <= rx <= 201.0 and 1.0 <= ry <= 201.0):
                np.testing.assert_array_equal(J[0, c, 0], unit)
                continue
            assert abs(J[0, c, 0, 0] / 0.001 - rx) < 1e-4 and abs(J[0, c, 0, 1] / 0.001 - ry) < 1e-4, (crval, c)


@pytest.mark.skipif(not oracle.have_refgeom(), reason="oracle/_ref not built")
@pytest.mark.parametrize("hwidth", [1, 2, 3, 4])
def test_interpolation_matches_the_reference(hwidth):
    """The oracle's Jones entries against the reference's own
    CUDABeamInterpPixel (CUDABeamInterp.h, compiled for the host by
    oracle/refgeom.cpp) at the reference's own pixel of each position, for
    smooth images with blanked patches, on a -SIN grid with a parallactic
    angle; where the reference blanks any of the 8 images the oracle gives
    the unit matrix (the reference lets blanks through the cross terms)."""
    r = np.random.default_rng(900 + hwidth)
    n, nplane = 31, 2
    y, x = np.mgrid[0:n, 0:n].astype(np.float64) / n
    px = np.zeros((1, 8, nplane, n, n), np.float32)
    for q in range(8):
        for k in range(nplane):
            a, b, c = r.uniform(-1, 1, 3)
            px[0, q, k] = (0.9 if q in (0, 2) else 0.05) + 0.05 * (a * x + b * y * y + c * np.sin(3 * x * y))
    for _ in range(3):
        i0, j0 = r.integers(0, n - 4, 2)
        q = int(r.integers(0, 8))
        px[0, q, :, i0:i0 + 3, j0:j0 + 3] = FBLANK
    im = BeamImages(px, np.array([1.4e9, 1.5e9]), crval=(10.0, 20.0), crpix=(16.0, 16.0), cdelt=(0.05, 0.05),
                    projection=1, hwidth=hwidth, fblank=FBLANK, refSizeFact=0.0)
    pos = (r.uniform(-0.8, 0.8, (300, 2)) + np.array(im.crval)).astype(np.float32)
    par = 0.3
    J = oracle.beam_jones_fp64(im, pos, par)
    unit = np.array([1, 0, 0, 0, 0, 0, 1, 0], np.float32)
    order = [0, 1, 4, 5, 6, 7, 2, 3]  # Jones XX, XY, YX, YY (re, im) from P1, X1, X2, P2
    compared = blanked = 0
    for c in range(pos.shape[0]):
        (rx, ry), rc = oracle.ref_position_xypix(pos[c].astype(np.float64), "RA---SIN", im.crval, im.crpix,
                                               im.cdelt, (0.0, 0.0), par)
        if rc != 0 or not (1.0 <= rx <= n and 1.0 <= ry <= n):
            np.testing.assert_array_equal(J[0, c, 0], unit)
            continue
        for k in range(nplane):
            v = [oracle.ref_beam_interp_pixel(px[0, q], FBLANK, hwidth, (rx, ry, k + 1)) for q in range(8)]
            if any(val == float(np.float32(FBLANK)) for val in v):
                np.testing.assert_array_equal(J[0, c, k], unit)
                blanked += 1
                continue
            np.testing.assert_allclose(J[0, c, k], [v[q] for q in order], atol=2e-6)
            compared += 1
    assert compared > 300 and blanked > 0
