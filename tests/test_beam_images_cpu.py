"""CPU checks of the oracle's Jones interpolation from beam images
(oracle_beam_jones): the Lagrange interpolator reproduces pixel values at
pixel centres and polynomials of its degree anywhere; off-grid positions,
blanked windows and gains past the limits give the unit matrix; the parallactic
angle rotates the lookup position."""
import numpy as np

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
