"""The component loader (obit_dft_load_comps) on CPU: the UVSub golden model
(13 CLEAN components entered twice at Factor 0.5, field 0.5 deg off the phase
centre with a 10 deg map rotation, 3-D image) must give the component table
the reference's geometry gives (tests/golden/make_uvsub_fixture.py restates it
from the reference's FP32/FP64 rounding points), and the merge / selection
rules of ObitTableCCUtilMergeSel and ObitSkyModelLoadComps
(ObitSystem/Obit/src/ObitTableCCUtil.c:1238-1361, ObitSkyModel.c:1682-2121)
hold against an independent numpy statement."""
import math
from pathlib import Path

import numpy as np
import pytest

from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.comps import CCField, CCModel, load_comps

GOLD = Path(__file__).resolve().parent / "golden"


def _uvsub_fields():
    d = np.load(GOLD / "uvsub_fixture.npz")
    cc = d["cc"]
    ra, dec, rot, do3d, xpo, ypo, cdx, cdy = d["im_geom"]
    uvra, uvdec, uvrot = d["uv_geom"]
    f = CCField(cc[:, 0], cc[:, 1], cc[:, 2], ra, dec, rotation=rot, do3D=bool(do3d), xPxOff=xpo,
                yPxOff=ypo, cdeltX=cdx, cdeltY=cdy)
    m = CCModel(uvra, uvdec, uvRotation=uvrot, factor=float(d["cc_factor"]))
    return [f] * int(d["cc_nfield"]), m, d["comps"]


def test_uvsub_model_matches_reference_geometry():
    fields, model, want = _uvsub_fields()
    sky, nrow = load_comps(fields, model)
    assert sky.modType == U.MOD_POINT and nrow == 26 and sky.ncomp == 26
    # the loader orders each field by decreasing |flux|, the fixture keeps table
    # order: compare as sets, bit for bit
    key = lambda a: a[np.lexsort((a[:, 1], -np.abs(a[:, 0])))]
    assert np.array_equal(key(sky.comps), key(want))


def test_uvsub_model_reproduces_master_through_oracle():
    """The loaded table, through the FP64 oracle's divide, reproduces the
    reference's master output at the pinned level."""
    import oracle
    from test_uvsub_golden import PIN_RMS, _fixture, _vis_compare

    uv, _, params, master = _fixture()
    fields, model, _ = _uvsub_fields()
    sky, _ = load_comps(fields, model)
    assert _vis_compare(oracle.apply_fp64(uv, sky, params), master) < PIN_RMS


# ---- merge and selection rules against numpy ----------------------------------


def _np_merge(f, factor=1.0, minflux=0.0, noneg=False, spec=False):
    """Independent statement: rows start..end minus deselected, equal positions
    summed (not for polynomial spectra), decreasing |flux|, selection."""
    n = len(f.flux)
    end = f.endComp if f.endComp > 0 else n
    rows = [i for i in range(max(1, f.startComp) - 1, min(end, n))
            if f.status is None or f.status[i] >= 0]
    groups = {}
    order = []
    for i in sorted(rows, key=lambda i: (f.deltaX[i], f.deltaY[i])):
        k = (float(f.deltaX[i]), float(f.deltaY[i])) if not spec else ("row", i)
        if k not in groups:
            groups[k] = np.float32(0.0)
            order.append(k)
        groups[k] = np.float32(groups[k] + np.float32(f.flux[i]))
    merged = sorted(order, key=lambda k: -abs(float(groups[k])))  # stable
    out = []
    for k in merged:
        fl = groups[k]
        if noneg and fl <= 0:
            break
        if abs(fl) > minflux:
            out.append(np.float32(fl * np.float32(factor)))
    return out


def _rand_field(rng, n, dup=0.3, **kw):
    pos = rng.integers(-20, 20, size=(n, 2)).astype(np.float32) * np.float32(1e-4)
    k = int(dup * n)
    pos[:k] = pos[rng.integers(k, n, size=k)]          # repeated positions
    flux = rng.normal(0.0, 1.0, n).astype(np.float32)
    flux[rng.random(n) < 0.05] = 0.0
    return CCField(flux, pos[:, 0], pos[:, 1], 10.0, 40.0, **kw)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_merge_sort_and_selection(seed):
    rng = np.random.default_rng(seed)
    f = _rand_field(rng, 200, startComp=5, endComp=180,
                    status=np.where(rng.random(200) < 0.1, -1, 1))
    for noneg, minflux in [(False, 0.0), (True, 0.0), (False, 0.5)]:
        m = CCModel(10.0, 40.0, factor=0.5, minFlux=minflux, noNeg=noneg)
        sky, nrow = load_comps([f], m)
        want = _np_merge(f, 0.5, minflux, noneg)
        assert nrow == 176 and sky.ncomp == len(want)
        assert np.array_equal(sky.comps[:, 0], np.array(want, np.float32))


def test_phase_centre_field_positions_are_2pi_offsets():
    """Field at the phase centre, no rotation: X, Y = 2 pi dx, dy (rad), Z = 0."""
    f = CCField(np.array([1.0, 2.0], np.float32), np.array([1e-3, -2e-3], np.float32),
                np.array([5e-4, 0.0], np.float32), 150.0, -30.0)
    sky, _ = load_comps([f], CCModel(150.0, -30.0))
    konst = np.float32(math.pi / 180.0 * 2.0 * math.pi)
    assert np.array_equal(sky.comps[:, 1], np.float32([-2e-3, 1e-3]) * konst)
    assert np.array_equal(sky.comps[:, 2], np.float32([0.0, 5e-4]) * konst)
    assert np.all(sky.comps[:, 3] == 0.0)


def test_gaussian_terms_and_mixed_fields():
    """A Gaussian field takes its FWHM and PA from its first row; a point field
    beside it carries zero Gaussian terms (the table is Gaussian)."""
    n = 4
    pg = np.zeros((n, 4), np.float32)
    pg[:, :4] = [10.0 / 3600, 5.0 / 3600, 30.0, 1.0]
    pg[1:, 0] = 99.0  # only the first row's shape is used
    g = CCField(np.ones(n, np.float32), np.arange(n, dtype=np.float32) * 1e-4, np.zeros(n, np.float32),
                0.0, 0.0, parms=pg)
    p = CCField(np.full(2, 3.0, np.float32), np.zeros(2, np.float32), np.array([1e-4, 2e-4], np.float32),
                0.0, 0.0)
    sky, _ = load_comps([g, p], CCModel(0.0, 0.0))
    assert sky.modType == U.MOD_GAUSS and sky.lcomp == 7 and sky.ncomp == 6
    g1, g2, g3 = U.gauss_coeffs(10.0 / 3600, 5.0 / 3600, 30.0)
    assert np.allclose(sky.comps[:4, 4:7], np.float32([g1, g2, g3]), rtol=1e-6)
    assert np.all(sky.comps[4:, 4:7] == 0.0)


def test_polynomial_spectra_are_not_merged():
    n = 3
    parms = np.zeros((n, 6), np.float32)
    parms[:, 3] = 10.0              # point with spectrum, two terms
    parms[:, 4] = [-0.7, -0.5, 0.2]
    parms[:, 5] = [0.01, 0.02, 0.03]
    f = CCField(np.float32([1.0, 2.0, 0.5]), np.zeros(n, np.float32), np.zeros(n, np.float32), 0.0, 0.0,
                parms=parms)
    sky, _ = load_comps([f], CCModel(0.0, 0.0))
    assert sky.modType == U.MOD_POINT_SPEC and sky.nterm == 2 and sky.ncomp == 3
    assert np.array_equal(sky.comps[:, 0], np.float32([2.0, 1.0, 0.5]))
    assert np.array_equal(sky.comps[:, 4:6], parms[[1, 0, 2], 4:6])


def test_unsupported_geometry_and_types_are_errors():
    f = CCField(np.ones(2, np.float32), np.zeros(2, np.float32), np.zeros(2, np.float32), 1.0, 2.0,
                do3D=False)
    with pytest.raises(_lib.DFTError) as e:
        load_comps([f], CCModel(0.0, 0.0))       # 2-D image away from the phase centre
    assert e.value.code == 3
    parms = np.zeros((2, 4), np.float32)
    parms[:, 3] = 3.0                              # uniform sphere
    g = CCField(np.ones(2, np.float32), np.zeros(2, np.float32), np.zeros(2, np.float32), 0.0, 0.0,
                parms=parms)
    with pytest.raises(_lib.DFTError):
        load_comps([g], CCModel(0.0, 0.0))


def test_fp64_positions_follow_the_table():
    """obit_dft_load_comps_d: the same table, plus X, Y, Z with every step of
    the geometry in FP64 -- at the phase centre exactly 2 pi dx (rad) in
    double; for the UVSub field (0.5 deg off, 10 deg rotation, 3-D) within the
    FP32 table's rounding of it, and not equal to it."""
    f = CCField(np.array([1.0, 2.0], np.float32), np.array([1e-3, -2e-3], np.float32),
                np.array([5e-4, 0.0], np.float32), 150.0, -30.0)
    sky, _ = load_comps([f], CCModel(150.0, -30.0))
    konst = math.pi / 180.0 * 2.0 * math.pi
    assert np.array_equal(sky.xyz[:, 0], np.float32([-2e-3, 1e-3]).astype(np.float64) * konst)
    assert np.array_equal(sky.xyz[:, 1], np.float32([0.0, 5e-4]).astype(np.float64) * konst)
    assert np.all(sky.xyz[:, 2] == 0.0)

    fields, model, _ = _uvsub_fields()
    sky, _ = load_comps(fields, model)
    d = np.abs(sky.xyz - sky.comps[:, 1:4].astype(np.float64))
    assert np.max(d) < 1e-6 * np.max(np.abs(sky.xyz))
    assert np.max(d) > 0.0
