"""CPU tests of the multi-frequency component loader (obit_dft_load_comps_mf,
the restatement of ObitSkyModelMFLoadComps with its spectral-index fit).

The reference fits each component's plane fluxes with GSL's lmder (MINPACK
Levenberg-Marquardt; GSL is not in this image), so the fit is checked against
SciPy's MINPACK Levenberg-Marquardt on the same weighted least squares, within
the reference's convergence test (1e-5); the surrounding control flow (the
constant model first, the 1.5 x chi^2 acceptance, the [-2, 2] sanity range) and
the table layout against values computed here from the inputs."""
import numpy as np
import pytest

from obit_b200 import _lib
from obit_b200.comps import CCField, CCModel, MFModel, load_comps, load_comps_mf

FREQS = np.array([1.0e9, 1.2e9, 1.45e9, 1.7e9, 2.0e9])


def _field(n, rng, gauss=False, alpha=None, noise=0.0, dup=0):
    x = rng.uniform(-0.3, 0.3, n)
    y = rng.uniform(-0.3, 0.3, n)
    s0 = np.exp(rng.uniform(np.log(0.01), np.log(2.0), n))
    a = rng.uniform(-1.5, 1.5, n) if alpha is None else np.full(n, alpha)
    planes = s0[:, None] * (FREQS[None, :] / FREQS[0]) ** a[:, None]
    planes = planes * (1.0 + noise * rng.standard_normal(planes.shape))
    flux = planes.mean(axis=1)
    typ = 21 if gauss else 20
    parms = np.zeros((n, 4 + len(FREQS)), np.float32)
    parms[:, 0:3] = (20.0 / 3600, 12.0 / 3600, 35.0) if gauss else 0.0
    parms[:, 3] = typ
    parms[:, 4:] = planes
    if dup:  # repeat the first rows at the same positions (merged, planes summed)
        idx = np.arange(dup)
        x, y, flux = np.r_[x, x[idx]], np.r_[y, y[idx]], np.r_[flux, flux[idx]]
        parms = np.r_[parms, parms[idx]]
    return CCField(flux=flux, deltaX=x, deltaY=y, crvalRA=150.0, crvalDec=30.0, parms=parms), a


def _model(**kw):
    return CCModel(uvRA=150.0, uvDec=30.0, **kw)


def test_exact_power_laws_are_recovered():
    rng = np.random.default_rng(1)
    f, a = _field(200, rng)
    sky, nrow = load_comps_mf([f], _model(), MFModel(FREQS))
    assert sky.modType == 20 and sky.lcomp == 5 + len(FREQS) and sky.ncomp == 200
    # rows are sorted by decreasing |flux|: match by plane fluxes
    order = np.argsort(-np.abs(np.asarray(f.flux, np.float32)), kind="stable")
    fitted = sky.comps[:, 4]
    planes = sky.comps[:, 5:]
    assert np.array_equal(planes, f.parms[order, 4:])
    assert np.max(np.abs(fitted - np.where(np.abs(a[order]) <= 2, a[order], 0))) < 1e-4


def test_fit_matches_minpack_levenberg_marquardt():
    """Noisy spectra: the fitted index against scipy's MINPACK LM on the same
    data, sigma and start (the weighted mean flux, index 0)."""
    scipy_opt = pytest.importorskip("scipy.optimize")
    rng = np.random.default_rng(2)
    f, _ = _field(150, rng, noise=0.05)
    sky, _ = load_comps_mf([f], _model(), MFModel(FREQS))
    L = np.log(FREQS / FREQS[0]).astype(np.float32).astype(np.float64)
    checked = 0
    for row in sky.comps:
        obs = row[5:].astype(np.float64)
        avg = float(np.float32(obs.mean()))
        res = scipy_opt.least_squares(lambda p: (p[0] * np.exp(p[1] * L) - obs) / 1e-4, x0=[avg, 0.0],
                                      method="lm", xtol=1e-12, ftol=1e-15, gtol=1e-15)
        chi_const = np.sum(((obs - obs.mean()) / 1e-4) ** 2) / (len(obs) - 1)
        chi_fit = np.sum(res.fun ** 2) / (len(obs) - 2)
        want = res.x[1] if chi_fit < 1.5 * chi_const else 0.0
        want = want if -2 <= want <= 2 else 0.0
        assert abs(row[4] - want) < 1e-4 * max(1.0, abs(want)), (row[4], want)
        checked += want != 0.0
    assert checked > 100


def test_merge_sums_planes_and_geometry_matches_the_base_loader():
    rng = np.random.default_rng(3)
    f, _ = _field(60, rng, dup=10)
    sky, _ = load_comps_mf([f], _model(factor=0.5), MFModel(FREQS))
    assert sky.ncomp == 60  # 10 duplicates merged
    # positions as the base loader places them (same field, point type)
    g = CCField(flux=f.flux, deltaX=f.deltaX, deltaY=f.deltaY, crvalRA=f.crvalRA, crvalDec=f.crvalDec)
    base, _ = load_comps([g], _model(factor=0.5))
    assert np.array_equal(sky.comps[:, :4], base.comps[:, :4])
    # a merged row carries the summed planes times factor
    k = int(np.argmax(np.isclose(sky.comps[:, 0], 0.5 * 2 * np.float32(f.flux[0]), rtol=1e-6)))
    assert np.allclose(sky.comps[k, 5:], 0.5 * 2 * f.parms[0, 4:], rtol=1e-6)


def test_gaussian_tabulated_layout_and_prior_alpha():
    rng = np.random.default_rng(4)
    f, _ = _field(40, rng, gauss=True)
    mf = MFModel(FREQS, doAlphaCorr=True, priorAlpha=-0.7, priorAlphaRefF=1.4e9)
    sky, _ = load_comps_mf([f], _model(), mf)
    assert sky.modType == 21 and sky.lcomp == 8 + len(FREQS)
    g = CCField(flux=f.flux, deltaX=f.deltaX, deltaY=f.deltaY, crvalRA=f.crvalRA, crvalDec=f.crvalDec,
                parms=np.c_[f.parms[:, :3], np.ones(len(f.flux))])
    base, _ = load_comps([g], _model())
    assert np.array_equal(sky.comps[:, 4:7], base.comps[:, 4:7])  # Gaussian terms
    corr = (FREQS / 1.4e9) ** -0.7
    order = np.argsort(-np.abs(np.asarray(f.flux, np.float32)), kind="stable")
    assert np.allclose(sky.comps[:, 8:], f.parms[order, 4:] * corr[None, :], rtol=1e-6)


def test_no_fit_cases():
    rng = np.random.default_rng(5)
    f, _ = _field(30, rng)
    sky, _ = load_comps_mf([f], _model(), MFModel(FREQS, noSIfit=True))  # polarized data
    assert np.all(sky.comps[:, 4] == 0.0)
    sky, _ = load_comps_mf([f], _model(), MFModel(FREQS[:1]))  # one plane
    assert np.all(sky.comps[:, 4] == 0.0)
    steep, _ = _field(10, rng, alpha=-3.0)  # outside the sanity range
    sky, _ = load_comps_mf([steep], _model(), MFModel(FREQS))
    assert np.all(sky.comps[:, 4] == 0.0)


def test_rejections():
    rng = np.random.default_rng(6)
    f, _ = _field(5, rng)
    g, _ = _field(5, rng, gauss=True)
    with pytest.raises(_lib.DFTError) as e:
        load_comps_mf([f, g], _model(), MFModel(FREQS))
    assert e.value.code == 3
    short = CCField(flux=f.flux, deltaX=f.deltaX, deltaY=f.deltaY, crvalRA=150.0, crvalDec=30.0,
                    parms=f.parms[:, :6])
    with pytest.raises(_lib.DFTError):
        load_comps_mf([short], _model(), MFModel(FREQS))
