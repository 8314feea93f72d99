"""Beam-corrected DFT (obit_dft_set_beam) on a B200 against the FP64 beam
oracle: random Jones matrices per antenna type, component and Jones plane,
2 or 4 correlations, subtract / replace / divide with flags, every model
family, Stokes I, Q, U and V skies; unit Jones matrices reproduce the plain
sky model; a record whose antennas fall outside the table is reported and
left untouched.  Uniformly spaced channels run the tensor-core form by
default and the FP32 block form under OBIT_DFT_RECUR_CHAIN: both are
checked."""
import numpy as np
import pytest

import oracle
from helpers import TOL_REL, run_gpu
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, GPUSkyModel, SkyModelParams
from test_beam_oracle_cpu import beam_case

pytestmark = pytest.mark.gpu


FORMS = [_lib.OBIT_DFT_RECUR, _lib.OBIT_DFT_RECUR_CHAIN]


def _run_beam(uv, sky, p, beam, torch, jones=None, flavor=None, info=None, xyz=None):
    out = uv.copy()
    d_jones = torch.from_numpy(np.ascontiguousarray(jones if jones is not None else beam.jones)).cuda()
    gm = GPUSkyModel("beam")
    try:
        gm.DFTInit(sky, out, SkyModelParams(**{**p.__dict__, "nVisPIO": uv.nvis}))
        if flavor is not None:
            gm.set_kernel(flavor)
        gm.set_beam(beam, d_jones.data_ptr())
        gm.DFTSetMod(sky)
        if xyz is not None:
            gm.set_positions_fp64(xyz)
        if info is not None:
            info.update(gm.beam_info())
        gm.DFTCalc(out)
        gm.DFTShutdown()
    finally:
        gm.close()
    return out.vis


def _check(uv, got, want, l1, op):
    shape = uv.vis_view().shape
    a = got[:, uv.nrparm:].reshape(shape)
    b = want[:, uv.nrparm:].reshape(shape)
    ncorr = 4 if uv.nstok >= 4 else min(2, uv.nstok)
    model_of = [0, 3, 1, 2]
    assert np.array_equal(a[..., ncorr:, :], uv.vis_view()[..., ncorr:, :])
    assert np.array_equal(a[..., 2], uv.vis_view()[..., 2])  # weights are never changed
    for p_ in range(ncorr):
        L = l1[..., model_of[p_]]
        if op == OP_DIV:
            sel = b[..., p_, 2] > 0
            g = 1.0 / (a[..., p_, 0] + 1j * a[..., p_, 1])
            w = 1.0 / (b[..., p_, 0] + 1j * b[..., p_, 1])
            rel = np.where(sel, np.abs(g - w) / np.maximum(L, 1e-30), 0)
            assert np.nanmax(rel) < 2 * TOL_REL
        else:
            d = np.abs((a[..., p_, 0] - b[..., p_, 0]) + 1j * (a[..., p_, 1] - b[..., p_, 1]))
            assert np.nanmax(d / np.maximum(L, 1e-30)) < TOL_REL + 1e-6


@pytest.mark.parametrize("flavor", FORMS)
@pytest.mark.parametrize("nstok", [2, 4])
@pytest.mark.parametrize("op", [OP_SUB, OP_REPL, OP_DIV])
def test_beam_matches_oracle(op, nstok, flavor):
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=nstok, nrow=70, nchan=24, nif=2, ncomp=150, seed=3 + op,
                              flag_frac=0.1)
    if op == OP_DIV:
        c = uv.vis_view()
        c[..., 0] = 1.0
        c[..., 1] = 0.0
    p = SkyModelParams(op=op)
    info = {}
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor, info=info)
    assert info["form"] == (1 if flavor == _lib.OBIT_DFT_RECUR else 0)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, op)


@pytest.mark.parametrize("flavor", FORMS)
@pytest.mark.parametrize("mt", [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS,
                                U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC])
def test_beam_every_family(mt, flavor):
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(mt=mt, nstok=4, nrow=40, nchan=20, nif=2, ncomp=90, seed=11 + mt)
    p = SkyModelParams(op=OP_SUB)
    info = {}
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor, info=info)
    assert info["form"] == (1 if flavor == _lib.OBIT_DFT_RECUR else 0)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


def test_unit_jones_reproduce_the_sky_model():
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=2, nrow=50, nchan=32, nif=2, ncomp=120, unit=True)
    p = SkyModelParams(op=OP_REPL)
    got = _run_beam(uv, sky, p, beam, torch)
    plain = run_gpu(uv, sky, SkyModelParams(op=OP_REPL)).vis
    _, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)[..., :2, :2]
    b = plain[:, uv.nrparm:].reshape(a.shape[:-1] + (3,))[..., :2]
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))
    assert np.max(d / l1[..., None]) < 2 * TOL_REL


def test_antenna_outside_the_table_is_reported():
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=2, nrow=20, nchan=8, nif=1, ncomp=30)
    uv.vis[5, 3] = 256.0 * 1 + 40  # antenna 40 of 12
    p = SkyModelParams(op=OP_SUB)
    with pytest.raises(_lib.DFTError) as e:
        _run_beam(uv, sky, p, beam, torch)
    assert e.value.code == 4 or "code 3" in str(e.value)


def test_beam_description_is_validated():
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=2, nrow=10, nchan=8, nif=1, ncomp=20)
    d_jones = torch.from_numpy(beam.jones).cuda()
    out = uv.copy()
    gm = GPUSkyModel("beam-bad")
    try:
        gm.DFTInit(sky, out, SkyModelParams(op=OP_SUB, nVisPIO=uv.nvis))
        bad_type = beam.antType.copy()
        bad_type[3] = 7
        from obit_b200.beam import Beam
        for b, msg in ((Beam(bad_type, beam.jchan, beam.jones), "antenna type"),
                       (Beam(beam.antType, beam.jchan + 5, beam.jones), "Jones plane"),
                       (Beam(beam.antType, beam.jchan, beam.jones, stokType=5), "Stokes type")):
            with pytest.raises(_lib.DFTError) as e:
                gm.set_beam(b, d_jones.data_ptr())
            assert msg in str(e.value)
        gm.DFTShutdown()
    finally:
        gm.close()


def test_beam_nonuniform_channels_take_the_direct_form():
    """Irregular channel frequencies: the per-evaluation form (FP64 phase per
    channel) instead of the recurrence, against the same oracle."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=4, nrow=40, nchan=24, nif=2, ncomp=100, seed=19, flag_frac=0.1)
    rng = np.random.default_rng(3)
    uv.freqArr = np.sort(uv.freqArr + rng.uniform(-3e5, 3e5, uv.freqArr.shape))
    p = SkyModelParams(op=OP_SUB)
    got = _run_beam(uv, sky, p, beam, torch)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


@pytest.mark.parametrize("flavor", FORMS)
@pytest.mark.parametrize("stok", [2, 3, 4])
def test_beam_polarized_skies(stok, flavor):
    """Stokes Q, U (with a parallactic angle) and V skies."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=4, nrow=50, nchan=20, nif=2, ncomp=110, seed=23 + stok, flag_frac=0.1,
                              stok=stok, par_ang=0.61)
    p = SkyModelParams(op=OP_SUB)
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


@pytest.mark.parametrize("flavor", FORMS + [_lib.OBIT_DFT_PLAIN])
@pytest.mark.parametrize("mt", [U.MOD_POINT_SPEC, U.MOD_GAUSS_TSPEC])
def test_beam_jones_planes_inside_blocks(flavor, mt):
    """Seven Jones planes over 2 x 27 channels: plane changes fall inside the
    block form's 8-channel blocks and the tensor-core form's 16-channel
    tiles, which the planner cuts there; every form matches the oracle."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(mt=mt, nstok=4, nrow=45, nchan=27, nif=2, ncomp=140, seed=41, njc=7,
                              flag_frac=0.1)
    p = SkyModelParams(op=OP_SUB)
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


def test_beam_selection_and_one_correlation():
    """A channel and IF selection on single-correlation records."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=1, nrow=40, nchan=30, nif=3, ncomp=100, seed=43, njc=4)
    p = SkyModelParams(op=OP_SUB, startChannel=4, numberChannel=19, startIF=2, numberIF=2)
    got = _run_beam(uv, sky, p, beam, torch)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(a.shape)
    src = uv.vis_view()
    mask = np.zeros(a.shape[:-1], bool)
    mask[:, 1:3, 3:22, :] = True
    assert np.array_equal(a[~mask], src[~mask])
    d = np.abs((a[..., 0, 0] - b[..., 0, 0]) + 1j * (a[..., 0, 1] - b[..., 0, 1]))[:, 1:3, 3:22]
    assert np.max(d / np.maximum(l1[:, 1:3, 3:22, 0], 1e-30)) < TOL_REL + 1e-6


@pytest.mark.parametrize("flavor", FORMS)
@pytest.mark.parametrize("stok", [1, 2, 3, 4])
def test_beam_circular_feeds(stok, flavor):
    """Circular feeds (records RR, LL, RL, LR; Jones matrices in the R, L basis),
    Stokes I, Q, U and V skies: the model J1 M J2^H of the CPU path's circular
    branch."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=4, nrow=45, nchan=20, nif=2, ncomp=110, seed=51 + stok, flag_frac=0.1,
                              stok=stok, circular=True)
    p = SkyModelParams(op=OP_SUB)
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor)
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


@pytest.mark.parametrize("mt", [U.MOD_POINT, U.MOD_POINT_SPEC, U.MOD_POINT_TSPEC, U.MOD_GAUSS,
                                U.MOD_GAUSS_SPEC, U.MOD_GAUSS_TSPEC])
@pytest.mark.parametrize("nstok", [1, 2, 4])
def test_beam_tensor_form_long_runs(mt, nstok):
    """The tensor-core form over runs longer than one 256-channel run (300
    channels: a full run and a 44-channel run ending in a partial tile), three
    antenna types, five Jones planes and enough components for several
    64-component tiles with a ragged last one."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(mt=mt, nstok=nstok, nrow=37, nchan=300, nif=2, ncomp=333, seed=61 + mt,
                              ntype=3, njc=5, flag_frac=0.1)
    p = SkyModelParams(op=OP_SUB)
    info = {}
    got = _run_beam(uv, sky, p, beam, torch, info=info)
    assert info["form"] == 1 and info["units"] >= 2 * 2
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


def test_beam_form_choice():
    """Irregular channels and single-channel selections keep the block form."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(nstok=4, nrow=20, nchan=24, nif=2, ncomp=40, seed=71)
    rng = np.random.default_rng(5)
    uv2 = uv.copy()
    uv2.freqArr = np.sort(uv2.freqArr + rng.uniform(-3e5, 3e5, uv2.freqArr.shape))
    info = {}
    _run_beam(uv2, sky, SkyModelParams(op=OP_SUB), beam, torch, info=info)
    assert info["form"] == 0
    info = {}
    _run_beam(uv, sky, SkyModelParams(op=OP_SUB, startChannel=5, numberChannel=1), beam, torch, info=info)
    assert info["form"] == 0
    info = {}
    _run_beam(uv, sky, SkyModelParams(op=OP_SUB), beam, torch, flavor=_lib.OBIT_DFT_PLAIN, info=info)
    assert info["form"] == 2


@pytest.mark.parametrize("mt", [U.MOD_POINT_SPEC, U.MOD_GAUSS])
def test_beam_tensor_form_many_antenna_types(mt):
    """Five antenna types (25 type pairs): the coefficient fragments of every
    pair shrink the tensor-core form's component tile below 64; records
    still match the oracle."""
    torch = pytest.importorskip("torch")
    uv, sky, beam = beam_case(mt=mt, nstok=4, nrow=30, nchan=48, nif=2, ncomp=150, seed=83, ntype=5, njc=3,
                              flag_frac=0.1)
    p = SkyModelParams(op=OP_SUB)
    info = {}
    got = _run_beam(uv, sky, p, beam, torch, info=info)
    assert info["form"] == 1 and 8 <= info["ct"] < 64
    want, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    _check(uv, got, want, l1, OP_SUB)


@pytest.mark.parametrize("flavor", FORMS + [_lib.OBIT_DFT_PLAIN])
def test_beam_fp64_positions(flavor):
    """FP64 component positions (obit_dft_set_mod_d) in the beam path: on the
    22 GHz, 8000 km sample the phases reach ~1e7 rad and the FP32 table moves
    the model far beyond the bound; with the side table every form matches
    the oracle evaluated at the FP64 positions."""
    torch = pytest.importorskip("torch")
    from test_fp64_positions_gpu import _vlbi_sample

    from obit_b200.beam import Beam, baseline_codes
    uv, sky = _vlbi_sample(nrow=24, ncomp=400)
    uv.vis[:, 3] = baseline_codes(12, uv.nvis)
    r = np.random.default_rng(91)
    jones = np.zeros((2, sky.ncomp, 3, 8), np.float32)
    jones[..., 0] = 1.0
    jones[..., 6] = 1.0
    jones += (0.2 * r.standard_normal(jones.shape)).astype(np.float32)
    nfreq = uv.nchan * uv.nif
    beam = Beam(r.integers(0, 2, 12), (np.arange(nfreq) * 3 // nfreq).astype(np.int32), jones)
    p = SkyModelParams(op=OP_REPL)
    want64, l1 = oracle.apply_beam_fp64(uv, sky, p, beam, xyz=sky.xyz)
    want32, _ = oracle.apply_beam_fp64(uv, sky, p, beam)
    shape = uv.vis_view().shape
    a = want32[:, uv.nrparm:].reshape(shape)[..., 0, :]
    b = want64[:, uv.nrparm:].reshape(shape)[..., 0, :]
    dev = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1])) / np.maximum(l1[..., 0], 1e-30)
    assert float(np.nanmax(dev)) > 1e-2  # the FP32 table alone is far from the FP64-position sky
    got = _run_beam(uv, sky, p, beam, torch, flavor=flavor, xyz=sky.xyz)
    _check(uv, got, want64, l1, OP_REPL)
