"""The beam-corrected DFT oracle (oracle/oracle_beam.c) on CPU: with unit Jones
matrices a Stokes I sky is the plain DFT oracle on XX and YY and zero on XY and
YX; with random Jones matrices every Stokes matches an independent numpy
statement of cudaJonesCor1_Lin_{I,Q,U,V} (ObitSystem/Obit/include/CUDALinCorSum.h:104-455)
applied per baseline, antenna type and Jones plane."""
import numpy as np
import pytest

import oracle
from helpers import small
from obit_b200 import uvdata as U
from obit_b200.beam import Beam, baseline_codes
from obit_b200.skymodel import OP_REPL, OP_SUB, SkyModelParams


def beam_case(mt=U.MOD_POINT_SPEC, nstok=4, nrow=30, nchan=12, nif=2, ncomp=25, seed=5, unit=False,
              ntype=2, njc=3, flag_frac=0.0, stok=1, par_ang=0.0, circular=False):
    uv, sky = small(mt, nrow=nrow, nchan=nchan, nif=nif, nstok=nstok, ncomp=ncomp, seed=seed,
                    flag_frac=flag_frac)
    uv.vis[:, 3] = baseline_codes(12, uv.nvis)
    r = np.random.default_rng(seed + 100)
    jones = np.zeros((ntype, sky.ncomp, njc, 8), np.float32)
    jones[..., 0] = 1.0  # XX
    jones[..., 6] = 1.0  # YY
    if not unit:
        jones += (0.2 * r.standard_normal(jones.shape)).astype(np.float32)
    ant_type = r.integers(0, ntype, 12)
    jchan = (np.arange(nchan * nif) * njc // (nchan * nif)).astype(np.int32)
    return uv, sky, Beam(ant_type, jchan, jones, stokType=stok, parAng=par_ang, circular=circular)


def np_beam_model(uv, sky, beam):
    """complex (nvis, nif, nchan, 4) model in XX, XY, YX, YY order."""
    m_rows = []
    c = sky.comps.astype(np.float64)
    fs = (uv.freqArr / uv.freq).reshape(uv.nif, uv.nchan)
    for r in range(uv.nvis):
        code = float(uv.vis[r, 3])
        a1 = int(code / 256.0 + 0.001)
        a2 = int(code - a1 * 256.0 + 0.001)
        t1, t2 = beam.antType[a1 - 1], beam.antType[a2 - 1]
        out = np.zeros((uv.nif, uv.nchan, 4), np.complex128)
        for i in range(uv.nif):
            for ch in range(uv.nchan):
                f = fs[i, ch]
                u, v, w = (uv.vis[r, :3].astype(np.float64) * f)
                nu = uv.freqArr.reshape(uv.nif, uv.nchan)[i, ch]
                amp = c[:, 0] * np.exp(c[:, 4] * np.log(nu / sky.refFreq)) if sky.modType == U.MOD_POINT_SPEC \
                    else c[:, 0]
                vv = amp * np.exp(1j * (c[:, 1] * u + c[:, 2] * v + c[:, 3] * w))
                jc = beam.jchan[i * uv.nchan + ch]
                J1 = beam.jones[t1, :sky.ncomp, jc].astype(np.float64)
                J2 = beam.jones[t2, :sky.ncomp, jc].astype(np.float64)
                j1 = J1[:, 0::2] + 1j * J1[:, 1::2]
                j2 = J2[:, 0::2] + 1j * J2[:, 1::2]
                P = lambda a, b: j1[:, a] * np.conj(j2[:, b])
                c2, s2 = (float(np.float32(np.cos(2 * beam.parAng))), float(np.float32(np.sin(2 * beam.parAng))))
                D = [P(0, 0) - P(1, 1), P(0, 2) - P(1, 3), P(2, 0) - P(3, 1), P(2, 2) - P(3, 3)]
                S = [P(1, 0) + P(0, 1), P(1, 2) + P(0, 3), P(3, 0) + P(2, 1), P(3, 2) + P(2, 3)]
                if beam.circular:
                    # J1 M J2^H per component, M the sky's matrix in the R, L basis
                    M = {1: [[1, 0], [0, 1]], 2: [[0, 1], [1, 0]], 3: [[0, 1j], [-1j, 0]],
                         4: [[1, 0], [0, -1]]}[beam.stokType]
                    m1 = j1.reshape(-1, 2, 2)
                    m2 = j2.reshape(-1, 2, 2)
                    prod = m1 @ np.asarray(M, np.complex128) @ np.conj(np.transpose(m2, (0, 2, 1)))
                    C = [prod[:, 0, 0], prod[:, 0, 1], prod[:, 1, 0], prod[:, 1, 1]]
                elif beam.stokType == 1:
                    C = [P(0, 0) + P(1, 1), P(1, 3) + P(0, 2), P(2, 0) + P(3, 1), P(2, 2) + P(3, 3)]
                elif beam.stokType == 2:
                    C = [c2 * D[q] - s2 * S[q] for q in range(4)]
                elif beam.stokType == 3:
                    C = [c2 * S[q] + s2 * D[q] for q in range(4)]
                else:
                    C = [1j * (P(0, 1) - P(1, 3)), 1j * (P(0, 3) - P(1, 2)), 1j * (P(2, 1) - P(3, 0)),
                         1j * (P(2, 3) - P(3, 2))]
                out[i, ch] = [np.sum(vv * Cq) for Cq in C]
        m_rows.append(out)
    return np.array(m_rows)


def test_unit_jones_is_the_plain_dft():
    uv, sky, beam = beam_case(unit=True)
    p = SkyModelParams(op=OP_REPL)
    got, l1 = oracle.apply_beam_fp64(uv, sky, p, beam)
    m, dl1 = oracle.model_fp64(uv, sky, SkyModelParams(op=OP_REPL, numberPoln=2))
    v = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    # record XX, YY = the DFT; XY, YX = 0
    for p_ in (0, 1):
        g = v[..., p_, 0] + 1j * v[..., p_, 1]
        assert np.max(np.abs(g - m) / dl1) < 1e-6
    assert np.all(v[..., 2:, :2] == 0.0)
    assert np.allclose(l1[..., 0], dl1) and np.allclose(l1[..., 3], dl1) and np.all(l1[..., 1] == 0)


@pytest.mark.parametrize("circular", [False, True])
@pytest.mark.parametrize("nstok,stok", [(2, 1), (4, 1), (4, 2), (4, 3), (4, 4)])
def test_random_jones_match_numpy(nstok, stok, circular):
    uv, sky, beam = beam_case(nstok=nstok, nrow=12, nchan=6, ncomp=9, stok=stok, par_ang=0.7,
                              circular=circular)
    got, l1 = oracle.apply_beam_fp64(uv, sky, SkyModelParams(op=OP_REPL), beam)
    want = np_beam_model(uv, sky, beam)
    v = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    rec_of_model = [0, 2, 3, 1]  # record position of model XX, XY, YX, YY
    for q in range(4):
        p_ = rec_of_model[q]
        if p_ >= v.shape[3] or (nstok < 4 and p_ >= 2):
            continue
        g = v[..., p_, 0] + 1j * v[..., p_, 1]
        assert np.max(np.abs(g - want[..., q]) / l1[..., q]) < 1e-6


def test_subtract_leaves_flagged_correlations():
    uv, sky, beam = beam_case(flag_frac=0.3)
    got, _ = oracle.apply_beam_fp64(uv, sky, SkyModelParams(op=OP_SUB), beam)
    src = uv.vis_view()
    v = got[:, uv.nrparm:].reshape(src.shape)
    flagged = src[..., 2] <= 0
    assert flagged.any() and np.array_equal(v[flagged], src[flagged])
    assert not np.array_equal(v[~flagged], src[~flagged])


@pytest.mark.skipif(not oracle.have_refjones(), reason="oracle/_ref not built")
@pytest.mark.parametrize("stok", [1, 2, 3, 4])
def test_coefficients_match_the_reference_code(stok):
    """The oracle's coefficients times the component term equal the sums of the
    reference's own cudaJonesCor1_Lin_{I,Q,U,V}, compiled for the host from its
    header (oracle/refjones.cpp), for random Jones pairs and parallactic angles."""
    r = np.random.default_rng(40 + stok)
    for _ in range(50):
        J1 = r.standard_normal(8).astype(np.float32)
        J2 = r.standard_normal(8).astype(np.float32)
        flux, ph, pa = float(r.uniform(0.1, 2.0)), float(r.uniform(-np.pi, np.pi)), float(r.uniform(0, np.pi))
        c2p, s2p = float(np.float32(np.cos(2 * pa))), float(np.float32(np.sin(2 * pa)))
        s, c = float(np.float32(np.sin(ph))), float(np.float32(np.cos(ph)))
        want = oracle.ref_jones_cor1(stok, flux, s, c, J1, J2, c2p, s2p)
        got = oracle.beam_coeffs(stok, c2p, s2p, J1, J2) * (flux * (c + 1j * s))
        scale = flux * np.abs(J1).sum() * np.abs(J2).sum()
        assert np.max(np.abs(got - want)) < 1e-6 * scale
