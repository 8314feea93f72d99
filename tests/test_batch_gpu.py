"""Multi-facet batch (obit_dft_batch_*): uneven facets -- different IF and
channel counts, row and component counts, an empty model and a one-row facet --
applied by one graph launch of the persistent batched kernel per model family,
checked facet by facet against the FP64 oracle; the per-facet comparator
launches and the autotuner on the same facets."""
import numpy as np
import pytest

import oracle
from helpers import TOL_REL, small
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.batch import DFTBatch, Facet, _descriptors
from obit_b200.skymodel import OP_DIV, OP_REPL, OP_SUB, SkyModelParams

SPECS = [  # (modType, nrow, nchan, nif, nstok, ncomp, seed, op)
    (U.MOD_POINT_SPEC, 301, 64, 3, 2, 700, 41, OP_SUB),
    (U.MOD_POINT_SPEC, 40, 32, 1, 4, 2500, 42, OP_REPL),
    (U.MOD_POINT_SPEC, 1, 32, 2, 2, 90, 43, OP_SUB),
    (U.MOD_POINT_SPEC, 77, 128, 1, 2, 0, 44, OP_SUB),     # empty model: records untouched
    (U.MOD_POINT_SPEC, 150, 32, 4, 2, 333, 45, OP_DIV),
]


def _facets(specs, torch, kinds=None):
    out, keep = [], []
    for i, (mt, nrow, nchan, nif, nstok, ncomp, seed, op) in enumerate(specs):
        mt = kinds[i] if kinds else mt
        uv, sky = small(mt, nrow=nrow, nchan=nchan, nif=nif, nstok=nstok, ncomp=max(ncomp, 1),
                        seed=seed, flag_frac=0.05)
        if ncomp == 0:
            sky.comps = sky.comps[:0]
        d_vis = torch.from_numpy(uv.vis.copy()).cuda()
        d_comps = torch.from_numpy(np.ascontiguousarray(sky.comps)).cuda() if ncomp else \
            torch.zeros(4, device="cuda")
        keep += [d_vis, d_comps]
        p = SkyModelParams(op=op)
        out.append((uv, sky, p, d_vis, Facet(uv, sky, p, d_vis.data_ptr(), nrow, d_comps.data_ptr())))
    return out, keep


def _check_facet(uv, sky, p, got):
    want = oracle.apply_fp64(uv, sky, p)
    if sky.ncomp == 0:
        assert np.array_equal(got, uv.vis)
        return
    m, l1 = oracle.model_fp64(uv, sky, p)
    a = got[:, uv.nrparm:].reshape(uv.vis_view().shape)
    b = want[:, uv.nrparm:].reshape(a.shape)
    d = np.abs((a[..., 0] - b[..., 0]) + 1j * (a[..., 1] - b[..., 1]))[..., :2]
    if p.op == OP_DIV:
        # Q = V / M: |dQ| / |Q| = |dM| / |M|, so the model error implied by the
        # quotient is |dQ| / |Q| * |M|, bounded like the other operations by
        # the L1 norm of the component terms
        q = np.maximum(np.abs(b[..., 0] + 1j * b[..., 1])[..., :2], 1e-30)
        dm = d / q * np.abs(m)[..., None]
        assert float(np.max(dm / l1[..., None])) < 2 * TOL_REL
        # weights become weight x |M| (input weights are 1 or flagged)
        assert float(np.max(np.abs(a[..., :2, 2] - b[..., :2, 2]) / l1[..., None])) < 2 * TOL_REL
    else:
        # the records are FP32: the result of a subtraction is rounded to the
        # data's precision, which a heavily tapered model's L1 norm may not reach
        ulp = 2.0 ** -22 * np.abs(b[..., 0] + 1j * b[..., 1])[..., :2]
        assert float(np.max((d - ulp) / l1[..., None])) < TOL_REL
    assert np.array_equal(a[..., 2:, :], b[..., 2:, :])  # unselected polarizations


@pytest.mark.gpu
def test_batch_graph_run_matches_oracle_per_facet():
    torch = pytest.importorskip("torch")
    fs, keep = _facets(SPECS, torch)
    b = DFTBatch([f[4] for f in fs])
    try:
        info = b.info()
        assert info["facets"] == 5 and info["launches"] == 1
        assert info["evals"] == sum(uv.nvis * uv.nchan * uv.nif * sky.ncomp for uv, sky, *_ in fs)
        b.run()
        b.check()
        for uv, sky, p, d_vis, _ in fs:
            _check_facet(uv, sky, p, d_vis.cpu().numpy())
    finally:
        b.close()


@pytest.mark.gpu
def test_batch_replays_deterministically_and_mixes_families():
    torch = pytest.importorskip("torch")
    kinds = [U.MOD_POINT, U.MOD_GAUSS_SPEC, U.MOD_POINT, U.MOD_GAUSS_SPEC, U.MOD_POINT_TSPEC]
    specs = [(k, *s[1:7], OP_REPL) for k, s in zip(kinds, SPECS)]
    fs, keep = _facets(specs, torch)
    b = DFTBatch([f[4] for f in fs])
    try:
        assert b.info()["launches"] == 3  # one persistent launch per model family
        b.run()
        first = [d.cpu().numpy() for *_, d, _ in fs]
        b.run()  # graph replay: replace is idempotent, bit for bit
        b.check()
        for (uv, sky, p, d_vis, _), x in zip(fs, first):
            y = d_vis.cpu().numpy()
            assert np.array_equal(x, y)
            _check_facet(uv, sky, p, y)
    finally:
        b.close()


@pytest.mark.gpu
def test_batch_per_facet_comparators_match_oracle():
    torch = pytest.importorskip("torch")
    for flavor in (_lib.OBIT_DFT_RECUR, _lib.OBIT_DFT_PLAIN):
        fs, keep = _facets(SPECS, torch)
        b = DFTBatch([f[4] for f in fs])
        try:
            b.run_per_facet(flavor)
            b.check()
            for uv, sky, p, d_vis, _ in fs:
                _check_facet(uv, sky, p, d_vis.cpu().numpy())
        finally:
            b.close()


@pytest.mark.gpu
def test_plans_of_one_kernel_with_different_tiles_interleave():
    """Facets 0 and 4 plan the same kernel with different shared-memory tiles
    (R x Bt = 128 x 2 and 64 x 4); repeated per-facet runs alternate between
    them, so each launch must still be allowed its own tile."""
    torch = pytest.importorskip("torch")
    specs = [(*s[:7], OP_REPL) for s in SPECS]
    fs, keep = _facets(specs, torch)
    b = DFTBatch([f[4] for f in fs])
    try:
        for _ in range(3):
            b.run_per_facet(_lib.OBIT_DFT_RECUR)
        b.run()
        b.run_per_facet(_lib.OBIT_DFT_RECUR)
        b.check()
        for uv, sky, p, d_vis, _ in fs:
            _check_facet(uv, sky, p, d_vis.cpu().numpy())
    finally:
        b.close()


@pytest.mark.gpu
def test_autotune_leaves_records_alone_and_keeps_parity():
    torch = pytest.importorskip("torch")
    fs, keep = _facets(SPECS, torch)
    b = DFTBatch([f[4] for f in fs])
    try:
        before = [d.clone() for *_, d, _ in fs]
        best = b.autotune()
        assert best["tried"] >= 4 and best["K"] in (16, 32) and best["threads"] in (128, 256)
        for x, (*_, d, _) in zip(before, fs):
            assert torch.equal(x, d)
        info = b.info()
        assert (info["K"], info["ct"], info["Bt"]) == (best["K"], best["ct"], best["Bt"])
        b.run()
        b.check()
        for uv, sky, p, d_vis, _ in fs:
            _check_facet(uv, sky, p, d_vis.cpu().numpy())
    finally:
        b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [(16, 32, 4, 128), (32, 64, 8, 256), (32, 32, 32, 256)])
def test_batch_explicit_tiles(tile):
    torch = pytest.importorskip("torch")
    fs, keep = _facets(SPECS, torch)
    b = DFTBatch([f[4] for f in fs])
    try:
        b.set_tile(*tile)
        i = b.info()
        # the component tile may shrink to fit shared memory; the rest is as set
        assert (i["K"], i["Bt"], i["threads"]) == (tile[0], tile[2], tile[3])
        assert 8 <= i["ct"] <= tile[1] and i["R"] == tile[3] // tile[2]
        b.run()
        b.check()
        for uv, sky, p, d_vis, _ in fs:
            _check_facet(uv, sky, p, d_vis.cpu().numpy())
    finally:
        b.close()


def test_facet_descriptors_follow_the_selection():
    """Host side only: the descriptors a facet turns into."""
    uv, sky = small(U.MOD_POINT_SPEC, nrow=3, nchan=16, nif=3, nstok=4, ncomp=5, seed=1)
    p = SkyModelParams(op=OP_DIV, startChannel=3, numberChannel=8, startIF=2, numberIF=2,
                       startPoln=2, numberPoln=1, stokFactor=-1.0, doFlip=True)
    keep = []
    fd = _descriptors(Facet(uv, sky, p, 0x1000, 3, 0x2000), keep)
    vi, mi = fd.visInfo.contents, fd.modelInfo.contents
    assert (vi.chanb, vi.chane, vi.IFb, vi.IFe, vi.stokb, vi.stoke) == (2, 9, 1, 2, 1, 1)
    assert (vi.incs, vi.incf, vi.incif) == (1, 4, 64) and vi.lenvis == uv.lrec
    assert (mi.type, mi.opType, mi.nmodel[0], mi.size) == (1, OP_DIV, 5, sky.lcomp)
    assert fd.cpuRules == 1 and fd.stokFactor == -1.0 and fd.doFlip == 1
    assert fd.freqArr[5] == uv.freqArr[5] and fd.d_vis == 0x1000 and fd.nvis == 3


@pytest.mark.gpu
def test_streamed_batch_over_host_records():
    """obit_dft_batch_run_host: the facets' records in pinned host memory,
    streamed through a small staging area (about a dozen waves, facets split
    across waves), mixed model families; every facet against the FP64 oracle,
    the device copies untouched, and a replay of the captured graph on fresh
    copies of the records bit-identical."""
    torch = pytest.importorskip("torch")
    kinds = [U.MOD_POINT_SPEC, U.MOD_POINT, U.MOD_GAUSS_SPEC, U.MOD_POINT_SPEC, U.MOD_POINT]
    fac, keep = _facets(SPECS, torch, kinds)
    hosts = [torch.from_numpy(uv.vis.copy()).pin_memory() for uv, *_ in fac]
    b = DFTBatch([f for *_, f in fac])
    try:
        stream = torch.cuda.Stream()
        staging = 2 * 50 * max(uv.lrec for uv, *_ in fac) * 4
        info = b.run_host([h.data_ptr() for h in hosts], staging, stream.cuda_stream)
        torch.cuda.synchronize()
        b.check()
        assert info["waves"] >= 8
        assert info["h2d_bytes"] == sum(uv.vis.nbytes for uv, *_ in fac)
        first = [h.numpy().copy() for h in hosts]
        for (uv, sky, p, d_vis, _), got in zip(fac, first):
            _check_facet(uv, sky, p, got)
            assert np.array_equal(d_vis.cpu().numpy(), uv.vis)  # device records untouched
        for (uv, *_), h in zip(fac, hosts):  # fresh inputs, same buffers: the graph replays
            h.numpy()[:] = uv.vis
        info2 = b.run_host([h.data_ptr() for h in hosts], staging, stream.cuda_stream)
        torch.cuda.synchronize()
        b.check()
        assert info2 == info
        for h, g in zip(hosts, first):
            assert np.array_equal(h.numpy(), g)
        with pytest.raises(_lib.DFTError):  # smaller than two records of the widest facet
            b.run_host([h.data_ptr() for h in hosts], 1024, stream.cuda_stream)
    finally:
        b.close()
