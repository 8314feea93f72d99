"""CPU tests of the host-side planner (channel blocks, log-frequency fits, tile
shape) through tests/planner_harness.cpp compiled against dft_planner.cpp."""
import json
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "obit_b200" / "csrc"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = tmp_path_factory.mktemp("planner") / "planner_harness"
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{CSRC}", f"-I{ROOT / 'include'}", f"-I{cuda_inc}",
                    str(ROOT / "tests" / "planner_harness.cpp"), str(CSRC / "dft_planner.cpp"),
                    "-o", str(exe)], check=True)
    return exe


def plan(exe, *, nchan=64, nif=2, nstok=2, chanb=0, chane=None, ifb=0, ife=None, kind=0, nterm=0,
         lcomp=4, nspec=0, flavor=0, K=0, ct=64, Bt=0, threads=256, fscale=None, lnspec=None,
         specIndex=None, compIndex=None, ngauss=0):
    nrparm = 5
    chane = nchan - 1 if chane is None else chane
    ife = nif - 1 if ife is None else ife
    nfreq = nchan * nif
    if fscale is None:
        f = 1.4e9 + (np.arange(nfreq) % nchan) * 1e6 + (np.arange(nfreq) // nchan) * 100e6
        fscale = f / 1.4e9
    lnspec = np.zeros(nfreq) if lnspec is None else lnspec
    specIndex = np.zeros(nfreq, int) if specIndex is None else specIndex
    incs, incf, incif = 3, 3 * nstok, 3 * nstok * nchan
    lrec = nrparm + 3 * nstok * nchan * nif
    lines = [f"{lrec} {nrparm} {nchan} {nif} {nstok} {incs} {incf} {incif} 1 {nchan}",
             f"{chanb} {chane} {ifb} {ife} 0 {min(2, nstok) - 1}",
             f"{kind} {nterm} {lcomp} 1000 {nspec}",
             f"{flavor} {K} {ct} {Bt} {threads}",
             str(nfreq), " ".join(repr(float(x)) for x in fscale),
             " ".join(repr(float(x)) for x in lnspec), " ".join(str(int(x)) for x in specIndex)]
    if compIndex is not None:
        lines += [str(len(compIndex)), " ".join(repr(float(x)) for x in compIndex), str(ngauss)]
    out = subprocess.run([str(exe)], input="\n".join(lines), capture_output=True, text=True,
                         check=True).stdout
    return json.loads(out)


def covered(p, nchan, nif, nstok=2, nrparm=5):
    """(ichan, iIF) pairs covered by the blocks, from their record offsets."""
    seen = []
    for b in p["blocks"]:
        off = b["off0"] - nrparm
        iif, rem = divmod(off, 3 * nstok * nchan)
        ch = rem // (3 * nstok)
        seen += [(ch + k, iif) for k in range(b["len"])]
    return seen


def test_blocks_cover_selection_once(harness):
    p = plan(harness, nchan=70, nif=3, chanb=3, chane=60, ifb=1, ife=2)
    assert p["rc"] == 0
    seen = covered(p, 70, 3)
    want = [(c, i) for i in (1, 2) for c in range(3, 61)]
    assert sorted(seen) == sorted(want)
    assert len(seen) == len(set(seen))
    assert all(b["len"] <= p["K"] for b in p["blocks"])


def test_default_channels_per_thread(harness):
    assert plan(harness, nchan=256, nif=4)["K"] == 32
    assert plan(harness, nchan=256, nif=4, kind=3, lcomp=7)["K"] == 32   # Gaussian
    assert plan(harness, nchan=256, nif=4, kind=1, nterm=2, lcomp=6)["K"] == 16  # 2 spectral terms
    assert plan(harness, nchan=5, nif=1)["K"] == 8                       # short runs
    assert plan(harness, nchan=1, nif=1)["K"] == 2
    assert plan(harness, nchan=64, flavor=1)["K"] == 8                   # plain comparator


@pytest.mark.parametrize("threads", [128, 256])
def test_tile_shape(harness, threads):
    for nchan, nif in [(256, 4), (64, 1), (48, 3), (1, 1), (512, 8)]:
        p = plan(harness, nchan=nchan, nif=nif, threads=threads)
        assert p["rc"] == 0
        assert p["R"] * p["Bt"] == threads and p["R"] >= 8
        assert p["R"] & (p["R"] - 1) == 0
        assert p["nBlockTiles"] * p["Bt"] >= p["nblocks"]
        # no smaller waste among power-of-two tile widths
        waste = p["nBlockTiles"] * p["Bt"] - p["nblocks"]
        for bt in [1, 2, 4, 8, 16, 32]:
            if threads // bt >= 8:
                assert waste <= math.ceil(p["nblocks"] / bt) * bt - p["nblocks"]


def test_shared_memory_budget(harness):
    for kind, lcomp, nterm in [(0, 4, 0), (1, 5, 1), (4, 8, 1), (5, 12, 0)]:
        p = plan(harness, nchan=256, nif=4, kind=kind, lcomp=lcomp, nterm=nterm, nspec=4 if kind == 5 else 0,
                 lnspec=np.zeros(1024), specIndex=np.zeros(1024, int))
        assert p["rc"] == 0
        assert p["smem"] <= 220 * 1024
        assert p["ct"] % 2 == 0


def test_channel_increment_classes(harness):
    nchan, nif = 32, 3
    f = np.concatenate([1.0 + np.arange(nchan) * d for d in (1e-3, 2e-3, 1e-3)])
    p = plan(harness, nchan=nchan, nif=nif, fscale=f)
    assert p["ndf"] == 2
    dfs = sorted(p["df"])
    assert abs(dfs[0] - 1e-3) < 1e-15 and abs(dfs[1] - 2e-3) < 1e-15


def test_nonuniform_frequencies_use_single_channel_blocks(harness):
    rng = np.random.default_rng(0)
    f = 1.0 + np.sort(rng.uniform(0, 0.05, 40))
    p = plan(harness, nchan=40, nif=1, fscale=f)
    assert p["rc"] == 0 and p["linear"] == 0
    assert p["K"] == 2
    assert all(b["len"] == 1 for b in p["blocks"])
    assert sorted(covered(p, 40, 1)) == [(c, 0) for c in range(40)]


def test_tabulated_planes_split_blocks(harness):
    nchan, nif = 64, 2
    idx = np.array([0] * 20 + [1] * 30 + [2] * 14 + [2] * 10 + [3] * 54)
    f = 1.4e9 + (np.arange(128) % nchan) * 1e6 + (np.arange(128) // nchan) * 100e6
    spec = np.array([1.39e9, 1.42e9, 1.46e9, 1.52e9])
    ln = np.log(f / spec[idx])
    p = plan(harness, nchan=nchan, nif=nif, kind=2, lcomp=9, nspec=4, fscale=f / 1.4e9, lnspec=ln,
             specIndex=idx)
    assert p["rc"] == 0
    for b in p["blocks"]:
        planes = {int(idx[b["ifq0"] + k]) for k in range(b["len"])}
        assert planes == {b["plane"]}
    assert len(covered(p, nchan, nif)) == 128


@pytest.mark.parametrize("nterm", [1, 2, 3])
def test_log_frequency_quadratic_fits(harness, nterm):
    """The per-block quadratic in k reproduces ln(nu/nu0)^(t+1) to < 1e-6."""
    nchan, nif = 256, 4
    nu = 0.888e9 + (np.arange(1024) % nchan) * 1e6 + (np.arange(1024) // nchan) * 256e6
    ln = np.log(nu / 1.4e9)
    p = plan(harness, nchan=nchan, nif=nif, kind=1, nterm=nterm, lcomp=4 + nterm, fscale=nu / 1.4e9,
             lnspec=ln)
    assert p["rc"] == 0
    worst = 0.0
    for b in p["blocks"]:
        for k in range(b["len"]):
            x = ln[b["ifq0"] + k]
            for t in range(nterm):
                l0, l1, l2 = b["l"][t]
                worst = max(worst, abs(l0 + l1 * k + l2 * k * k - x ** (t + 1)))
    assert worst < 1e-6, worst


def test_rejects_bad_selection(harness):
    assert plan(harness, nchan=16, chanb=4, chane=20)["rc"] == 3
    assert plan(harness, nchan=16, K=3)["rc"] == 3


def test_default_cta_size_for_short_rows(harness):
    """Left to the planner (threads 0), recurrence plans take 128-thread CTAs
    when the rows have at most two channel blocks (a 256-thread tile would
    span 128 rows), 256 otherwise; the plain comparator keeps 256."""
    p = plan(harness, nchan=64, nif=1, threads=0)  # 2 blocks of 32
    assert p["rc"] == 0 and p["threads"] == 128 and p["Bt"] == 2 and p["R"] == 64
    p = plan(harness, nchan=256, nif=4, threads=0)
    assert p["rc"] == 0 and p["threads"] == 256
    p = plan(harness, nchan=64, nif=1, threads=0, flavor=1)
    assert p["rc"] == 0 and p["threads"] == 256


def test_factored_point_tiles_keep_128_components(harness):
    """The factored point kernels (compensation terms and s^8 in shared memory,
    plus the low-part region) still take 128-component tiles at the tile
    shapes the autotuner and planner use: two 128-thread CTAs per SM (110 KB
    each) and one 256-thread CTA (200 KB)."""
    p = plan(harness, kind=0, lcomp=4, nchan=256, nif=1, threads=128, Bt=8, ct=128)
    assert p["rc"] == 0 and p["K"] == 32 and p["R"] == 16 and p["ct"] == 128
    assert p["smem"] <= 110 * 1024
    p = plan(harness, kind=0, lcomp=4, nchan=512, nif=8, threads=256, Bt=16, ct=128)
    assert p["rc"] == 0 and p["ct"] == 128 and p["smem"] <= 200 * 1024


def test_spectral_factored_choice(harness):
    """Point components with one spectral index take the spectral-factored form
    only when the table order is known and every tile's spread of indices keeps
    the residual quadratic below the bound; otherwise the chain form."""
    nchan, nif = 256, 4
    f = 1.4e9 + (np.arange(nchan * nif) % nchan) * 1e6 + (np.arange(nchan * nif) // nchan) * 256e6
    ln = np.log(f / 1.4e9)
    kw = dict(nchan=nchan, nif=nif, kind=1, nterm=1, lcomp=5, fscale=f / 1.4e9, lnspec=ln, ct=128)
    rng = np.random.default_rng(5)
    alpha = rng.uniform(-1.5, 0.5, 20000).astype(np.float32)
    p = plan(harness, **kw, compIndex=np.sort(alpha))
    assert p["rc"] == 0 and p["specFactored"] == 1 and p["K"] == 32
    # the same indices in random order: tiles span the whole range
    assert plan(harness, **kw, compIndex=alpha)["specFactored"] == 0
    # order unknown, or turned off, or more than one spectral term
    assert plan(harness, **kw)["specFactored"] == 0
    # tabulated spectra take it too
    p = plan(harness, **{**kw, "kind": 2, "nterm": 0, "lcomp": 9, "nspec": 4,
                         "specIndex": (np.arange(nchan * nif) // nchan)}, compIndex=np.sort(alpha))
    assert p["specFactored"] == 1
    # the layout with the factored table fits the shared-memory budget
    assert p["smem"] <= 220 * 1024
    # a handful of components with indices far apart share one tile: chain form
    assert plan(harness, **kw, compIndex=np.array([-2.0, 0.0, 2.0], np.float32))["specFactored"] == 0
    # equal indices: any spread is zero
    assert plan(harness, **kw, compIndex=np.full(300, -0.7, np.float32))["specFactored"] == 1


def test_mixed_gaussian_plan(harness):
    """A Gaussian table split into ordered point rows and Gaussian rows plans
    mixed; layouts that cannot (short blocks from non-uniform frequencies, or
    point rows failing the residual bound) report 4 so that the caller plans
    the unsplit table."""
    nchan, nif = 256, 4
    f = 1.4e9 + (np.arange(nchan * nif) % nchan) * 1e6 + (np.arange(nchan * nif) // nchan) * 256e6
    kw = dict(nchan=nchan, nif=nif, kind=4, nterm=1, lcomp=8, fscale=f / 1.4e9, lnspec=np.log(f / 1.4e9),
              ct=128)
    alpha = np.sort(np.random.default_rng(6).uniform(-1.5, 0.5, 35000)).astype(np.float32)
    p = plan(harness, **kw, compIndex=alpha, ngauss=15000)
    assert p["rc"] == 0 and p["mixed"] == 1 and p["specFactored"] == 0 and p["K"] == 32
    assert p["smem"] <= 220 * 1024
    assert plan(harness, **kw, compIndex=alpha[::700], ngauss=15000)["rc"] == 4   # wide tiles
    g = f.copy()
    g[3] += 17.0  # one channel off the uniform grid: short blocks
    assert plan(harness, **{**kw, "fscale": g / 1.4e9}, compIndex=alpha, ngauss=15000)["rc"] == 4
    # tabulated spectra
    p = plan(harness, **{**kw, "kind": 5, "nterm": 0, "lcomp": 12, "nspec": 4,
                         "specIndex": (np.arange(nchan * nif) // nchan)}, compIndex=alpha, ngauss=100)
    assert p["rc"] == 0 and p["mixed"] == 1
