"""obit_dft_calc_noalloc, the entry point for callers that cannot let a
library allocate device memory (processes whose own pool owns every device
byte, latency-bound callers that cannot take cudaFree's device-wide
synchronization): through the C ABI, on two calls
in a row, its records must match those of the regular device-resident entry
point obit_dft_calc_device on the same inputs, within the parity tolerance.

Collected last so that a run stopping at the first failure has run every other
test before this one; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import TOL_REL, small
from obit_b200 import _lib
from obit_b200 import uvdata as U
from obit_b200.skymodel import OP_REPL, OP_SUB, GPUSkyModel, SkyModelParams

pytestmark = pytest.mark.gpu


def _regular(uv, sky, params, torch):
    """Records after obit_dft_calc_device on a device copy."""
    d_vis = torch.from_numpy(uv.vis.copy()).cuda()
    p = SkyModelParams(**{**params.__dict__, "nVisPIO": uv.nvis})
    gm = GPUSkyModel("regular")
    try:
        gm.DFTInit(sky, uv, p)
        gm.DFTSetMod(sky)
        gm.calc_device(d_vis.data_ptr(), uv.nvis, 0)
        gm.check()
        gm.DFTShutdown()
    finally:
        gm.close()
    return d_vis.cpu().numpy()


def _noalloc(uv, sky, params, torch, check_mem=False):
    """Records after obit_dft_calc_noalloc; inputs and outputs in device memory
    the test owns, descriptors filled as ObitGPUSkyModelDFTInit/SetMod would.
    check_mem: the device's free memory must be the same before and after the
    call (use it on a repeated call: the first launch of a kernel may load its
    code, which takes device memory)."""
    lib = _lib.load()
    keep = []
    fscale = torch.from_numpy(uv.fscale).cuda()
    comps = torch.from_numpy(np.ascontiguousarray(sky.comps)).cuda()
    d_vis = torch.from_numpy(uv.vis.copy()).cuda()
    vi = _lib.GPUVisInfo()
    vi.nvis, vi.nprod, vi.nrparm, vi.lenvis = uv.nvis, uv.ncorr, uv.nrparm, uv.lrec
    vi.nchan, vi.nIF, vi.nstok = uv.nchan, uv.nif, uv.nstok
    vi.ilocu, vi.ilocv, vi.ilocw = uv.ilocu, uv.ilocv, uv.ilocw
    vi.iloct = vi.ilocb = vi.ilocsu = -1
    vi.chanb, vi.chane, vi.IFb, vi.IFe = 0, uv.nchan - 1, 0, uv.nif - 1
    vi.stokb, vi.stoke = 0, min(2, uv.nstok) - 1
    vi.incf, vi.incif, vi.incs = uv.incf // 3, uv.incif // 3, uv.incs // 3
    vi.kincf, vi.kincif = uv.kincf, uv.kincif
    vi.stype = 1
    vi.freqScale = fscale.data_ptr()
    mi = _lib.GPUModelInfo()
    mi.nterm, mi.size, mi.doSwap, mi.type = sky.nterm, sky.lcomp, 0, sky.gpu_type
    mi.opType = params.op
    mi.nmodel[0] = sky.ncomp
    mi.model[0] = comps.data_ptr()
    for i in range(4):
        mi.stokFact[i] = 1.0
    spec = None
    if sky.is_tspec:
        si = np.ascontiguousarray(sky.specIndex, dtype=np.int32)
        keep.append(si)
        mi.specIndex = si.ctypes.data_as(C.POINTER(C.c_int))
        spec = np.ascontiguousarray(sky.specFreq, dtype=np.float64)
        keep.append(spec)
    fa = np.ascontiguousarray(uv.freqArr, dtype=np.float64)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0] if check_mem else None
    rc = lib.obit_dft_calc_noalloc(
        C.byref(vi), C.byref(mi), fa.ctypes.data_as(C.POINTER(C.c_double)), uv.freq,
        sky.refFreq if sky.refFreq > 0 else uv.freq,
        spec.ctypes.data_as(C.POINTER(C.c_double)) if spec is not None else None,
        0 if spec is None else len(spec), C.c_void_p(d_vis.data_ptr()), uv.nvis, None)
    _lib.check(rc)
    if check_mem:
        assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
    return d_vis.cpu().numpy()


def _max_rel(a, b, uv, sky, params):
    _, l1 = oracle.model_fp64(uv, sky, params)
    x = a[:, uv.nrparm:].reshape(uv.nvis, uv.nif, uv.nchan, uv.nstok, 3)
    y = b[:, uv.nrparm:].reshape(x.shape)
    d = np.abs((x[..., 0] - y[..., 0]) + 1j * (x[..., 1] - y[..., 1]))[..., :2]
    assert np.array_equal(x[..., 2], y[..., 2])
    return float(np.max(d / l1[..., None]))


def test_noalloc_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    cases = [
        (small(U.MOD_POINT_SPEC, nrow=90, nchan=48, nif=3, nstok=4, ncomp=301, seed=21),
         SkyModelParams(op=OP_SUB)),
        (small(U.MOD_GAUSS_TSPEC, nrow=57, nchan=33, nif=2, nstok=2, ncomp=77, seed=22),
         SkyModelParams(op=OP_REPL)),
    ]
    for (uv, sky), params in cases:  # two calls in a row, different models
        want = _regular(uv, sky, params, torch)
        got = _noalloc(uv, sky, params, torch)
        assert not np.array_equal(got, uv.vis)
        assert _max_rel(got, want, uv, sky, params) < TOL_REL
        # the same call again, its kernel now loaded: no device memory is taken
        again = _noalloc(uv, sky, params, torch, check_mem=True)
        assert np.array_equal(again, got)


def test_noalloc_rejects_models_beyond_the_static_limit():
    torch = pytest.importorskip("torch")
    uv, sky = small(U.MOD_POINT_SPEC, nrow=4, nchan=8, nif=1, ncomp=300000, seed=23)
    with pytest.raises(_lib.DFTError) as e:
        _noalloc(uv, sky, SkyModelParams(op=OP_SUB), torch)
    assert e.value.code == 3 and "static limit" in str(e.value)
