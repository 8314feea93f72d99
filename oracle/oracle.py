"""Test infrastructure: ctypes front end of the CPU oracles (oracle_dft.c and
the reference-derived restatement in _ref/).  Only tests, the smoke check and
bench.py's CPU-baseline leg import this module; the product never does.

A job is described with the same objects the product takes (UVData, SkyComps,
SkyModelParams), mapped to the reference CPU semantics used by the host mirror:
polarization factors follow stokFactor/doFlip (ObitSkyModel.c:2787-2849) and the
channel frequency ratio is FP64 freqArr/freq (exact=True) or the FP32
freqScale the reference GPU interface carries (exact=False).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_A = HERE / "liboracle_dft.so"
LIB_B = HERE / "_ref" / "libobit_refcpu.so"
LIB_J = HERE / "_ref" / "libobit_refjones.so"
LIB_G = HERE / "_ref" / "libobit_refgeom.so"


class OracleJob(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nvis", "lrec", "nrparm", "ilocu", "ilocv", "ilocw", "incs", "incf", "incif", "nchan",
        "nif", "kincf", "kincif", "startChannel", "numberChannel", "startIF", "numberIF",
        "startPoln", "numberPoln", "modType", "nterm", "lcomp", "ncomp")] + [
        ("comps", C.POINTER(C.c_float)),
        ("doDivide", C.c_int), ("doReplace", C.c_int), ("flipMask", C.c_int),
        ("stokFactor", C.c_float), ("polFact", C.c_float * 4),
        ("fscale", C.POINTER(C.c_double)), ("fscale32", C.POINTER(C.c_float)),
        ("lnspec", C.POINTER(C.c_double)), ("specIndex", C.POINTER(C.c_int)),
        ("xyz", C.POINTER(C.c_double)),
    ]


_libA = None
_libB = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def lib_a() -> C.CDLL:
    global _libA
    if _libA is None:
        if not LIB_A.exists():
            build()
        _libA = C.CDLL(str(LIB_A))
        for fn in (_libA.oracle_model_fp64,):
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(OracleJob), C.POINTER(C.c_float), C.POINTER(C.c_double),
                           C.POINTER(C.c_double), C.c_int]
        _libA.oracle_apply_fp64.restype = C.c_int
        _libA.oracle_apply_fp64.argtypes = [C.POINTER(OracleJob), C.POINTER(C.c_float), C.c_int]
    return _libA


def have_refcpu() -> bool:
    return LIB_B.exists()


def lib_b() -> C.CDLL:
    global _libB
    if _libB is None:
        if not LIB_B.exists():
            raise FileNotFoundError(f"{LIB_B} not built (needs the reference sources once)")
        _libB = C.CDLL(str(LIB_B))
        _libB.refcpu_apply.restype = C.c_int
        _libB.refcpu_apply.argtypes = [C.POINTER(OracleJob), C.POINTER(C.c_float), C.c_int]
    return _libB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Job:
    """An OracleJob plus the arrays it points into."""

    def __init__(self, uv, sky, params=None, exact: bool = True, xyz=None, gpu_rules=None):
        from obit_b200.skymodel import OP_DIV, OP_REPL, SkyModelParams
        p = params or SkyModelParams()
        j = OracleJob()
        j.nvis = uv.nvis
        j.lrec = uv.lrec
        j.nrparm = uv.nrparm
        j.ilocu, j.ilocv, j.ilocw = uv.ilocu, uv.ilocv, uv.ilocw
        j.incs, j.incf, j.incif = uv.incs, uv.incf, uv.incif
        j.nchan, j.nif = uv.nchan, uv.nif
        j.kincf, j.kincif = uv.kincf, uv.kincif
        j.startChannel = (p.startChannel if p.startChannel > 0 else 1) - 1
        j.numberChannel = p.numberChannel if p.numberChannel > 0 else uv.nchan - j.startChannel
        j.startIF = (p.startIF if p.startIF > 0 else 1) - 1
        j.numberIF = p.numberIF if p.numberIF > 0 else uv.nif - j.startIF
        j.startPoln = (p.startPoln if p.startPoln > 0 else 1) - 1
        j.numberPoln = p.numberPoln if p.numberPoln > 0 else min(2, uv.nstok)
        j.modType = sky.gpu_type
        j.nterm = sky.nterm
        self.comps = np.ascontiguousarray(sky.comps, dtype=np.float32)
        j.lcomp = self.comps.shape[1]
        j.ncomp = self.comps.shape[0]
        j.comps = _p(self.comps, C.c_float)
        j.doDivide = int(p.op == OP_DIV)
        j.doReplace = int(p.op == OP_REPL)
        j.flipMask = 0xF if p.doFlip else 0
        j.stokFactor = p.stokFactor
        for i in range(4):
            j.polFact[i] = 1.0
        if gpu_rules is not None:
            # the reference GPU plug-in's rules (ObitCUDASkyModel.cu:134-160): the
            # model times stokFact of each polarization, i on polarization 3 when
            # doSwap, no running stokFactor product
            stok_fact, do_swap = gpu_rules
            j.stokFactor = 1.0
            j.flipMask = 0
            for i in range(j.numberPoln):
                ist = j.startPoln + i
                j.polFact[i] = float(stok_fact[ist]) if ist < 4 else 1.0
                if do_swap and ist == 3:
                    j.flipMask |= 1 << i
        fa = np.asarray(uv.freqArr, dtype=np.float64)
        self.fscale32 = np.ascontiguousarray(uv.fscale, dtype=np.float32)
        if exact:
            self.fscale = np.ascontiguousarray(fa / uv.freq)
        else:
            self.fscale = self.fscale32.astype(np.float64)
        j.fscale = _p(self.fscale, C.c_double)
        j.fscale32 = _p(self.fscale32, C.c_float)
        self.lnspec = None
        self.specIndex = None
        if sky.gpu_type in (1, 4):
            ref = sky.refFreq if sky.refFreq > 0 else uv.freq
            nu = fa if exact else self.fscale * uv.freq
            self.lnspec = np.ascontiguousarray(np.log(nu / ref))
        elif sky.gpu_type in (2, 5):
            self.specIndex = np.ascontiguousarray(sky.specIndex, dtype=np.int32)
            nu = fa if exact else self.fscale * uv.freq
            self.lnspec = np.ascontiguousarray(np.log(nu / sky.specFreq[self.specIndex]))
            j.specIndex = _p(self.specIndex, C.c_int)
        if self.lnspec is not None:
            j.lnspec = _p(self.lnspec, C.c_double)
        self.xyz = None
        if xyz is not None:  # FP64 positions in place of the table's FP32 X, Y, Z
            self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
            assert self.xyz.shape[0] >= j.ncomp
            j.xyz = _p(self.xyz, C.c_double)
        self.job = j
        self.uv = uv


def nthreads_default() -> int:
    return max(1, len(os.sched_getaffinity(0)))


def model_fp64(uv, sky, params=None, exact: bool = True, nthreads: int | None = None, xyz=None,
               gpu_rules=None):
    """FP64 component sum and L1 norm per (row, IF, channel):
    returns (model complex128 (nvis, nif, nchan), l1 float64 (nvis, nif, nchan));
    unselected entries are NaN.  xyz: optional (ncomp, 3) FP64 positions used
    for the phase instead of the table's FP32 fields 1-3."""
    jb = Job(uv, sky, params, exact, xyz, gpu_rules)
    nfreq = uv.nchan * uv.nif
    model = np.full((uv.nvis, nfreq, 2), np.nan)
    l1 = np.full((uv.nvis, nfreq), np.nan)
    vis = np.ascontiguousarray(uv.vis, dtype=np.float32)
    rc = lib_a().oracle_model_fp64(C.byref(jb.job), _p(vis, C.c_float), _p(model, C.c_double),
                                   _p(l1, C.c_double), nthreads or nthreads_default())
    if rc:
        raise ValueError(f"oracle_model_fp64 returned {rc}")
    # table index ifq = ichan*kincf + iIF*kincif with kincf=1, kincif=nchan
    m = (model[..., 0] + 1j * model[..., 1]).reshape(uv.nvis, uv.nif, uv.nchan)
    return m, l1.reshape(uv.nvis, uv.nif, uv.nchan)


def apply_fp64(uv, sky, params=None, exact: bool = True, nthreads: int | None = None, xyz=None,
               gpu_rules=None):
    """FP64 oracle applied to a copy of uv.vis; returns the new float32 records.
    gpu_rules: None for the CPU DFT's polarization rules, or (stokFact[4],
    doSwap) for those of the reference GPU plug-in."""
    jb = Job(uv, sky, params, exact, xyz, gpu_rules)
    out = np.ascontiguousarray(uv.vis, dtype=np.float32).copy()
    rc = lib_a().oracle_apply_fp64(C.byref(jb.job), _p(out, C.c_float), nthreads or nthreads_default())
    if rc:
        raise ValueError(f"oracle_apply_fp64 returned {rc}")
    return out


class OracleBeam(C.Structure):
    _fields_ = [
        ("numAnt", C.c_int), ("numAntType", C.c_int), ("numJChan", C.c_int),
        ("antType", C.POINTER(C.c_int)), ("jchan", C.POINTER(C.c_int)),
        ("ilocb", C.c_int), ("iloca1", C.c_int), ("iloca2", C.c_int),
        ("jones", C.POINTER(C.c_float)), ("stokType", C.c_int), ("c2p", C.c_double), ("s2p", C.c_double),
        ("circular", C.c_int),
    ]


def apply_beam_fp64(uv, sky, params, beam, nthreads: int | None = None, xyz=None):
    """FP64 beam-corrected model (oracle_beam.c) applied to a copy of uv.vis:
    returns (records, l1 of shape (nvis, nif, nchan, 4) over the model
    correlations XX, XY, YX, YY).  beam: obit_b200.beam.Beam (host Jones
    table); the first min(2, nstok) correlations, or all four, are modelled.
    xyz: optional (ncomp, 3) FP64 positions used in place of the table's."""
    jb = Job(uv, sky, params, exact=True, xyz=xyz)
    jb.job.startPoln = 0
    jb.job.numberPoln = 4 if uv.nstok >= 4 else min(2, uv.nstok)
    for i in range(4):
        jb.job.polFact[i] = 1.0
    at = np.ascontiguousarray(beam.antType, dtype=np.int32)
    jc = np.ascontiguousarray(beam.jchan, dtype=np.int32)
    jo = np.ascontiguousarray(beam.jones, dtype=np.float32)
    assert jo.shape[1] >= sky.ncomp
    # the parallactic terms as the library forms them (FP64 sin/cos, rounded to float)
    c2p = float(np.float32(np.cos(2.0 * float(beam.parAng))))
    s2p = float(np.float32(np.sin(2.0 * float(beam.parAng))))
    ob = OracleBeam(len(at), jo.shape[0], jo.shape[2], _p(at, C.c_int), _p(jc, C.c_int), beam.ilocb,
                    beam.iloca1, beam.iloca2, _p(jo, C.c_float), int(beam.stokType), c2p, s2p,
                    int(bool(getattr(beam, "circular", False))))
    # the oracle indexes the table with the model's component count
    if jo.shape[1] != sky.ncomp:
        jo = np.ascontiguousarray(jo[:, :sky.ncomp])
        ob.jones = _p(jo, C.c_float)
    out = np.ascontiguousarray(uv.vis, dtype=np.float32).copy()
    l1 = np.full((uv.nvis, uv.nchan * uv.nif, 4), np.nan)
    lib = lib_a()
    lib.oracle_beam_apply.restype = C.c_int
    lib.oracle_beam_apply.argtypes = [C.POINTER(OracleJob), C.POINTER(OracleBeam), C.POINTER(C.c_float),
                                      C.POINTER(C.c_double), C.c_int]
    rc = lib.oracle_beam_apply(C.byref(jb.job), C.byref(ob), _p(out, C.c_float), _p(l1, C.c_double),
                               nthreads or nthreads_default())
    if rc:
        raise ValueError(f"oracle_beam_apply returned {rc}")
    return out, l1.reshape(uv.nvis, uv.nif, uv.nchan, 4)


def beam_coeffs(stok: int, c2p: float, s2p: float, J1, J2):
    """The beam oracle's four model coefficients (XX, XY, YX, YY) of one Jones
    pair (8 floats each): complex128 (4,)."""
    lib = lib_a()
    lib.oracle_beam_coeffs.restype = None
    lib.oracle_beam_coeffs.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_float),
                                       C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    a = np.ascontiguousarray(J1, dtype=np.float32)
    b = np.ascontiguousarray(J2, dtype=np.float32)
    cr, ci = np.zeros(4), np.zeros(4)
    lib.oracle_beam_coeffs(stok, c2p, s2p, _p(a, C.c_float), _p(b, C.c_float), _p(cr, C.c_double),
                           _p(ci, C.c_double))
    return cr + 1j * ci


def have_refjones() -> bool:
    return LIB_J.exists()


def ref_jones_cor1(stok: int, flux: float, sin_ph: float, cos_ph: float, J1, J2, c2p: float, s2p: float):
    """The reference's own cudaJonesCor1_Lin_{I,Q,U,V} for one component (compiled
    for the host): the XX, XY, YX, YY sums as complex128 (4,)."""
    lib = C.CDLL(str(LIB_J))
    lib.ref_jones_cor1.restype = C.c_int
    lib.ref_jones_cor1.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), C.c_float, C.c_float, C.POINTER(C.c_float)]
    a = np.ascontiguousarray(J1, dtype=np.float32)
    b = np.ascontiguousarray(J2, dtype=np.float32)
    out = np.zeros(8, np.float32)
    rc = lib.ref_jones_cor1(stok, flux, sin_ph, cos_ph, _p(a, C.c_float), _p(b, C.c_float), c2p, s2p,
                            _p(out, C.c_float))
    if rc:
        raise ValueError(f"ref_jones_cor1 returned {rc}")
    o = out.astype(np.float64)
    return o[0::2] + 1j * o[1::2]


def have_refgeom() -> bool:
    return LIB_G.exists()


def ref_position_xypix(coord, ctype: str, crval, crpix, cdelt, crota=(0.0, 0.0), rotar: float = 0.0):
    """The reference's own CUDAPositionXYpix (compiled for the host): the
    1-relative pixel of position coord (deg) and the reference's status
    (0 placed, else not)."""
    lib = C.CDLL(str(LIB_G))
    lib.ref_position_xypix.restype = C.c_long
    d2, f2 = C.c_double * 2, C.c_float * 2
    px = f2()
    rc = lib.ref_position_xypix(d2(*coord), ctype.encode(), d2(*crval), f2(*crpix), f2(*cdelt), f2(*crota),
                                C.c_float(rotar), px)
    return (float(px[0]), float(px[1])), int(rc)


def ref_beam_interp_pixel(plane_stack, fblank: float, hwidth: int, pixel) -> float:
    """The reference's own CUDABeamInterpPixel (compiled for the host) on one
    image, plane_stack float32 (nplane, ny, nx), at pixel (x, y, plane), all
    1-relative."""
    lib = C.CDLL(str(LIB_G))
    lib.ref_beam_interp_pixel.restype = C.c_float
    a = np.ascontiguousarray(plane_stack, dtype=np.float32)
    nplane, ny, nx = a.shape
    px = (C.c_float * 3)(*pixel)
    return float(lib.ref_beam_interp_pixel(_p(a, C.c_float), nx, ny, nplane, C.c_float(fblank), hwidth, px))


def apply_refcpu(uv, sky, params=None, nthreads: int | None = None):
    """Reference-faithful CPU restatement (FP32 phase, reference sin/cos)
    applied to a copy of uv.vis; returns the new float32 records."""
    jb = Job(uv, sky, params, exact=True)
    out = np.ascontiguousarray(uv.vis, dtype=np.float32).copy()
    rc = lib_b().refcpu_apply(C.byref(jb.job), _p(out, C.c_float), nthreads or nthreads_default())
    if rc:
        raise ValueError(f"refcpu_apply returned {rc}")
    return out


def beam_jones_fp64(images, pos, par_ang: float):
    """FP64 Jones table from beam images (oracle_beam.c: oracle_beam_jones).
    images: obit_b200.beam.BeamImages (host pixels); pos: (ncomp, 2) offsets in
    degrees.  Returns float32 (ntype, ncomp, nplane, 8)."""
    px = np.ascontiguousarray(images.pixels, dtype=np.float32)
    ntype, _, nplane, ny, nx = px.shape
    pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 2)
    out = np.zeros((ntype, pos.shape[0], nplane, 8), np.float32)
    d3 = C.c_double * 2
    pf = np.ascontiguousarray(images.planeFreq, dtype=np.float64)
    lib = lib_a()
    lib.oracle_beam_jones.restype = None
    lib.oracle_beam_jones(ntype, nx, ny, nplane, _p(px, C.c_float), C.c_float(images.fblank),
                          int(images.hwidth), int(images.projection), d3(*images.crval), d3(*images.crpix),
                          d3(*images.cdelt), C.c_double(images.crota), _p(pf, C.c_double),
                          C.c_double(images.refSizeFact),
                          C.c_double(par_ang), _p(pos, C.c_float), pos.shape[0], _p(out, C.c_float))
    return out
