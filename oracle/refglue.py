"""Test infrastructure: the reference's own host glue (ObitSystem/Obit/src/
ObitGPUSkyModel.c and ObitCUDAUtil.cu, compiled unmodified by oracle/Makefile
with refglue.c standing in for Obit's object system) driven over a CUDA
sky-model layer:

  which="ours"  _ref/libobit_refglue.so      -> this repository's libobit_dft.so
                                                 (the drop-in, through its void
                                                 ObitCUDASkyModelDFT* symbols)
  which="ref"   _ref/libobit_refglue_ref.so  -> the reference's ObitCUDASkyModel.cu

The GPUInfo is therefore filled exactly as the reference fills it
(ObitGPUSkyModel.c:207-491): stokFact = factor on every polarization, doSwap =
doFlip, the FP32 freqScale only, the first two polarizations, no call of this
library's status-returning additions.

The glue resets its own CUDA context in DFTInit (ObitCUDAResetGPU) and the
reference's layer again at shutdown, so every run is a child process of its
own: `python refglue.py <which> <in.npz> <out.npz>`.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBS = {"ours": HERE / "_ref" / "libobit_refglue.so", "ref": HERE / "_ref" / "libobit_refglue_ref.so"}


class RefGlueJob(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nvis", "lrec", "nrparm", "ilocu", "ilocv", "ilocw",
                                       "nstok", "nchan", "nif")] + [
        ("crvalStokes", C.c_double), ("uvFreq", C.c_double), ("fscale", C.POINTER(C.c_float)),
    ] + [(n, C.c_int) for n in ("startChann", "numberChann", "startIF", "numberIF", "modType",
                                "nSpecTerm")] + [
        ("factor", C.c_float), ("doDivide", C.c_int), ("doReplace", C.c_int), ("doFlip", C.c_int),
        ("imageFreq", C.c_double), ("isMF", C.c_int), ("nSpec", C.c_int),
        ("specFreq", C.POINTER(C.c_double)), ("specIndex", C.POINTER(C.c_int)),
        ("comps", C.POINTER(C.c_float)), ("ncomp", C.c_int), ("lcomp", C.c_int),
        ("gpu", C.c_int), ("nVisPIO", C.c_int), ("vis", C.POINTER(C.c_float)),
    ]


def available(which: str = "ours") -> bool:
    return LIBS[which].exists()


def _child(which: str, src: str, dst: str) -> int:
    d = dict(np.load(src, allow_pickle=False))
    vis = np.ascontiguousarray(d["vis"], dtype=np.float32)
    fscale = np.ascontiguousarray(d["fscale"], dtype=np.float32)
    comps = np.ascontiguousarray(d["comps"], dtype=np.float32)
    spec_freq = np.ascontiguousarray(d["specFreq"], dtype=np.float64)
    spec_index = np.ascontiguousarray(d["specIndex"], dtype=np.int32)
    i = {k: int(v) for k, v in zip(d["int_keys"], d["int_vals"])}
    f = {k: float(v) for k, v in zip(d["flt_keys"], d["flt_vals"])}
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    j = RefGlueJob()
    for k in ("nvis", "lrec", "nrparm", "ilocu", "ilocv", "ilocw", "nstok", "nchan", "nif",
              "startChann", "numberChann", "startIF", "numberIF", "modType", "nSpecTerm",
              "doDivide", "doReplace", "doFlip", "isMF", "nSpec", "ncomp", "lcomp", "gpu", "nVisPIO"):
        setattr(j, k, i[k])
    j.crvalStokes, j.uvFreq, j.factor, j.imageFreq = f["crvalStokes"], f["uvFreq"], f["factor"], f["imageFreq"]
    j.fscale = P(fscale, C.c_float)
    j.comps = P(comps, C.c_float)
    j.specFreq = P(spec_freq, C.c_double)
    j.specIndex = P(spec_index, C.c_int)
    j.vis = P(vis, C.c_float)
    lib = C.CDLL(str(LIBS[which]))
    lib.refglue_run.restype = C.c_int
    lib.refglue_run.argtypes = [C.POINTER(RefGlueJob)]
    lib.refglue_nvispio.restype = C.c_int
    rc = lib.refglue_run(C.byref(j))
    np.savez(dst, vis=vis, rc=np.int32(rc), nvispio=np.int32(lib.refglue_nvispio()))
    return rc


def run(uv, sky, factor: float = 1.0, op: int = 0, doFlip: bool = False, startChann: int = 1,
        numberChann: int = 0, startIF: int = 1, numberIF: int = 0, which: str = "ours",
        gpu: int = 0, timeout: float = 600.0):
    """Apply `sky` to a copy of uv.vis through ObitGPUSkyModelDFTInit / SetMod /
    Calc / Shutdown over the chosen CUDA layer.  The table is used as given
    (the reference's tables already hold flux x factor; `factor` is what the
    glue also puts into stokFact).  op: 0 subtract, 1 divide, 2 replace.
    Returns (records, the glue's buffer size in records)."""
    from obit_b200 import uvdata as U

    nfreq = uv.nchan * uv.nif
    is_mf = sky.modType in (U.MOD_POINT_TSPEC, U.MOD_GAUSS_TSPEC)
    ints = {"nvis": uv.nvis, "lrec": uv.lrec, "nrparm": uv.nrparm, "ilocu": uv.ilocu,
            "ilocv": uv.ilocv, "ilocw": uv.ilocw, "nstok": uv.nstok, "nchan": uv.nchan,
            "nif": uv.nif, "startChann": startChann,
            "numberChann": numberChann or uv.nchan - startChann + 1, "startIF": startIF,
            "numberIF": numberIF or uv.nif - startIF + 1, "modType": sky.modType,
            "nSpecTerm": sky.nterm, "doDivide": int(op == 1), "doReplace": int(op == 2),
            "doFlip": int(doFlip), "isMF": int(is_mf), "nSpec": sky.nspec if is_mf else 0,
            "ncomp": sky.ncomp, "lcomp": sky.lcomp, "gpu": gpu, "nVisPIO": uv.nvis}
    flts = {"crvalStokes": uv.crval_stokes, "uvFreq": uv.freq, "factor": factor,
            "imageFreq": sky.refFreq if sky.refFreq > 0 else uv.freq}
    spec_freq = np.asarray(sky.specFreq if is_mf else np.zeros(1), dtype=np.float64)
    spec_index = np.asarray(sky.specIndex if is_mf else np.zeros(nfreq), dtype=np.int32)
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.npz"), os.path.join(d, "out.npz")
        np.savez(src, vis=uv.vis, fscale=uv.fscale, comps=sky.comps, specFreq=spec_freq,
                 specIndex=spec_index, int_keys=np.array(list(ints)), int_vals=np.array(list(ints.values())),
                 flt_keys=np.array(list(flts)), flt_vals=np.array(list(flts.values()), dtype=np.float64))
        p = subprocess.run([sys.executable, str(Path(__file__).resolve()), which, src, dst],
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0 or not os.path.exists(dst):
            raise RuntimeError(f"refglue ({which}) failed, rc={p.returncode}:\n{p.stdout}\n{p.stderr}")
        out = dict(np.load(dst))
    if int(out["rc"]) != 0:
        raise RuntimeError(f"refglue ({which}): the glue reported an Obit error")
    return out["vis"], int(out["nvispio"])


if __name__ == "__main__":
    sys.exit(_child(sys.argv[1], sys.argv[2], sys.argv[3]))
