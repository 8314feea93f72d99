"""ctypes bindings of libobit_dft.so (include/obit_dft.h, include/obit_gpu_skymodel.h).

Loading fails loudly if the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import build as _build

# ---- reference-layout structures (ObitCUDASkyModelInfoDef.h:66-195) --------


class GPUVisInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nvis", "nprod", "nrparm", "lenvis", "nchan", "ilocu", "ilocv", "ilocw", "iloct",
        "ilocb", "ilocsu", "chanb", "chane", "incf", "nIF", "IFb", "IFe", "incif", "nstok",
        "stokb", "stoke", "incs", "stype", "kincif", "kincf")] + [
        ("freqRat", C.POINTER(C.c_float)),
        ("d_freqRat", C.c_void_p),
        ("freqScale", C.c_void_p),
    ]


class GPUModelInfo(C.Structure):
    _fields_ = [
        ("nterm", C.c_int), ("size", C.c_int), ("doSwap", C.c_int), ("type", C.c_int),
        ("opType", C.c_int), ("specIndex", C.POINTER(C.c_int)), ("d_specIndex", C.c_void_p),
        ("nmodel", C.c_int * 4), ("model", C.c_void_p * 4), ("stokFact", C.c_float * 4),
    ]


class GPUInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nvis", "nchan", "nrparm", "lenvis", "modelSize", "nstream", "prtLv", "oldnVisPIO",
        "cuda_device", "bufferSize")] + [
        ("nmodel", C.c_int * 4), ("d_model", C.c_void_p * 4), ("d_freq", C.c_void_p),
        ("h_data", C.c_void_p), ("d_data", C.POINTER(C.c_void_p)),
        ("d_visInfo", C.POINTER(GPUVisInfo)), ("h_visInfo", C.POINTER(GPUVisInfo)),
        ("d_modelInfo", C.POINTER(GPUModelInfo)), ("h_modelInfo", C.POINTER(GPUModelInfo)),
        ("stream", C.POINTER(C.c_void_p)), ("cycleDone", C.POINTER(C.c_void_p)),
    ]


# ---- host-mirror structures (obit_gpu_skymodel.h) ----------------------------


class ObitDFTUVData(C.Structure):
    _fields_ = [
        ("nvis", C.c_int), ("numVisBuff", C.c_int), ("lrec", C.c_int), ("nrparm", C.c_int),
        ("ncorr", C.c_int), ("ilocu", C.c_int), ("ilocv", C.c_int), ("ilocw", C.c_int),
        ("inaxes", C.c_int * 7), ("jlocs", C.c_int), ("jlocf", C.c_int), ("jlocif", C.c_int),
        ("incs", C.c_int), ("incf", C.c_int), ("incif", C.c_int),
        ("crvalStokes", C.c_double), ("freq", C.c_double),
        ("freqArr", C.POINTER(C.c_double)), ("fscale", C.POINTER(C.c_float)),
        ("buffer", C.POINTER(C.c_float)),
    ]


class ObitDFTSkyModel(C.Structure):
    _fields_ = [
        ("modType", C.c_int), ("nSpecTerm", C.c_int), ("factor", C.c_float),
        ("doDivide", C.c_int), ("doReplace", C.c_int), ("doFlip", C.c_int),
        ("stokFactor", C.c_float), ("startChannelPB", C.c_int), ("numberChannelPB", C.c_int),
        ("startIFPB", C.c_int), ("numberIFPB", C.c_int), ("startPoln", C.c_int),
        ("numberPoln", C.c_int), ("modelRefFreq", C.c_double), ("isMF", C.c_int),
        ("nSpec", C.c_int), ("specFreq", C.POINTER(C.c_double)),
        ("specIndex", C.POINTER(C.c_int)), ("GPU_no", C.c_int), ("nVisPIO", C.c_int),
    ]


class ObitDFTErr(C.Structure):
    _fields_ = [("error", C.c_int), ("prtLv", C.c_int), ("message", C.c_char * 512)]


class ObitDFTCCField(C.Structure):
    _fields_ = [
        ("nrow", C.c_int), ("flux", C.POINTER(C.c_float)), ("deltaX", C.POINTER(C.c_float)),
        ("deltaY", C.POINTER(C.c_float)), ("deltaZ", C.POINTER(C.c_float)),
        ("parms", C.POINTER(C.c_float)), ("nparms", C.c_int), ("status", C.POINTER(C.c_int)),
        ("startComp", C.c_int), ("endComp", C.c_int), ("crvalRA", C.c_double),
        ("crvalDec", C.c_double), ("rotation", C.c_float), ("do3D", C.c_int),
        ("xPxOff", C.c_float), ("yPxOff", C.c_float), ("cdeltX", C.c_float), ("cdeltY", C.c_float),
        ("xShift", C.c_float), ("yShift", C.c_float), ("ncpProjection", C.c_int),
    ]


class ObitDFTCCModel(C.Structure):
    _fields_ = [
        ("uvRA", C.c_double), ("uvDec", C.c_double), ("uvRotation", C.c_float),
        ("factor", C.c_float), ("minFlux", C.c_float), ("minDFT", C.c_float), ("noNeg", C.c_int),
        ("do3D", C.c_int),
    ]


class ObitDFTCCModelMF(C.Structure):
    _fields_ = [
        ("nSpec", C.c_int), ("specFreq", C.POINTER(C.c_double)), ("noSIfit", C.c_int),
        ("doAlphaCorr", C.c_int), ("priorAlpha", C.c_float), ("priorAlphaRefF", C.c_double),
    ]


class ObitDFTFacet(C.Structure):
    _fields_ = [
        ("visInfo", C.POINTER(GPUVisInfo)), ("modelInfo", C.POINTER(GPUModelInfo)),
        ("freqArr", C.POINTER(C.c_double)), ("uvRefFreq", C.c_double),
        ("modelRefFreq", C.c_double), ("specFreq", C.POINTER(C.c_double)), ("nSpec", C.c_int),
        ("cpuRules", C.c_int), ("stokFactor", C.c_float), ("doFlip", C.c_int),
        ("d_vis", C.c_void_p), ("nvis", C.c_int),
    ]


class ObitDFTBeam(C.Structure):
    _fields_ = [
        ("numAnt", C.c_int), ("numAntType", C.c_int), ("numJChan", C.c_int),
        ("antType", C.POINTER(C.c_int)), ("jchan", C.POINTER(C.c_int)),
        ("ilocb", C.c_int), ("iloca1", C.c_int), ("iloca2", C.c_int), ("stokType", C.c_int),
        ("jones", C.c_void_p), ("jonesComps", C.c_int), ("parAng", C.c_float), ("circular", C.c_int),
    ]


class ObitDFTGridImage(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("crpixX", C.c_float), ("crpixY", C.c_float)]


class ObitDFTBeamImages(C.Structure):
    _fields_ = [
        ("numAntType", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nplane", C.c_int),
        ("pixels", C.c_void_p), ("fblank", C.c_float), ("hwidth", C.c_int), ("projection", C.c_int),
        ("crval", C.c_double * 2), ("crpix", C.c_float * 2), ("cdelt", C.c_float * 2),
        ("planeFreq", C.POINTER(C.c_float)), ("refSizeFact", C.c_float), ("crota", C.c_float),
    ]


# ---- exported symbols, with C signatures ------------------------------------

_GPUINFO_P = C.POINTER(GPUInfo)
SIGNATURES = {
    # level 1: the reference's CUDA-layer entry points
    "ObitCUDASkyModelDFTInit": (None, [_GPUINFO_P]),
    "ObitCUDASkyModelDFTSetMod": (None, [_GPUINFO_P]),
    "ObitCUDASkyModelDFTCalc": (None, [_GPUINFO_P]),
    "ObitCUDASkyModelDFTShutdown": (None, [_GPUINFO_P]),
    "ObitCUDASkyModelDFTSetModD": (None, [_GPUINFO_P, C.POINTER(C.c_double), C.c_int]),
    # level 2: status-returning API
    "obit_dft_init": (C.c_int, [_GPUINFO_P]),
    "obit_dft_set_mod": (C.c_int, [_GPUINFO_P]),
    "obit_dft_calc": (C.c_int, [_GPUINFO_P]),
    "obit_dft_shutdown": (C.c_int, [_GPUINFO_P]),
    "obit_dft_set_freq": (C.c_int, [_GPUINFO_P, C.POINTER(C.c_double), C.c_int, C.c_double,
                                    C.c_double, C.POINTER(C.c_double), C.c_int]),
    "obit_dft_set_poln": (C.c_int, [_GPUINFO_P, C.c_int, C.c_float, C.c_int]),
    "obit_dft_set_mod_d": (C.c_int, [_GPUINFO_P, C.POINTER(C.c_double), C.c_int]),
    "obit_dft_set_beam": (C.c_int, [_GPUINFO_P, C.POINTER(ObitDFTBeam)]),
    "obit_dft_beam_jones": (C.c_int, [C.POINTER(ObitDFTBeamImages), C.c_void_p, C.c_int, C.c_float,
                                      C.c_void_p, C.c_void_p]),
    "obit_dft_set_kernel": (C.c_int, [_GPUINFO_P, C.c_int, C.c_int, C.c_int]),
    "obit_dft_set_tile": (C.c_int, [_GPUINFO_P, C.c_int, C.c_int]),
    "obit_dft_calc_device": (C.c_int, [_GPUINFO_P, C.c_void_p, C.c_int, C.c_void_p]),
    "obit_dft_plan_info": (C.c_int, [_GPUINFO_P, C.POINTER(C.c_int), C.c_int]),
    "obit_dft_beam_info": (C.c_int, [_GPUINFO_P, C.POINTER(C.c_int), C.c_int]),
    "obit_dft_sub_uv_image": (C.c_int, [C.POINTER(C.c_void_p), C.c_float, C.POINTER(ObitDFTCCField), C.c_int,
                                        C.POINTER(ObitDFTGridImage), C.POINTER(ObitDFTCCModel),
                                        C.POINTER(ObitDFTSkyModel), C.POINTER(ObitDFTUVData), C.c_int,
                                        C.POINTER(C.c_longlong), C.POINTER(ObitDFTErr)]),
    "obit_dft_sub_uv": (C.c_int, [C.POINTER(ObitDFTCCField), C.c_int, C.POINTER(ObitDFTGridImage),
                                  C.POINTER(ObitDFTCCModel), C.POINTER(ObitDFTSkyModel),
                                  C.POINTER(ObitDFTUVData), C.c_int, C.c_int, C.c_float, C.c_int,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(ObitDFTErr)]),
    "obit_dft_calc_noalloc": (C.c_int, [C.POINTER(GPUVisInfo), C.POINTER(GPUModelInfo),
                                        C.POINTER(C.c_double), C.c_double, C.c_double,
                                        C.POINTER(C.c_double), C.c_int, C.c_void_p, C.c_int,
                                        C.c_void_p]),
    "obit_dft_batch_create": (C.c_int, [C.POINTER(ObitDFTFacet), C.c_int, C.POINTER(C.c_void_p)]),
    "obit_dft_batch_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "obit_dft_batch_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "obit_dft_batch_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "obit_dft_batch_run_per_facet": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "obit_dft_batch_run_host": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_longlong, C.c_void_p,
                                          C.POINTER(C.c_longlong)]),
    "obit_dft_batch_check": (C.c_int, [C.c_void_p]),
    "obit_dft_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.c_int]),
    "obit_dft_batch_destroy": (C.c_int, [C.c_void_p]),
    "obit_dft_load_comps": (C.c_int, [C.POINTER(ObitDFTCCField), C.c_int, C.POINTER(ObitDFTCCModel),
                                      C.POINTER(C.c_float), C.c_longlong, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    "obit_dft_load_comps_d": (C.c_int, [C.POINTER(ObitDFTCCField), C.c_int, C.POINTER(ObitDFTCCModel),
                                        C.POINTER(C.c_float), C.c_longlong, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "obit_dft_load_comps_mf": (C.c_int, [C.POINTER(ObitDFTCCField), C.c_int, C.POINTER(ObitDFTCCModel),
                                         C.POINTER(ObitDFTCCModelMF), C.POINTER(C.c_float), C.c_longlong,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
    # gridded model FT (obit_dft_grid.h)
    "obit_dft_grid_create": (C.c_int, [C.POINTER(ObitDFTCCField), C.POINTER(ObitDFTGridImage),
                                       C.POINTER(ObitDFTCCModel), C.c_float, C.c_int, C.c_void_p,
                                       C.POINTER(C.c_void_p)]),
    "obit_dft_grid_create_image": (C.c_int, [C.c_void_p, C.c_float, C.POINTER(ObitDFTCCField),
                                             C.POINTER(ObitDFTGridImage), C.POINTER(ObitDFTCCModel), C.c_int,
                                             C.c_void_p, C.POINTER(C.c_void_p)]),
    "obit_dft_grid_apply": (C.c_int, [C.c_void_p, C.POINTER(GPUVisInfo), C.c_int, C.c_float, C.c_int,
                                      C.c_void_p, C.c_int, C.c_void_p]),
    "obit_dft_grid_apply_host": (C.c_int, [C.c_void_p, C.POINTER(GPUVisInfo), C.c_int, C.c_float, C.c_int,
                                           C.c_void_p, C.c_int, C.c_void_p]),
    "obit_dft_grid_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.c_int]),
    "obit_dft_grid_plane": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_longlong]),
    "obit_dft_grid_destroy": (C.c_int, [C.c_void_p]),
    "obit_dft_choose_mode": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.c_int, C.c_longlong, C.c_int]),
    # records resident across major cycles
    "obit_dft_resident_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "obit_dft_resident_reset": (C.c_int, [C.c_void_p, C.c_void_p]),
    "obit_dft_resident_records": (C.c_void_p, [C.c_void_p]),
    "obit_dft_resident_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "obit_dft_resident_destroy": (C.c_int, [C.c_void_p]),
    "obit_dft_choose_mode_measured": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                C.POINTER(C.c_int), C.c_int, C.c_longlong, C.c_int, C.c_double,
                                                C.c_double, C.c_double]),
    "obit_dft_check": (C.c_int, [_GPUINFO_P]),
    "obit_dft_set_wait_limit": (C.c_int, [_GPUINFO_P, C.c_int]),
    "obit_dft_last_error": (C.c_char_p, []),
    "obit_dft_version": (C.c_int, []),
    # host mirror of the GPU sky-model class
    "obit_gpu_skymodel_create": (C.c_void_p, [C.c_char_p]),
    "obit_gpu_skymodel_dft_init": (C.c_int, [C.c_void_p, C.POINTER(ObitDFTSkyModel),
                                             C.POINTER(ObitDFTUVData), C.POINTER(ObitDFTErr)]),
    "obit_gpu_skymodel_dft_setmod": (C.c_int, [C.c_void_p, C.POINTER(ObitDFTSkyModel),
                                               C.POINTER(C.c_float), C.c_int, C.c_int,
                                               C.POINTER(ObitDFTErr)]),
    "obit_gpu_skymodel_dft_calc": (C.c_int, [C.c_void_p, C.POINTER(ObitDFTUVData),
                                             C.POINTER(ObitDFTErr)]),
    "obit_gpu_skymodel_dft_shutdown": (C.c_int, [C.c_void_p, C.POINTER(ObitDFTErr)]),
    "obit_gpu_skymodel_unref": (None, [C.c_void_p]),
    "obit_gpu_skymodel_info": (_GPUINFO_P, [C.c_void_p]),
}

OBIT_DFT_RECUR = 0
OBIT_DFT_PLAIN = 1
OBIT_DFT_RECUR_CHAIN = 2  # recurrence without the spectral-factored form (comparator)
OBIT_DFT_GRID_KERNEL_REFERENCE = 0  # the reference's interpolation-kernel table
OBIT_DFT_GRID_KERNEL_EXACT = 1      # Lagrange weights at the requested point

_lib = None


class DFTError(RuntimeError):
    """Error status returned by libobit_dft.so."""

    def __init__(self, code: int, message: str):
        super().__init__(f"obit_dft error {code}: {message}")
        self.code = code


def lib_path() -> Path:
    return _build.LIB


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load libobit_dft.so (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ["OBIT_DFT_LIB"]) if os.environ.get("OBIT_DFT_LIB") else _build.LIB
    if not path.exists() and path == _build.LIB:
        if build_if_missing and os.environ.get("OBIT_DFT_NO_BUILD") != "1":
            _build.build()
        if not path.exists():
            raise RuntimeError(f"{path} is missing and could not be built; the CUDA path "
                               "is the only implementation")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = _lib.obit_dft_last_error().decode() if _lib is not None else ""
        raise DFTError(rc, msg)
