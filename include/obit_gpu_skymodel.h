/*
 * obit_gpu_skymodel.h - host-side mirror of Obit's GPU sky-model class for the
 * DFT path, in C, over the C ABI of obit_dft.h.
 *
 * It does what ObitGPUSkyModel.c does for one sky model and one uv data set
 * (ObitSystem/Obit/src/ObitGPUSkyModel.c:207-579; class API in
 * ObitSystem/Obit/include/ObitGPUSkyModel.h:95-125): fills a GPUInfo with
 * pinned and device buffers, streams, the visibility and model descriptions,
 * and calls the four CUDA-layer entry points.  Because Obit's object system
 * (ObitUV, ObitSkyModel, ObitErr) is not part of this library, the inputs are
 * small plain structs carrying the fields those objects supply to the
 * reference code; errors go to an ObitErr-like record instead of aborting.
 *
 * Deliberate differences from ObitGPUSkyModel.c, each a reference defect:
 *   - the device is never reset (ObitGPUSkyModel.c:228, ObitCUDASkyModel.cu:780);
 *   - `factor` is applied once (it is already in the component table,
 *     ObitSkyModel.c:1965; the reference sets stokFact = factor again,
 *     ObitGPUSkyModel.c:464-467) and the CPU polarization rules are used
 *     (stokFactor, doFlip), via obit_dft_set_poln;
 *   - the FP64 channel frequencies are passed with obit_dft_set_freq when the
 *     caller supplies them;
 *   - the tabulated-spectrum plane index is copied from host memory rather
 *     than read through a host pointer on the device (ObitCUDASkyModel.cu:295).
 */
#ifndef OBIT_GPU_SKYMODEL_H
#define OBIT_GPU_SKYMODEL_H
#include "obit_dft.h"
#ifdef __cplusplus
extern "C" {
#endif

/* The fields of ObitUV / ObitUVDesc the DFT path reads (ObitUVDesc.h). */
typedef struct {
  int nvis;        /* records in the data set (desc->nvis) */
  int numVisBuff;  /* records now in `buffer` (desc->numVisBuff) */
  int lrec;        /* floats per record */
  int nrparm;      /* random parameters per record */
  int ncorr;       /* correlations per record */
  int ilocu, ilocv, ilocw;
  int inaxes[7];   /* regular axis lengths */
  int jlocs, jlocf, jlocif; /* axis numbers of Stokes, frequency, IF (-1 absent) */
  int incs, incf, incif;    /* float increments (desc->incs ...) */
  double crvalStokes;       /* crval[jlocs]: <0 correlation, >0 Stokes */
  double freq;              /* reference frequency, Hz */
  const double *freqArr;    /* Hz per (channel, IF) in data order, or NULL */
  const float *fscale;      /* freqArr/freq in FP32 (desc->fscale) */
  float *buffer;            /* numVisBuff records (uvdata->buffer) */
} ObitDFTUVData;

/* The fields of ObitSkyModel / ObitSkyModelMF the DFT path reads. */
typedef struct {
  int modType;     /* ObitSkyModelCompType: 0 point, 1 Gaussian, +10 spectrum,
                      +20 tabulated spectrum (ObitSkyModel.h:130-164) */
  int nSpecTerm;   /* spectral terms */
  float factor;    /* already applied in the component table */
  int doDivide, doReplace, doFlip;
  float stokFactor;
  int startChannelPB, numberChannelPB; /* 1-relative channel range */
  int startIFPB, numberIFPB;           /* 1-relative IF range */
  int startPoln, numberPoln;           /* 1-relative polarization range */
  double modelRefFreq;  /* image reference frequency of polynomial spectra */
  int isMF;             /* tabulated spectra (ObitSkyModelMF) */
  int nSpec;            /* coarse planes */
  const double *specFreq; /* Hz per coarse plane */
  const int *specIndex;   /* coarse plane per (channel, IF) */
  int GPU_no;           /* CUDA device (uvdata info "GPU_no") */
  int nVisPIO;          /* records per buffer; <= 0 means the reference's 10000 */
} ObitDFTSkyModel;

/* ObitErr stand-in: error flag, print level and the last message. */
typedef struct {
  int error;
  int prtLv;
  char message[512];
} ObitDFTErr;

/* Opaque instance (ObitGPUSkyModel). */
typedef struct ObitDFTGPUSkyModel ObitDFTGPUSkyModel;

/* ObitGPUSkyModelCreate (ObitGPUSkyModel.h:95). */
ObitDFTGPUSkyModel *obit_gpu_skymodel_create(const char *name);

/* ObitGPUSkyModelDFTInit (ObitGPUSkyModel.h:109, ObitGPUSkyModel.c:207-403). */
int obit_gpu_skymodel_dft_init(ObitDFTGPUSkyModel *in, const ObitDFTSkyModel *sky,
                               const ObitDFTUVData *uv, ObitDFTErr *err);

/* ObitGPUSkyModelDFTSetMod (ObitGPUSkyModel.h:115, ObitGPUSkyModel.c:416-491):
 * model is the component table (ObitFArray comps), naxis0 floats per component,
 * naxis1 components; trailing zero-flux components are dropped. */
int obit_gpu_skymodel_dft_setmod(ObitDFTGPUSkyModel *in, const ObitDFTSkyModel *sky,
                                 const float *model, int naxis0, int naxis1, ObitDFTErr *err);

/* ObitGPUSkyModelDFTCalc (ObitGPUSkyModel.h:121, ObitGPUSkyModel.c:500-520):
 * applies the model to uv->buffer (uv->numVisBuff records) in place. */
int obit_gpu_skymodel_dft_calc(ObitDFTGPUSkyModel *in, ObitDFTUVData *uv, ObitDFTErr *err);

/* ObitGPUSkyModelDFTShutdown (ObitGPUSkyModel.h:125, ObitGPUSkyModel.c:530-579). */
int obit_gpu_skymodel_dft_shutdown(ObitDFTGPUSkyModel *in, ObitDFTErr *err);

/* Release the instance (ObitGPUSkyModelUnref). */
void obit_gpu_skymodel_unref(ObitDFTGPUSkyModel *in);

/* The GPUInfo this instance drives (for kernel selection / device calls). */
GPUInfo *obit_gpu_skymodel_info(ObitDFTGPUSkyModel *in);

#ifdef __cplusplus
}
#endif
#endif
