/*
 * Host-side mirror of ObitGPUSkyModel.c (DFT path) in C; see
 * include/obit_gpu_skymodel.h for the interface and the deliberate
 * differences from the reference.
 */
#include "obit_gpu_skymodel.h"

#include <cuda_runtime_api.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NSTREAM 4 /* STREAM_COUNT, ObitCUDASkyModelInfoDef.h:30 */

struct ObitDFTGPUSkyModel {
  char name[64];
  GPUInfo *gpuInfo;
  int nfreq;
};

static int set_err(ObitDFTErr *err, const char *routine, const char *fmt, ...) {
  if (err) {
    char buf[400];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err->error = 1;
    snprintf(err->message, sizeof(err->message), "%s: %s", routine, buf);
  }
  return 1;
}

#define CU(call, routine)                                                                   \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return set_err(err, routine, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define DFT(call, routine)                                                     \
  do {                                                                         \
    int r_ = (call);                                                           \
    if (r_) return set_err(err, routine, "%s: %s", #call, obit_dft_last_error()); \
  } while (0)

/* ObitSkyModelCompType -> GPUModType (ObitGPUSkyModel.c:445-458). */
static int gpu_mod_type(int modType) {
  switch (modType) {
    case 0: return GPUModTypePoint;
    case 10: return GPUModTypePointSpec;
    case 20: return GPUModTypePointTSpec;
    case 1: return GPUModTypeGauss;
    case 11: return GPUModTypeGaussSpec;
    case 21: return GPUModTypeGaussTSpec;
    default: return -1;
  }
}

ObitDFTGPUSkyModel *obit_gpu_skymodel_create(const char *name) {
  ObitDFTGPUSkyModel *in = (ObitDFTGPUSkyModel *)calloc(1, sizeof(ObitDFTGPUSkyModel));
  if (!in) return NULL;
  snprintf(in->name, sizeof(in->name), "%s", name ? name : "GPUSkyModel");
  in->gpuInfo = (GPUInfo *)calloc(1, sizeof(GPUInfo));
  if (!in->gpuInfo) {
    free(in);
    return NULL;
  }
  return in;
}

GPUInfo *obit_gpu_skymodel_info(ObitDFTGPUSkyModel *in) { return in ? in->gpuInfo : NULL; }

int obit_gpu_skymodel_dft_init(ObitDFTGPUSkyModel *in, const ObitDFTSkyModel *sky,
                               const ObitDFTUVData *uv, ObitDFTErr *err) {
  const char *routine = "obit_gpu_skymodel_dft_init";
  if (err && err->error) return 1;
  if (!in || !in->gpuInfo || !sky || !uv) return set_err(err, routine, "NULL argument");
  GPUInfo *g = in->gpuInfo;
  if (uv->jlocf < 0 || uv->jlocs < 0 || uv->lrec <= 0 || uv->nrparm < 3)
    return set_err(err, routine, "uv descriptor lacks frequency/Stokes axes or u,v,w");
  if (!uv->fscale) return set_err(err, routine, "uv descriptor has no frequency scaling table");
  g->cuda_device = sky->GPU_no;
  CU(cudaSetDevice(g->cuda_device), routine);
  g->prtLv = err ? err->prtLv : 0;

  const int nchan = uv->inaxes[uv->jlocf];
  const int nif = (uv->jlocif >= 0) ? uv->inaxes[uv->jlocif] : 1;
  const int nstok = uv->inaxes[uv->jlocs];
  int nVisPIO = sky->nVisPIO > 0 ? sky->nVisPIO : 10000; /* ObitGPUSkyModel.c:236 */
  if (nVisPIO > uv->nvis) nVisPIO = uv->nvis;
  if (nVisPIO < 1) nVisPIO = 1;
  in->nfreq = nchan * nif;

  g->bufferSize = nVisPIO * uv->lrec;
  CU(cudaMallocHost((void **)&g->h_data, sizeof(float) * (size_t)g->bufferSize), routine);
  g->nvis = nVisPIO;
  g->nchan = nchan;
  g->nrparm = uv->nrparm;
  g->lenvis = uv->lrec;
  g->nstream = NSTREAM;

  CU(cudaMalloc((void **)&g->d_freq, sizeof(float) * (size_t)in->nfreq), routine);
  CU(cudaMemcpy(g->d_freq, uv->fscale, sizeof(float) * (size_t)in->nfreq, cudaMemcpyHostToDevice),
     routine);

  int kincf = 1, kincif = 1; /* ObitGPUSkyModel.c:263-275 */
  if (uv->jlocif >= 0) {
    if (uv->jlocf < uv->jlocif) {
      kincf = 1;
      kincif = nchan;
    } else {
      kincif = 1;
      kincf = nif;
    }
  }
  GPUVisInfo *v;
  CU(cudaMallocHost((void **)&g->h_visInfo, sizeof(GPUVisInfo)), routine);
  CU(cudaMalloc((void **)&g->d_visInfo, sizeof(GPUVisInfo)), routine);
  v = g->h_visInfo;
  memset(v, 0, sizeof(*v));
  v->freqScale = g->d_freq;
  v->nvis = g->nvis;
  v->nprod = uv->ncorr;
  v->nrparm = uv->nrparm;
  v->lenvis = uv->lrec;
  v->nchan = nchan;
  v->ilocu = uv->ilocu;
  v->ilocv = uv->ilocv;
  v->ilocw = uv->ilocw;
  v->iloct = v->ilocb = v->ilocsu = -1;
  v->chanb = sky->startChannelPB - 1;
  v->chane = sky->startChannelPB + (sky->numberChannelPB > 0 ? sky->numberChannelPB : 1) - 2;
  v->incf = uv->incf / 3;
  v->nIF = nif;
  v->IFb = sky->startIFPB - 1;
  v->IFe = sky->startIFPB + (sky->numberIFPB > 0 ? sky->numberIFPB : 1) - 2;
  v->incif = uv->incif / 3;
  v->nstok = nstok;
  v->stokb = sky->startPoln - 1;
  v->stoke = v->stokb + (sky->numberPoln > 0 ? sky->numberPoln : 1) - 1;
  v->incs = uv->incs / 3;
  v->kincif = kincif;
  v->kincf = kincf;
  v->stype = (uv->crvalStokes > 0.0) ? 0 : ((uv->crvalStokes < -4.0) ? 2 : 1);
  /* frequency ratios: per coarse plane for tabulated spectra, else one
   * (ObitGPUSkyModel.c:314-343) */
  const int nrat = sky->isMF ? (sky->nSpec > 0 ? sky->nSpec : 1) : 1;
  CU(cudaMallocHost((void **)&v->freqRat, sizeof(float) * (size_t)nrat), routine);
  if (sky->isMF) {
    for (int i = 0; i < nrat; i++)
      v->freqRat[i] = (sky->specFreq && sky->specFreq[i] > 0) ? (float)(uv->freq / sky->specFreq[i]) : 1.0f;
  } else {
    v->freqRat[0] = (sky->modelRefFreq > 0.0) ? (float)(uv->freq / sky->modelRefFreq) : 1.0f;
  }
  CU(cudaMalloc((void **)&v->d_freqRat, sizeof(float) * (size_t)nrat), routine);
  CU(cudaMemcpy(v->d_freqRat, v->freqRat, sizeof(float) * (size_t)nrat, cudaMemcpyHostToDevice), routine);
  CU(cudaMemcpy(g->d_visInfo, v, sizeof(GPUVisInfo), cudaMemcpyHostToDevice), routine);

  GPUModelInfo *m;
  CU(cudaMallocHost((void **)&g->h_modelInfo, sizeof(GPUModelInfo)), routine);
  CU(cudaMalloc((void **)&g->d_modelInfo, sizeof(GPUModelInfo)), routine);
  m = g->h_modelInfo;
  memset(m, 0, sizeof(*m));
  m->nterm = sky->nSpecTerm;
  m->size = g->modelSize;
  m->type = GPUModTypePoint; /* set for real in SetMod */
  if (sky->isMF) {
    if (!sky->specIndex) return set_err(err, routine, "tabulated spectra need specIndex");
    CU(cudaMallocHost((void **)&m->specIndex, sizeof(int) * (size_t)in->nfreq), routine);
    memcpy(m->specIndex, sky->specIndex, sizeof(int) * (size_t)in->nfreq);
    CU(cudaMalloc((void **)&m->d_specIndex, sizeof(int) * (size_t)in->nfreq), routine);
    CU(cudaMemcpy(m->d_specIndex, m->specIndex, sizeof(int) * (size_t)in->nfreq, cudaMemcpyHostToDevice),
       routine);
  }

  /* per-stream device buffers, (nvis+3)*lenvis/nstream floats each
   * (ObitGPUSkyModel.c:383-389) */
  g->d_data = (float **)calloc(NSTREAM, sizeof(float *));
  const size_t per = sizeof(float) * ((size_t)(g->nvis + 3) * g->lenvis / NSTREAM);
  for (int i = 0; i < NSTREAM; i++) CU(cudaMalloc((void **)&g->d_data[i], per), routine);
  g->stream = (void **)calloc(NSTREAM, sizeof(void *));
  g->cycleDone = (void **)calloc(NSTREAM, sizeof(void *));
  for (int i = 0; i < NSTREAM; i++) {
    cudaStream_t st;
    cudaEvent_t ev;
    CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), routine);
    CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), routine);
    g->stream[i] = (void *)st;
    g->cycleDone[i] = (void *)ev;
  }

  DFT(obit_dft_init(g), routine);
  if (uv->freqArr) {
    double mref = sky->modelRefFreq > 0.0 ? sky->modelRefFreq : uv->freq;
    DFT(obit_dft_set_freq(g, uv->freqArr, in->nfreq, uv->freq, mref, sky->isMF ? sky->specFreq : NULL,
                          sky->isMF ? sky->nSpec : 0),
        routine);
  }
  DFT(obit_dft_set_poln(g, 1, sky->stokFactor, sky->doFlip), routine);
  return 0;
}

int obit_gpu_skymodel_dft_setmod(ObitDFTGPUSkyModel *in, const ObitDFTSkyModel *sky,
                                 const float *model, int naxis0, int naxis1, ObitDFTErr *err) {
  const char *routine = "obit_gpu_skymodel_dft_setmod";
  if (err && err->error) return 1;
  if (!in || !in->gpuInfo || !in->gpuInfo->h_modelInfo || !sky)
    return set_err(err, routine, "instance not initialized");
  if (naxis0 <= 0 || naxis1 < 0 || (naxis1 > 0 && !model))
    return set_err(err, routine, "bad component table %d x %d", naxis0, naxis1);
  GPUInfo *g = in->gpuInfo;
  const int type = gpu_mod_type(sky->modType);
  if (type < 0) return set_err(err, routine, "Model type not supported in GPU %d", sky->modType);
  /* last non-zero flux entry (ObitGPUSkyModel.c:422-425) */
  int high = 0;
  for (int i = 0; i < naxis1; i++)
    if (model[(size_t)i * naxis0] != 0.0f) high = i + 1;
  if (err && err->prtLv > 0) fprintf(stderr, "SkyModel by GPU with %d components\n", high);
  if (g->nmodel[0] != high || g->modelSize != naxis0 || !g->d_model[0]) {
    if (g->d_model[0]) cudaFree(g->d_model[0]);
    g->d_model[0] = NULL;
    const size_t bytes = sizeof(float) * (size_t)(high > 0 ? high : 1) * naxis0;
    CU(cudaMalloc((void **)&g->d_model[0], bytes), routine);
    for (int i = 0; i < 4; i++) g->nmodel[i] = high;
    g->d_model[1] = g->d_model[2] = g->d_model[3] = g->d_model[0];
    g->modelSize = naxis0;
  }
  GPUModelInfo *m = g->h_modelInfo;
  m->nterm = sky->nSpecTerm;
  for (int i = 0; i < 4; i++) {
    m->model[i] = g->d_model[0];
    m->nmodel[i] = high;
    m->stokFact[i] = 1.0f; /* factor is already in the table */
  }
  m->type = (GPUModType)type;
  m->opType = GPUOpTypeSub;
  if (sky->doDivide) m->opType = GPUOpTypeDiv;
  if (sky->doReplace) m->opType = GPUOpTypeRepl;
  m->doSwap = sky->doFlip ? 1 : 0;
  m->size = naxis0;
  if (high > 0)
    CU(cudaMemcpy(g->d_model[0], model, sizeof(float) * (size_t)high * naxis0, cudaMemcpyHostToDevice),
       routine);
  CU(cudaMemcpy(g->d_modelInfo, m, sizeof(GPUModelInfo), cudaMemcpyHostToDevice), routine);
  DFT(obit_dft_set_mod(g), routine);
  return 0;
}

int obit_gpu_skymodel_dft_calc(ObitDFTGPUSkyModel *in, ObitDFTUVData *uv, ObitDFTErr *err) {
  const char *routine = "obit_gpu_skymodel_dft_calc";
  if (err && err->error) return 1;
  if (!in || !in->gpuInfo || !in->gpuInfo->h_data || !uv) return set_err(err, routine, "not initialized");
  GPUInfo *g = in->gpuInfo;
  const int nvis = uv->numVisBuff;
  if (nvis < 0) return set_err(err, routine, "negative buffer count");
  if ((long long)nvis * g->lenvis > (long long)g->bufferSize)
    return set_err(err, routine, "buffer of %d records exceeds nVisPIO %d", nvis, g->bufferSize / g->lenvis);
  if (nvis == 0) return 0;
  if (!uv->buffer) return set_err(err, routine, "uv buffer is NULL");
  g->nvis = nvis;
  g->h_visInfo->nvis = nvis;
  g->h_visInfo->nprod = uv->ncorr;
  const size_t bytes = sizeof(float) * (size_t)nvis * g->lenvis;
  memcpy(g->h_data, uv->buffer, bytes); /* ObitGPUSkyModel.c:511 */
  DFT(obit_dft_calc(g), routine);
  memcpy(uv->buffer, g->h_data, bytes); /* ObitGPUSkyModel.c:517 */
  return 0;
}

int obit_gpu_skymodel_dft_shutdown(ObitDFTGPUSkyModel *in, ObitDFTErr *err) {
  const char *routine = "obit_gpu_skymodel_dft_shutdown";
  if (!in || !in->gpuInfo) return 0;
  GPUInfo *g = in->gpuInfo;
  int rc = obit_dft_shutdown(g);
  if (g->h_data) cudaFreeHost(g->h_data);
  if (g->h_visInfo) {
    if (g->h_visInfo->d_freqRat) cudaFree(g->h_visInfo->d_freqRat);
    if (g->h_visInfo->freqRat) cudaFreeHost(g->h_visInfo->freqRat);
    cudaFreeHost(g->h_visInfo);
  }
  if (g->d_visInfo) cudaFree(g->d_visInfo);
  if (g->h_modelInfo) {
    if (g->h_modelInfo->d_specIndex) cudaFree(g->h_modelInfo->d_specIndex);
    if (g->h_modelInfo->specIndex) cudaFreeHost(g->h_modelInfo->specIndex);
    cudaFreeHost(g->h_modelInfo);
  }
  if (g->d_modelInfo) cudaFree(g->d_modelInfo);
  if (g->d_model[0]) cudaFree(g->d_model[0]);
  if (g->d_freq) cudaFree(g->d_freq);
  for (int i = 0; i < NSTREAM; i++) {
    if (g->stream && g->stream[i]) cudaStreamDestroy((cudaStream_t)g->stream[i]);
    if (g->cycleDone && g->cycleDone[i]) cudaEventDestroy((cudaEvent_t)g->cycleDone[i]);
    if (g->d_data && g->d_data[i]) cudaFree(g->d_data[i]);
  }
  free(g->stream);
  free(g->cycleDone);
  free(g->d_data);
  memset(g, 0, sizeof(*g));
  if (rc) return set_err(err, routine, "%s", obit_dft_last_error());
  return 0;
}

void obit_gpu_skymodel_unref(ObitDFTGPUSkyModel *in) {
  if (!in) return;
  if (in->gpuInfo && in->gpuInfo->h_data) obit_gpu_skymodel_dft_shutdown(in, NULL);
  free(in->gpuInfo);
  free(in);
}
