/*
 * Test infrastructure only: runs the reference's own host glue,
 * ObitSystem/Obit/src/ObitGPUSkyModel.c and ObitSystem/Obit/src/ObitCUDAUtil.cu
 * compiled unmodified, over the four ObitCUDASkyModelDFT* entry points of a
 * CUDA sky-model layer -- this repository's libobit_dft.so (the drop-in), or the
 * reference's own ObitCUDASkyModel.cu (libobit_refgpu.so, the comparator).
 * oracle/Makefile links this file with those sources into
 * _ref/libobit_refglue.so and _ref/libobit_refglue_ref.so.
 *
 * ObitGPUSkyModel.c needs Obit's object system around it.  This file stands in
 * for the few pieces it calls -- the UV open/close pair, the InfoList items it
 * reads and writes (nVisPIO, GPU_no, doCalSelect), the error stack, class
 * membership tests and the GLib helpers -- and builds the objects it reads
 * (ObitUV with its descriptor and selector, ObitSkyModel or ObitSkyModelMF
 * with a one-image mosaic, the component ObitFArray) from the plain arrays of
 * a RefGlueJob, using the reference's own structure definitions.  The driver
 * then follows ObitSkyModel's SubUV loop: Create, DFTInit, DFTSetMod, one
 * DFTCalc per buffer of at most nVisPIO records, DFTShutdown
 * (ObitSkyModel.c:747-760, 811-840, 850-1087, 1485-1492, 793-802).
 *
 * The reference's DFTInit calls ObitCUDAResetGPU (a device synchronize and
 * reset of this process's own context) before it allocates anything, and the
 * reference's CUDA layer resets again at shutdown: run this in a process of its
 * own.  Nothing in the product links or calls this file.
 */
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ObitGPUSkyModel.h"
#include "ObitSkyModelMF.h"
#include "ObitImageMosaic.h"

/* ---- GLib helpers ------------------------------------------------------- */

void g_error(const gchar *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  abort();
}
gpointer g_malloc0(gsize n) { return calloc(1, n ? n : 1); }
void g_free(gpointer p) { free(p); }
gchar *g_strdup(const gchar *s) {
  if (!s) return NULL;
  gchar *o = (gchar *)malloc(strlen(s) + 1);
  strcpy(o, s);
  return o;
}
gchar *g_strconcat(const gchar *s, ...) {
  size_t n = 1;
  va_list ap;
  va_start(ap, s);
  for (const gchar *p = s; p; p = va_arg(ap, const gchar *)) n += strlen(p);
  va_end(ap);
  gchar *o = (gchar *)malloc(n);
  o[0] = 0;
  va_start(ap, s);
  for (const gchar *p = s; p; p = va_arg(ap, const gchar *)) strcat(o, p);
  va_end(ap);
  return o;
}
gint g_snprintf(gchar *s, gulong n, const gchar *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = vsnprintf(s, n, fmt, ap);
  va_end(ap);
  return r;
}

/* ---- Obit object system: only what ObitGPUSkyModel.c calls --------------- */

static ObitClassInfo g_base_class;        /* the Obit base class: no functions */
static ObitClassInfo g_skymodel_mf_class; /* marker of ObitSkyModelMF objects */

gconstpointer ObitGetClass(void) { return &g_base_class; }
gconstpointer ObitSkyModelMFGetClass(void) { return &g_skymodel_mf_class; }
gboolean ObitIsA(gpointer in, gconstpointer type) {
  return in != NULL && ((Obit *)in)->ClassInfo == type;
}

static int g_errors;
void ObitErrPush(ObitErr *in, ObitErrCode errLevel, gchar *errMsg) {
  if (errLevel >= OBIT_Error) {
    g_errors++;
    if (in) in->error = 1;
    fprintf(stderr, "refglue: Obit error: %s\n", errMsg ? errMsg : "");
  }
}
void ObitErrLog(ObitErr *in) { (void)in; }

/* InfoList: one list per UV object here; the glue reads GPU_no, nVisPIO and
 * doCalSelect and writes nVisPIO. */
static olong g_nVisPIO = 0, g_gpu_no = 0, g_have_nvispio = 0;
static int g_buf_records = 0; /* records per DFTCalc buffer of the last run */
void ObitInfoListAlwaysPut(ObitInfoList *in, gchar *name, ObitInfoType type, gint32 *dim,
                           gconstpointer data) {
  (void)in, (void)type, (void)dim;
  if (!strcmp(name, "nVisPIO")) {
    g_nVisPIO = *(const olong *)data;
    g_have_nvispio = 1;
  }
}
gboolean ObitInfoListGetTest(ObitInfoList *in, gchar *name, ObitInfoType *type, gint32 *dim,
                             gpointer data) {
  (void)in, (void)dim;
  if (!strcmp(name, "GPU_no")) {
    *(olong *)data = g_gpu_no;
    if (type) *type = OBIT_long;
    return TRUE;
  }
  if (!strcmp(name, "nVisPIO") && g_have_nvispio) {
    *(olong *)data = g_nVisPIO;
    if (type) *type = OBIT_long;
    return TRUE;
  }
  return FALSE; /* doCalSelect: absent (read-only access) */
}

/* Reopening with a new nVisPIO sizes the I/O buffer to nVisPIO records. */
ObitIOCode ObitUVOpen(ObitUV *in, ObitIOAccess access, ObitErr *err) {
  (void)access, (void)err;
  in->bufferSize = (ollong)g_nVisPIO * in->myDesc->lrec;
  return OBIT_IO_OK;
}
ObitIOCode ObitUVClose(ObitUV *in, ObitErr *err) {
  (void)in, (void)err;
  return OBIT_IO_OK;
}

/* ---- the job ------------------------------------------------------------- */

/* Records in the Obit layout (nrparm random parameters, then the regular axes
 * COMPLEX, STOKES, FREQ, IF), the component table and the sky-model settings
 * that ObitGPUSkyModel.c reads. */
typedef struct {
  int nvis, lrec, nrparm, ilocu, ilocv, ilocw;
  int nstok, nchan, nif;     /* axes STOKES, FREQ, IF in that order */
  double crvalStokes;        /* -1: RR, LL, RL, LR */
  double uvFreq;             /* desc->freq */
  const float *fscale;       /* nchan*nif, channel-major within IF (kincf 1, kincif nchan) */
  int startChann, numberChann, startIF, numberIF; /* selection, 1-relative */
  int modType;               /* ObitSkyModelCompType */
  int nSpecTerm;
  float factor;
  int doDivide, doReplace, doFlip;
  double imageFreq;          /* CRVAL of the image's frequency axis (> 0: a mosaic is set) */
  int isMF;                  /* an ObitSkyModelMF: tabulated spectra */
  int nSpec;
  const double *specFreq;    /* nSpec coarse-plane frequencies */
  const int *specIndex;      /* nchan*nif coarse plane per (channel, IF) */
  const float *comps;        /* ncomp rows of lcomp floats (the model ObitFArray) */
  int ncomp, lcomp;
  int gpu;                   /* GPU_no */
  int nVisPIO;               /* records per DFTCalc buffer (the glue caps it at 10000) */
  float *vis;                /* nvis records, modified in place */
} RefGlueJob;

int refglue_run(const RefGlueJob *j) {
  g_errors = 0;
  g_buf_records = 0;
  g_gpu_no = j->gpu;
  g_nVisPIO = j->nVisPIO > 0 ? j->nVisPIO : j->nvis;
  g_have_nvispio = 1;

  ObitErr err;
  memset(&err, 0, sizeof(err));

  ObitUVDesc desc;
  memset(&desc, 0, sizeof(desc));
  desc.nvis = j->nvis;
  desc.lrec = j->lrec;
  desc.nrparm = j->nrparm;
  desc.ilocu = j->ilocu;
  desc.ilocv = j->ilocv;
  desc.ilocw = j->ilocw;
  desc.iloct = desc.ilocb = desc.ilocsu = -1;
  desc.jlocs = 1;
  desc.jlocf = 2;
  desc.jlocif = 3;
  desc.inaxes[0] = 3;
  desc.inaxes[1] = j->nstok;
  desc.inaxes[2] = j->nchan;
  desc.inaxes[3] = j->nif;
  desc.crval[1] = j->crvalStokes;
  desc.incs = 3;
  desc.incf = 3 * j->nstok;
  desc.incif = 3 * j->nstok * j->nchan;
  desc.ncorr = j->nstok * j->nchan * j->nif;
  desc.freq = j->uvFreq;
  desc.fscale = (ofloat *)j->fscale;

  ObitUVSel sel;
  memset(&sel, 0, sizeof(sel));
  sel.startChann = j->startChann;
  sel.numberChann = j->numberChann;
  sel.startIF = j->startIF;
  sel.numberIF = j->numberIF;

  static char info_dummy[64];
  ObitUV uv;
  memset(&uv, 0, sizeof(uv));
  uv.myDesc = &desc;
  uv.mySel = &sel;
  uv.info = (ObitInfoList *)info_dummy;
  uv.name = "refglue";

  ObitImageDesc imDesc;
  memset(&imDesc, 0, sizeof(imDesc));
  imDesc.jlocf = 2;
  imDesc.crval[2] = j->imageFreq;
  ObitImage image;
  memset(&image, 0, sizeof(image));
  image.myDesc = &imDesc;
  ObitImage *images[1] = {&image};
  ObitImageMosaic mosaic;
  memset(&mosaic, 0, sizeof(mosaic));
  mosaic.numberImages = 1;
  mosaic.images = images;

  ObitSkyModelMF skyMF; /* a superset of ObitSkyModel */
  memset(&skyMF, 0, sizeof(skyMF));
  ObitSkyModel *sky = (ObitSkyModel *)&skyMF;
  sky->ClassInfo = j->isMF ? (gpointer)&g_skymodel_mf_class : (gpointer)&g_base_class;
  sky->mosaic = j->imageFreq > 0.0 ? &mosaic : NULL;
  sky->modType = (ObitSkyModelCompType)j->modType;
  sky->nSpecTerm = j->nSpecTerm;
  sky->factor = j->factor;
  sky->doDivide = j->doDivide;
  sky->doReplace = j->doReplace;
  sky->doFlip = j->doFlip;
  olong *specIndex = NULL;
  if (j->isMF) {
    skyMF.nSpec = j->nSpec;
    skyMF.specFreq = (odouble *)j->specFreq;
    specIndex = (olong *)calloc((size_t)j->nchan * j->nif, sizeof(olong));
    for (int i = 0; i < j->nchan * j->nif; i++) specIndex[i] = j->specIndex[i];
    skyMF.specIndex = specIndex;
  }

  olong naxis[2] = {j->lcomp, j->ncomp};
  ObitFArray model;
  memset(&model, 0, sizeof(model));
  model.ndim = 2;
  model.naxis = naxis;
  model.arraySize = j->lcomp * j->ncomp;
  model.array = (ofloat *)j->comps;

  ObitGPUSkyModel *gm = ObitGPUSkyModelCreate("refglue", "DFT");
  ObitGPUSkyModelDFTInit(gm, (Obit *)sky, &uv, &err);
  if (!err.error) ObitGPUSkyModelDFTSetMod(gm, (Obit *)sky, &model, &err);
  /* SubUV: one DFTCalc per I/O buffer of at most nVisPIO records */
  const int per = (int)(uv.bufferSize / j->lrec);
  g_buf_records = per;
  for (int r0 = 0; !err.error && per > 0 && r0 < j->nvis; r0 += per) {
    const int n = (j->nvis - r0 < per) ? j->nvis - r0 : per;
    desc.numVisBuff = n;
    uv.buffer = j->vis + (size_t)r0 * j->lrec;
    ObitGPUSkyModelDFTCalc(gm, &uv, &err);
  }
  ObitGPUSkyModelDFTShutdown(gm, &uv, &err);
  free(gm->gpuInfo);
  free(gm->name);
  free(gm);
  free(specIndex);
  return (err.error || g_errors) ? 1 : 0;
}

/* Records per DFTCalc buffer of the last run: the nVisPIO the glue chose at
 * DFTInit (its DFTShutdown puts the caller's old value back into the list). */
int refglue_nvispio(void) { return g_buf_records; }
