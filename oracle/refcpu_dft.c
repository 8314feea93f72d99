/*
 * Test infrastructure only: restatement (B) of the reference CPU DFT, kept
 * faithful to its FP32 rounding points and linked against the reference's own
 * vector math (ObitSinCosVec from ObitSystem/Obit/src/ObitSinCos.c:105-215,
 * ObitExpVec from ObitSystem/Obit/src/ObitExp.c:60-134) compiled from the
 * reference sources by oracle/Makefile into oracle/_ref/libobit_refcpu.so.
 * It is the timed CPU baseline and the "reference's own DFT" for parity on
 * low-phase cases; nothing in the product links it.
 *
 * Base-class types (Point, PointSpec, Gauss, GaussSpec) follow
 * ThreadSkyModelFTDFT, ObitSystem/Obit/src/ObitSkyModel.c:2354-2857:
 *   - u,v,w = (double)u_f32 * fscale_f32; phase summed in double and stored
 *     as FP32 (FazArr, :2504); components in blocks of 100 (FazArrSize, :2379);
 *   - amplitude and exp arguments in FP32, the sum over components in double.
 * TSpec types follow ThreadSkyModelMFFTDFT, ObitSkyModelMF.c:1971-2440:
 *   - u,v,w passed to SkyModel2DDot as FP32 (:1835-1901), phase rounded to FP32;
 *   - blocks of 256 (:1992), per-block sums in FP32 (SkyModelDot, :1795-1822).
 * Rows are split over threads like ObitSkyModelFTDFT (:2298-2327).
 */
#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_dft.h"

/* The reference's vector math (its own sources, built beside this file). */
void ObitSinCosVec(int n, float *angle, float *sin, float *cos);
void ObitExpVec(int n, float *argarr, float *exparr);

/* Link-time stubs for the GLib calls the reference headers declare. */
void g_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  abort();
}
void *g_malloc0(size_t n) { return calloc(1, n); }
void g_free(void *p) { free(p); }
char *g_strdup(const char *s) { return s ? strdup(s) : NULL; }
int g_snprintf(char *s, unsigned long n, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = vsnprintf(s, n, fmt, ap);
  va_end(ap);
  return r;
}

#define BASE_BLOCK 100
#define MF_BLOCK 256

typedef struct {
  const OracleJob *job;
  float *vis;
  int lo, hi;
  int mcomp;
} Slice;

/* Component sum for the base-class types; returns double sums. */
static void base_sum(const OracleJob *j, int mcomp, double u, double v, double w,
                     double lnspec, double *sr, double *si) {
  float AmpArr[BASE_BLOCK], FazArr[BASE_BLOCK], CosArr[BASE_BLOCK], SinArr[BASE_BLOCK];
  float ExpArg[BASE_BLOCK], ExpVal[BASE_BLOCK];
  double sumReal = 0.0, sumImag = 0.0;
  const float *cc = j->comps;
  const float ll = (float)lnspec;
  for (int it = 0; it < mcomp; it += BASE_BLOCK) {
    int itcnt = 0;
    const int lim = (mcomp < it + BASE_BLOCK) ? mcomp : it + BASE_BLOCK;
    for (int ic = it; ic < lim; ic++, cc += j->lcomp, itcnt++) {
      const double tx = cc[1] * u, ty = cc[2] * v, tz = cc[3] * w;
      if (j->modType != ORACLE_POINT && cc[0] == 0.0f) {
        AmpArr[itcnt] = 0.0f;
        FazArr[itcnt] = 0.0f;
        ExpArg[itcnt] = 0.0f;
        continue;
      }
      FazArr[itcnt] = (float)(tx + ty + tz);
      AmpArr[itcnt] = cc[0];
      if (j->modType == ORACLE_POINT_SPEC) {
        float arg = 0.0f, lll = ll;
        for (int t = 0; t < j->nterm; t++) { arg += cc[4 + t] * lll; lll *= ll; }
        ExpArg[itcnt] = arg;
      } else if (j->modType == ORACLE_GAUSS) {
        ExpArg[itcnt] = (float)(cc[4] * u * u + cc[5] * v * v + cc[6] * u * v);
      } else if (j->modType == ORACLE_GAUSS_SPEC) {
        float arg = 0.0f, lll = ll;
        for (int t = 0; t < j->nterm; t++) { arg += cc[7 + t] * lll; lll *= ll; }
        const float specFact = (float)exp(arg);
        AmpArr[itcnt] = specFact * cc[0];
        ExpArg[itcnt] = (float)(cc[4] * u * u + cc[5] * v * v + cc[6] * u * v);
      }
    }
    ObitSinCosVec(itcnt, FazArr, SinArr, CosArr);
    if (j->modType != ORACLE_POINT) ObitExpVec(itcnt, ExpArg, ExpVal);
    for (int jt = 0; jt < itcnt; jt++) {
      float amp = AmpArr[jt];
      if (j->modType != ORACLE_POINT) amp *= ExpVal[jt];
      sumReal += amp * CosArr[jt];
      sumImag += amp * SinArr[jt];
    }
  }
  *sr = sumReal;
  *si = sumImag;
}

/* FP32 dot product as SkyModelDot without AVX-512 (ObitSkyModelMF.c:1795-1822). */
static float dot32(int n, const float *a, const float *b) {
  float o = 0.0f;
  for (int i = 0; i < n; i++) o += a[i] * b[i];
  return o;
}

/* Component sum for the tabulated-spectrum types (MF class). */
static void mf_sum(const OracleJob *j, int mcomp, double ud, double vd, double wd,
                   double lnspec, int plane, double *sr, double *si) {
  float AmpArr[MF_BLOCK], FazArr[MF_BLOCK], CosArr[MF_BLOCK], SinArr[MF_BLOCK];
  float ExpArg[MF_BLOCK], ExpVal[MF_BLOCK], ExpArg2[MF_BLOCK], ExpVal2[MF_BLOCK];
  float VecL[MF_BLOCK], VecM[MF_BLOCK], VecN[MF_BLOCK];
  const float logNuONu0 = (float)lnspec;
  /* SkyModel2DDot takes u, v, w as FP32 scalars */
  const float u = (float)ud, v = (float)vd, w = (float)wd;
  const int gauss = (j->modType == ORACLE_GAUSS_TSPEC);
  const int itab = (gauss ? 8 : 5) + plane;
  double sumReal = 0.0, sumImag = 0.0;
  const float *cc = j->comps;
  for (int it = 0; it < mcomp; it += MF_BLOCK) {
    int itcnt = 0;
    const int lim = (mcomp < it + MF_BLOCK) ? mcomp : it + MF_BLOCK;
    for (int ic = it; ic < lim; ic++, cc += j->lcomp) {
      if (cc[itab] == 0.0f) continue;
      VecL[itcnt] = cc[1];
      VecM[itcnt] = cc[2];
      VecN[itcnt] = cc[3];
      AmpArr[itcnt] = cc[itab];
      if (gauss) {
        ExpArg[itcnt] = (float)(cc[4] * ud * ud + cc[5] * vd * vd + cc[6] * ud * vd);
        ExpArg2[itcnt] = logNuONu0 * cc[7];
      } else {
        ExpArg2[itcnt] = logNuONu0 * cc[4];
      }
      itcnt++;
    }
    for (int i = 0; i < itcnt; i++)
      FazArr[i] = (float)((double)VecL[i] * (double)u + (double)VecM[i] * (double)v +
                          (double)VecN[i] * (double)w);
    ObitSinCosVec(itcnt, FazArr, SinArr, CosArr);
    if (gauss) {
      ObitExpVec(itcnt, ExpArg, ExpVal);
      for (int i = 0; i < itcnt; i++) AmpArr[i] *= ExpVal[i];
    }
    ObitExpVec(itcnt, ExpArg2, ExpVal2);
    for (int i = 0; i < itcnt; i++) AmpArr[i] *= ExpVal2[i];
    sumReal += dot32(itcnt, AmpArr, CosArr);
    sumImag += dot32(itcnt, AmpArr, SinArr);
  }
  *sr = sumReal;
  *si = sumImag;
}

static void *slice_fn(void *arg) {
  Slice *s = (Slice *)arg;
  const OracleJob *j = s->job;
  const int tspec = (j->modType == ORACLE_POINT_TSPEC || j->modType == ORACLE_GAUSS_TSPEC);
  for (int r = s->lo; r < s->hi; r++) {
    float *rec = s->vis + (size_t)r * j->lrec;
    for (int iIF = j->startIF; iIF < j->startIF + j->numberIF; iIF++) {
      const int offIF = j->nrparm + iIF * j->incif;
      for (int ich = j->startChannel; ich < j->startChannel + j->numberChannel; ich++) {
        const int offCh = offIF + ich * j->incf;
        int any = 0;
        for (int p = j->startPoln; p < j->startPoln + j->numberPoln; p++)
          any = any || (rec[offCh + p * j->incs + 2] > 0.0f);
        if (!any && !j->doReplace) continue;
        const int ifq = ich * j->kincf + iIF * j->kincif;
        const float freqFact = j->fscale32[ifq];
        const double u = (double)rec[j->ilocu] * freqFact;
        const double v = (double)rec[j->ilocv] * freqFact;
        const double w = (double)rec[j->ilocw] * freqFact;
        const double L = j->lnspec ? j->lnspec[ifq] : 0.0;
        double sr, si;
        if (tspec)
          mf_sum(j, s->mcomp, u, v, w, L, j->specIndex[ifq], &sr, &si);
        else
          base_sum(j, s->mcomp, u, v, w, L, &sr, &si);
        float modReal = (float)sr, modImag = (float)si, wt = 0.0f;
        int written = 0;
        for (int jp = 0; jp < j->numberPoln; jp++) {
          const int off = offCh + (j->startPoln + jp) * j->incs;
          if (rec[off + 2] <= 0.0f && !j->doReplace) continue;
          float mr = modReal * j->polFact[jp], mi = modImag * j->polFact[jp];
          for (int k = 0; k < written; k++) { mr *= j->stokFactor; mi *= j->stokFactor; }
          if (j->flipMask & (1 << jp)) { const float t = mr; mr = -mi; mi = t; }
          if (j->doDivide) {
            wt = mr * mr + mi * mi;
            mr /= wt;
            mi /= wt;
            wt = sqrtf(wt);
            const float temp = mr * rec[off] + mi * rec[off + 1];
            rec[off + 1] = mr * rec[off + 1] - mi * rec[off];
            rec[off] = temp;
            rec[off + 2] *= wt;
          } else if (j->doReplace) {
            rec[off] = mr;
            rec[off + 1] = mi;
          } else {
            rec[off] -= mr;
            rec[off + 1] -= mi;
          }
          written++;
        }
      }
    }
  }
  return NULL;
}

int refcpu_apply(const OracleJob *j, float *vis, int nthreads) {
  if (j->modType < ORACLE_POINT || j->modType > ORACLE_GAUSS_TSPEC) return -1;
  if (j->nvis <= 0 || j->ncomp <= 0) return 0;
  /* number of components up to the last non-zero flux (ObitSkyModel.c:2411-2416) */
  int mcomp = 0;
  for (int ic = 0; ic < j->ncomp; ic++)
    if (j->comps[(size_t)ic * j->lcomp] != 0.0f) mcomp = ic + 1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > j->nvis) nthreads = j->nvis;
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  Slice *sl = (Slice *)calloc((size_t)nthreads, sizeof(Slice));
  const int per = j->nvis / nthreads;
  for (int t = 0; t < nthreads; t++) {
    sl[t].job = j;
    sl[t].vis = vis;
    sl[t].mcomp = mcomp;
    sl[t].lo = t * per;
    sl[t].hi = (t == nthreads - 1) ? j->nvis : (t + 1) * per;
  }
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, slice_fn, &sl[t]);
  slice_fn(&sl[0]);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
  free(th);
  free(sl);
  return 0;
}
