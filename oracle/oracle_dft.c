/*
 * Test infrastructure only: FP64 oracle (A) for the Obit DFT sky-model
 * predict / subtract.  Nothing in the product links or calls this file; tests,
 * the smoke check and bench.py's CPU-baseline leg use it as the checker.
 *
 * Semantics follow the reference CPU DFT:
 *   ThreadSkyModelFTDFT    ObitSystem/Obit/src/ObitSkyModel.c:2354-2857
 *   ThreadSkyModelMFFTDFT  ObitSystem/Obit/src/ObitSkyModelMF.c:1971-2440
 * with every FP32 input promoted to double and phase, sin/cos, exp and the
 * component sum evaluated in FP64 (libm).  Per-type amplitude rules:
 *   Point      amp = A                                  (ObitSkyModel.c:2493-2520)
 *   PointSpec  amp = A exp(+sum_t a_t L^(t+1))          (ObitSkyModel.c:2521-2556)
 *   Gauss      amp = A exp(g1 u^2 + g2 v^2 + g3 u v)     (ObitSkyModel.c:2557-2593)
 *   GaussSpec  Gauss x exp(+sum_t a_t L^(t+1))           (ObitSkyModel.c:2594-2635)
 *   PointTSpec amp = tab[plane] exp(+alpha L_plane)      (ObitSkyModelMF.c:2141-2173)
 *   GaussTSpec Gauss x tab[plane] exp(+alpha L_plane)    (ObitSkyModelMF.c:2203-2240)
 * where u,v,w are the record's (u,v,w) times the channel's frequency ratio and
 * phase = X u + Y v + Z w.  The spectral sign is the CPU one (S ~ nu^+alpha);
 * the Gaussian exponent is the base-class +arg with negative coefficients.
 *
 * Application per (row, channel, IF) follows ObitSkyModel.c:2787-2849:
 * a row/channel with no selected polarization of positive weight is skipped
 * unless replacing; a flagged polarization is skipped (and does not advance
 * the stokFactor product) unless replacing.
 */
#include "oracle_dft.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  const OracleJob *job;
  const float *vis_in;
  float *vis_out;
  double *model;
  double *l1;
  int lo, hi;
  int status;
} Slice;

static int type_ok(int t) { return t >= ORACLE_POINT && t <= ORACLE_GAUSS_TSPEC; }

void oracle_comp_term(const OracleJob *j, int ic, double u, double v, double w, double L, int plane,
                      double *amp_out, double *ph_out) {
  const float *c = j->comps + (size_t)ic * j->lcomp;
  double amp, expo = 0.0;
  switch (j->modType) {
    case ORACLE_POINT:
      amp = c[0];
      break;
    case ORACLE_POINT_SPEC: {
      double p = L;
      for (int t = 0; t < j->nterm; t++) { expo += (double)c[4 + t] * p; p *= L; }
      amp = c[0];
      break;
    }
    case ORACLE_POINT_TSPEC:
      amp = c[5 + plane];
      expo = (double)c[4] * L;
      break;
    case ORACLE_GAUSS:
      amp = c[0];
      expo = (double)c[4] * u * u + (double)c[5] * v * v + (double)c[6] * u * v;
      break;
    case ORACLE_GAUSS_SPEC: {
      double p = L;
      expo = (double)c[4] * u * u + (double)c[5] * v * v + (double)c[6] * u * v;
      for (int t = 0; t < j->nterm; t++) { expo += (double)c[7 + t] * p; p *= L; }
      amp = c[0];
      break;
    }
    default: /* ORACLE_GAUSS_TSPEC */
      amp = c[8 + plane];
      expo = (double)c[4] * u * u + (double)c[5] * v * v + (double)c[6] * u * v +
             (double)c[7] * L;
      break;
  }
  if (expo != 0.0) amp *= exp(expo);
  const double *x = j->xyz ? j->xyz + 3 * (size_t)ic : NULL;
  *ph_out = x ? x[0] * u + x[1] * v + x[2] * w
              : (double)c[1] * u + (double)c[2] * v + (double)c[3] * w;
  *amp_out = amp;
}

/* Raw component sum for one record at one (channel, IF) table index. */
static void comp_sum(const OracleJob *j, const float *rec, int ifq, double *sr,
                     double *si, double *l1) {
  const double f = j->fscale[ifq];
  const double u = (double)rec[j->ilocu] * f;
  const double v = (double)rec[j->ilocv] * f;
  const double w = (double)rec[j->ilocw] * f;
  const double L = j->lnspec ? j->lnspec[ifq] : 0.0;
  const int plane = j->specIndex ? j->specIndex[ifq] : 0;
  double accr = 0.0, acci = 0.0, accl = 0.0;
  for (int ic = 0; ic < j->ncomp; ic++) {
    double amp, ph;
    oracle_comp_term(j, ic, u, v, w, L, plane, &amp, &ph);
    accr += amp * cos(ph);
    acci += amp * sin(ph);
    accl += fabs(amp);
  }
  *sr = accr;
  *si = acci;
  *l1 = accl;
}

static void *model_slice(void *arg) {
  Slice *s = (Slice *)arg;
  const OracleJob *j = s->job;
  const int nfreq = j->nchan * j->nif;
  for (int r = s->lo; r < s->hi; r++) {
    const float *rec = s->vis_in + (size_t)r * j->lrec;
    for (int iIF = j->startIF; iIF < j->startIF + j->numberIF; iIF++)
      for (int ich = j->startChannel; ich < j->startChannel + j->numberChannel; ich++) {
        const int ifq = ich * j->kincf + iIF * j->kincif;
        double sr, si, l1;
        comp_sum(j, rec, ifq, &sr, &si, &l1);
        const size_t o = (size_t)r * nfreq + ifq;
        s->model[2 * o] = sr;
        s->model[2 * o + 1] = si;
        if (s->l1) s->l1[o] = l1;
      }
  }
  return NULL;
}

static void *apply_slice(void *arg) {
  Slice *s = (Slice *)arg;
  const OracleJob *j = s->job;
  for (int r = s->lo; r < s->hi; r++) {
    float *rec = s->vis_out + (size_t)r * j->lrec;
    for (int iIF = j->startIF; iIF < j->startIF + j->numberIF; iIF++) {
      const int offIF = j->nrparm + iIF * j->incif;
      for (int ich = j->startChannel; ich < j->startChannel + j->numberChannel; ich++) {
        const int offCh = offIF + ich * j->incf;
        int any = 0;
        for (int p = j->startPoln; p < j->startPoln + j->numberPoln; p++)
          any = any || (rec[offCh + p * j->incs + 2] > 0.0f);
        if (!any && !j->doReplace) continue;
        const int ifq = ich * j->kincf + iIF * j->kincif;
        double sr, si, l1;
        comp_sum(j, rec, ifq, &sr, &si, &l1);
        double cum = 1.0;
        for (int jp = 0; jp < j->numberPoln; jp++) {
          const int off = offCh + (j->startPoln + jp) * j->incs;
          if (rec[off + 2] <= 0.0f && !j->doReplace) continue;
          const double fac = cum * (double)j->polFact[jp];
          double mr = fac * sr, mi = fac * si;
          if (j->flipMask & (1 << jp)) { const double t = mr; mr = -mi; mi = t; }
          if (j->doDivide) {
            const double a2 = mr * mr + mi * mi;
            const double dr = mr / a2, di = mi / a2;
            const double vr = rec[off], vi = rec[off + 1];
            rec[off] = (float)(dr * vr + di * vi);
            rec[off + 1] = (float)(dr * vi - di * vr);
            rec[off + 2] = (float)((double)rec[off + 2] * sqrt(a2));
          } else if (j->doReplace) {
            rec[off] = (float)mr;
            rec[off + 1] = (float)mi;
          } else {
            rec[off] = (float)((double)rec[off] - mr);
            rec[off + 1] = (float)((double)rec[off + 1] - mi);
          }
          cum *= (double)j->stokFactor;
        }
      }
    }
  }
  return NULL;
}

/* Split rows over threads the way ObitSkyModelFTDFT does
 * (ObitSkyModel.c:2298-2327): nvis/nThreads rows each, the last takes the rest. */
static int run_sliced(const OracleJob *j, const float *vin, float *vout,
                      double *model, double *l1, int nthreads,
                      void *(*fn)(void *)) {
  if (!type_ok(j->modType)) return -1;
  if (j->nvis <= 0 || j->ncomp <= 0) return 0;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > j->nvis) nthreads = j->nvis;
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  Slice *sl = (Slice *)calloc((size_t)nthreads, sizeof(Slice));
  const int per = j->nvis / nthreads;
  for (int t = 0; t < nthreads; t++) {
    sl[t].job = j;
    sl[t].vis_in = vin;
    sl[t].vis_out = vout;
    sl[t].model = model;
    sl[t].l1 = l1;
    sl[t].lo = t * per;
    sl[t].hi = (t == nthreads - 1) ? j->nvis : (t + 1) * per;
  }
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, fn, &sl[t]);
  fn(&sl[0]);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
  free(th);
  free(sl);
  return 0;
}

int oracle_model_fp64(const OracleJob *j, const float *vis, double *model,
                      double *l1, int nthreads) {
  return run_sliced(j, vis, NULL, model, l1, nthreads, model_slice);
}

int oracle_apply_fp64(const OracleJob *j, float *vis, int nthreads) {
  return run_sliced(j, vis, vis, NULL, NULL, nthreads, apply_slice);
}
