/* Test infrastructure (never linked into the product): FP64 oracle of the
 * beam-corrected DFT, the model of ObitCUDABeamModel's beam*Kernel family
 * (ObitSystem/Obit/src/ObitCUDABeamModel.cu:139-1226) for a Stokes I sky and
 * linear feeds.
 *
 * For a record of baseline (a1, a2) with antenna types t1, t2 and a (channel,
 * IF) whose Jones plane is jc, each component contributes v = amp e^{i phase}
 * (amplitude and phase as in the DFT oracle, oracle_comp_term) times the
 * coefficients of cudaJonesCor1_Lin_I (ObitSystem/Obit/include/CUDALinCorSum.h:104-134),
 * with J1 = Jones[t1][c][jc], J2 = Jones[t2][c][jc] and P(i, j) = J1[i] conj(J2[j]):
 *   XX: P(0,0) + P(1,1)   XY: P(1,3) + P(0,2)   YX: P(2,0) + P(3,1)   YY: P(2,2) + P(3,3)
 * Antenna numbers come from the BASELINE random parameter (256 a1 + a2, plus a
 * subarray fraction) or from ANTENNA1/ANTENNA2, as GetAnts does
 * (ObitCUDABeamModel.cu:82-99).  The records hold XX, YY, XY, YX; each modelled
 * correlation with positive weight (any, when replacing) is subtracted from,
 * divided into (weight unchanged) or replaced by its model times polFact[p];
 * correlations are applied independently.  Every (channel, IF) of the job's
 * selection is processed, for every IF (the reference kernel's product index
 * stops at the first IF's channels). */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>

#include "oracle_dft.h"

typedef struct {
  const OracleJob *job;
  const OracleBeam *beam;
  float *vis;
  double *l1;
  int lo, hi;
} BeamSlice;

static int beam_ants(const OracleBeam *b, const float *rec, int *a1, int *a2) {
  if (b->ilocb >= 0) {
    const double cbase = rec[b->ilocb];
    *a1 = (int)(cbase / 256.0 + 0.001);
    *a2 = (int)(cbase - (double)(*a1) * 256.0 + 0.001);
  } else {
    *a1 = (int)(rec[b->iloca1] + 0.5);
    *a2 = (int)(rec[b->iloca2] + 0.5);
  }
  *a1 -= 1;
  *a2 -= 1;
  return *a1 >= 0 && *a1 < b->numAnt && *a2 >= 0 && *a2 < b->numAnt;
}

/* model correlation (0 XX, 1 XY, 2 YX, 3 YY) of record polarization p (XX, YY, XY, YX) */
static const int kModelOf[4] = {0, 3, 1, 2};

static void *beam_slice(void *arg) {
  BeamSlice *s = (BeamSlice *)arg;
  const OracleJob *j = s->job;
  const OracleBeam *b = s->beam;
  const int nfreq = j->nchan * j->nif;
  const int ncorr = j->numberPoln;
  for (int r = s->lo; r < s->hi; r++) {
    float *rec = s->vis + (size_t)r * j->lrec;
    int a1, a2;
    if (!beam_ants(b, rec, &a1, &a2)) continue;
    const int t1 = b->antType[a1], t2 = b->antType[a2];
    for (int iIF = j->startIF; iIF < j->startIF + j->numberIF; iIF++) {
      const int offIF = j->nrparm + iIF * j->incif;
      for (int ich = j->startChannel; ich < j->startChannel + j->numberChannel; ich++) {
        const int offCh = offIF + ich * j->incf;
        const int ifq = ich * j->kincf + iIF * j->kincif;
        const int jc = b->jchan[ifq];
        const double f = j->fscale[ifq];
        const double u = (double)rec[j->ilocu] * f;
        const double v = (double)rec[j->ilocv] * f;
        const double w = (double)rec[j->ilocw] * f;
        const double L = j->lnspec ? j->lnspec[ifq] : 0.0;
        const int plane = j->specIndex ? j->specIndex[ifq] : 0;
        double mr[4] = {0, 0, 0, 0}, mi[4] = {0, 0, 0, 0}, ml[4] = {0, 0, 0, 0};
        for (int ic = 0; ic < j->ncomp; ic++) {
          double amp, ph;
          oracle_comp_term(j, ic, u, v, w, L, plane, &amp, &ph);
          const double vr = amp * cos(ph), vi = amp * sin(ph);
          const float *J1 = b->jones + (((size_t)t1 * j->ncomp + ic) * b->numJChan + jc) * 8;
          const float *J2 = b->jones + (((size_t)t2 * j->ncomp + ic) * b->numJChan + jc) * 8;
          /* P(x, y) = J1[x] conj(J2[y]) */
#define PR(x, y) ((double)J1[2 * (x)] * J2[2 * (y)] + (double)J1[2 * (x) + 1] * J2[2 * (y) + 1])
#define PI(x, y) ((double)J1[2 * (x) + 1] * J2[2 * (y)] - (double)J1[2 * (x)] * J2[2 * (y) + 1])
          const double cr[4] = {PR(0, 0) + PR(1, 1), PR(1, 3) + PR(0, 2), PR(2, 0) + PR(3, 1),
                                PR(2, 2) + PR(3, 3)};
          const double ci[4] = {PI(0, 0) + PI(1, 1), PI(1, 3) + PI(0, 2), PI(2, 0) + PI(3, 1),
                                PI(2, 2) + PI(3, 3)};
#undef PR
#undef PI
          for (int q = 0; q < 4; q++) {
            mr[q] += cr[q] * vr - ci[q] * vi;
            mi[q] += cr[q] * vi + ci[q] * vr;
            ml[q] += fabs(amp) * sqrt(cr[q] * cr[q] + ci[q] * ci[q]);
          }
        }
        if (s->l1)
          for (int q = 0; q < 4; q++) s->l1[((size_t)r * nfreq + ifq) * 4 + q] = ml[q];
        for (int p = 0; p < ncorr; p++) {
          const int off = offCh + p * j->incs;
          if (rec[off + 2] <= 0.0f && !j->doReplace) continue;
          const int q = kModelOf[p];
          const double Mr = mr[q] * (double)j->polFact[p], Mi = mi[q] * (double)j->polFact[p];
          if (j->doReplace) {
            rec[off] = (float)Mr;
            rec[off + 1] = (float)Mi;
          } else if (j->doDivide) {
            const double a2m = Mr * Mr + Mi * Mi;
            const double Vr = rec[off], Vi = rec[off + 1];
            rec[off] = (float)((Vr * Mr + Vi * Mi) / a2m);
            rec[off + 1] = (float)((Vi * Mr - Vr * Mi) / a2m);
          } else {
            rec[off] = (float)((double)rec[off] - Mr);
            rec[off + 1] = (float)((double)rec[off + 1] - Mi);
          }
        }
      }
    }
  }
  return NULL;
}

int oracle_beam_apply(const OracleJob *j, const OracleBeam *b, float *vis, double *l1, int nthreads) {
  if (j->modType < ORACLE_POINT || j->modType > ORACLE_GAUSS_TSPEC) return -1;
  if (j->numberPoln < 1 || j->numberPoln > 4) return -2;
  if (j->nvis <= 0 || j->ncomp <= 0) return 0;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > j->nvis) nthreads = j->nvis;
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  BeamSlice *sl = (BeamSlice *)calloc((size_t)nthreads, sizeof(BeamSlice));
  const int per = j->nvis / nthreads;
  for (int t = 0; t < nthreads; t++) {
    sl[t].job = j;
    sl[t].beam = b;
    sl[t].vis = vis;
    sl[t].l1 = l1;
    sl[t].lo = t * per;
    sl[t].hi = (t == nthreads - 1) ? j->nvis : (t + 1) * per;
  }
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, beam_slice, &sl[t]);
  beam_slice(&sl[0]);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
  free(th);
  free(sl);
  return 0;
}
