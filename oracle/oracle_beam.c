/* Test infrastructure (never linked into the product): FP64 oracle of the
 * beam-corrected DFT, the model of ObitCUDABeamModel's beam*Kernel family
 * (ObitSystem/Obit/src/ObitCUDABeamModel.cu:139-1226) for linear feeds and a
 * Stokes I, Q, U or V sky, and of the CPU path's circular-feed branch.
 *
 * For a record of baseline (a1, a2) with antenna types t1, t2 and a (channel,
 * IF) whose Jones plane is jc, each component contributes v = amp e^{i phase}
 * (amplitude and phase as in the DFT oracle, oracle_comp_term) times the
 * coefficients of its Stokes (beam_coeffs below) with J1 = Jones[t1][c][jc],
 * J2 = Jones[t2][c][jc] and P(i, j) = J1[i] conj(J2[j]); for Stokes I
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
#include <string.h>

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

/* Coefficients of the four model correlations (XX, XY, YX, YY) for one
 * component from P(i, j) = J1[i] conj(J2[j]), as cudaJonesCor1_Lin_{I,Q,U,V}
 * (ObitSystem/Obit/include/CUDALinCorSum.h:104-455) and the CPU
 * ObitSkyModelVMBeamJonesCorSum (ObitSystem/Obit/src/ObitSkyModelVMBeam.c:1117-1240)
 * form them. */
static void beam_coeffs(const OracleBeam *b, const float *J1, const float *J2, double cr[4],
                        double ci[4]) {
  if (b->circular) {
    /* Circular feeds: the model matrix is J1 M conj(J2)^T with the sky's
     * pseudo-visibility matrix M of ObitSkyModelVMBeamJonesCorSum
     * (ObitSystem/Obit/src/ObitSkyModelVMBeam.c:1039-1073, product at
     * :1263-1268), per unit visibility:
     *   I [[1, 0], [0, 1]]  Q [[0, 1], [1, 0]]  U [[0, i], [-i, 0]]  V [[1, 0], [0, -1]]
     * element (a, b) -> correlation RR, RL, LR, LL = 2a + b. */
    double mr[2][2] = {{0, 0}, {0, 0}}, mi[2][2] = {{0, 0}, {0, 0}};
    switch (b->stokType) {
      case 1: mr[0][0] = mr[1][1] = 1.0; break;
      case 2: mr[0][1] = mr[1][0] = 1.0; break;
      case 3: mi[0][1] = 1.0; mi[1][0] = -1.0; break;
      default: mr[0][0] = 1.0; mr[1][1] = -1.0; break;
    }
    for (int a = 0; a < 2; a++)
      for (int c = 0; c < 2; c++) {
        double sr = 0.0, si = 0.0;
        for (int i = 0; i < 2; i++)
          for (int j = 0; j < 2; j++) {
            /* J1(a, i) M(i, j) conj(J2(c, j)) */
            const double ar = J1[2 * (2 * a + i)], ai = J1[2 * (2 * a + i) + 1];
            const double br = J2[2 * (2 * c + j)], bi = -(double)J2[2 * (2 * c + j) + 1];
            const double tr = ar * mr[i][j] - ai * mi[i][j], ti = ar * mi[i][j] + ai * mr[i][j];
            sr += tr * br - ti * bi;
            si += tr * bi + ti * br;
          }
        cr[2 * a + c] = sr;
        ci[2 * a + c] = si;
      }
    return;
  }
  double pr[4][4], pi[4][4];
  for (int x = 0; x < 4; x++)
    for (int y = 0; y < 4; y++) {
      pr[x][y] = (double)J1[2 * x] * J2[2 * y] + (double)J1[2 * x + 1] * J2[2 * y + 1];
      pi[x][y] = (double)J1[2 * x + 1] * J2[2 * y] - (double)J1[2 * x] * J2[2 * y + 1];
    }
  /* the (a, b) terms of each correlation: XX (0,0)(1,1) ...; see the table below */
  static const int A[4][4] = {{0, 1, 1, 0}, {0, 1, 1, 0}, {2, 3, 3, 2}, {2, 3, 3, 2}};
  static const int B[4][4] = {{0, 1, 0, 1}, {2, 3, 2, 3}, {0, 1, 0, 1}, {2, 3, 2, 3}};
  /* per correlation q: D = P(A0,B0) - P(A1,B1) ("difference"), S = P(A2,B2) + P(A3,B3) ("sum") */
  for (int q = 0; q < 4; q++) {
    const double Dr = pr[A[q][0]][B[q][0]] - pr[A[q][1]][B[q][1]];
    const double Di = pi[A[q][0]][B[q][0]] - pi[A[q][1]][B[q][1]];
    const double Sr = pr[A[q][2]][B[q][2]] + pr[A[q][3]][B[q][3]];
    const double Si = pi[A[q][2]][B[q][2]] + pi[A[q][3]][B[q][3]];
    switch (b->stokType) {
      case 2: /* Q: c2p D - s2p S */
        cr[q] = b->c2p * Dr - b->s2p * Sr;
        ci[q] = b->c2p * Di - b->s2p * Si;
        break;
      case 3: /* U: c2p S + s2p D */
        cr[q] = b->c2p * Sr + b->s2p * Dr;
        ci[q] = b->c2p * Si + b->s2p * Di;
        break;
      default: break;
    }
  }
  if (b->stokType == 1) { /* I: XX P00+P11, XY P13+P02, YX P20+P31, YY P22+P33 */
    cr[0] = pr[0][0] + pr[1][1]; ci[0] = pi[0][0] + pi[1][1];
    cr[1] = pr[1][3] + pr[0][2]; ci[1] = pi[1][3] + pi[0][2];
    cr[2] = pr[2][0] + pr[3][1]; ci[2] = pi[2][0] + pi[3][1];
    cr[3] = pr[2][2] + pr[3][3]; ci[3] = pi[2][2] + pi[3][3];
  } else if (b->stokType == 4) { /* V: i (P01-P13), i (P03-P12), i (P21-P30), i (P23-P32) */
    const int a0[4] = {0, 0, 2, 2}, b0[4] = {1, 3, 1, 3}, a1[4] = {1, 1, 3, 3}, b1[4] = {3, 2, 0, 2};
    for (int q = 0; q < 4; q++) {
      const double dr = pr[a0[q]][b0[q]] - pr[a1[q]][b1[q]];
      const double di = pi[a0[q]][b0[q]] - pi[a1[q]][b1[q]];
      cr[q] = -di;
      ci[q] = dr;
    }
  }
}

/* The coefficients for one Jones pair, exported for the check against the
 * reference's own cudaJonesCor1_Lin_* (oracle/refjones.cpp). */
void oracle_beam_coeffs(int stokType, double c2p, double s2p, const float *J1, const float *J2,
                        double *cr, double *ci) {
  OracleBeam b;
  memset(&b, 0, sizeof(b));
  b.stokType = stokType;
  b.circular = 0;
  b.c2p = c2p;
  b.s2p = s2p;
  beam_coeffs(&b, J1, J2, cr, ci);
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
          double cr[4], ci[4];
          beam_coeffs(b, J1, J2, cr, ci);
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
  if (b->stokType < 1 || b->stokType > 4) return -3;
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

/* Grid offsets (deg) of position (x, y) (deg) in projection proj (0 linear,
 * 1..8 -SIN -TAN -ARC -NCP -GLS -MER -AIT -STG) about crval, as
 * CUDAPositionXYpixLM (ObitSystem/Obit/include/CUDASkyGeom.h:91-250) defines
 * them; returns 0 where the position cannot be projected.  The zenithal
 * projections are written here through the angle theta from the reference
 * and their radial functions (sin, tan, theta, 2 tan(theta / 2)); the others
 * follow the AIPS definitions, with the grid-scaled -MER and -AIT factors. */
static int grid_offsets(int proj, const double crval[2], const double cdelt[2], double crota, double x,
                        double y, double *lo, double *mo) {
  const double d2r = 1.745329252e-2, halfPi = 6.28318530717959 / 4.0;
  const double dx = x - crval[0];
  if (dx > 180.0) x -= 360.0;
  if (dx < -180.0) x += 360.0;
  *lo = x - crval[0];
  *mo = y - crval[1];
  if (proj == 0) return 1;
  const double a0 = crval[0] * d2r, d0 = crval[1] * d2r, a = x * d2r, d = y * d2r;
  const double east = sin(a - a0) * cos(d);
  const double north = sin(d) * cos(d0) - cos(d) * sin(d0) * cos(a - a0);
  const double ct = sin(d) * sin(d0) + cos(d) * cos(d0) * cos(a - a0);
  double L, M;
  if (proj == 1 || proj == 2 || proj == 3 || proj == 8) {
    if (proj == 1 && ct < 0.0) return 0;
    if (proj == 2 && ct <= 0.0) return 0;
    if (proj == 8 && (fabs(d) > halfPi || fabs(1.0 + ct) < 1.0e-5)) return 0;
    const double st = sqrt(east * east + north * north);
    const double th = atan2(st, ct);
    double R;
    if (proj == 1) R = sin(th);
    else if (proj == 2) R = tan(th);
    else if (proj == 3) R = th;
    else R = 2.0 * tan(th / 2.0);
    const double f = st > 1e-12 ? R / st : 1.0; /* R(theta) / sin(theta) */
    L = east * f;
    M = north * f;
  } else if (proj == 4) {
    if (d0 == 0.0) return 0;
    L = east;
    M = (cos(d0) - cos(d) * cos(a - a0)) / sin(d0);
  } else if (proj == 5) {
    if (fabs(d) > halfPi || fabs(d0) > halfPi) return 0;
    L = (a - a0) * cos(d);
    M = d - d0;
  } else if (proj == 6) {
    const double rot = crota * d2r;
    double dy = cdelt[1] * cos(rot) + cdelt[0] * sin(rot);
    if (dy == 0.0) dy = 1.0;
    const double q0 = log(tan((crval[1] / 2.0 + 45.0) * d2r));
    const double q1 = log(tan((crval[1] / 2.0 + 45.0) * d2r + dy / 2.0 * d2r));
    const double gy = dy * d2r / (q1 - q0);
    double gx = cos(crval[1] * d2r);
    if (gx <= 0.0) gx = 1.0;
    const double t = tan(d / 2.0 + halfPi / 2.0);
    if (t < 1.0e-5) return 0;
    L = gx * (a - a0);
    M = gy * (log(t) - q0);
  } else if (proj == 7) {
    const double h = (a - a0) / 2.0;
    if (fabs(h) > halfPi) return 0;
    const double rot = crota * d2r;
    double sy = (cdelt[1] * cos(rot) + cdelt[0] * sin(rot));
    if (sy == 0.0) sy = 1.0;
    sy *= d2r;
    double sx = (cdelt[0] * cos(rot) - cdelt[1] * sin(rot));
    if (sx == 0.0) sx = 1.0;
    sx *= d2r;
    /* Hammer-Aitoff y(dec) at the reference declination, normalised so that
       one increment along each axis is one increment of the grid */
#define HA_Y(dec) (sin(dec) / sqrt((1.0 + cos(dec)) / 2.0))
    double ny = HA_Y(d0 + sy) - HA_Y(d0);
    if (ny == 0.0) ny = 1.0;
    double nx = 2.0 * cos(d0) * sin(sx / 2.0);
    if (nx == 0.0) nx = 1.0;
    const double gy = sy / ny;
    const double gx = sx * sqrt((1.0 + cos(d0) * cos(sx / 2.0)) / 2.0) / nx;
    const double z = sqrt((1.0 + cos(d) * cos(h)) / 2.0);
    if (fabs(z) < 1.0e-5) return 0;
    L = 2.0 * gx * cos(d) * sin(h) / z;
    M = gy * (sin(d) / z - HA_Y(d0));
#undef HA_Y
  } else {
    return 0;
  }
  *lo = L / d2r;
  *mo = M / d2r;
  return 1;
}

/* Jones table from beam images, FP64 (test infrastructure): the computation of
 * GetJonesKernel (ObitSystem/Obit/src/ObitCUDABeamModel.cu:1228-1299) with
 * CUDAPositionXYpix (ObitSystem/Obit/include/CUDASkyGeom.h:91-286, linear grids
 * and the eight projections of grid_offsets), the Lagrange interpolator of CUDABeamInterpPixel /
 * SetConvKernal (ObitSystem/Obit/include/CUDABeamInterp.h) and InvBeam
 * (ObitCUDABeamModel.cu:66-72), with the unit matrix where the position is
 * off the grid, the gain factor is 10 or more, a parallel hand's real part
 * exceeds 1.3 or an interpolant is blank.  pixels: [ntype][8][nplane][ny][nx]
 * (P1 re, im, P2 re, im, X1 re, im, X2 re, im); pos: [ncomp][2] (deg);
 * jones out: [ntype][ncomp][nplane][8] (XX = P1, XY = X1, YX = X2, YY = P2). */
void oracle_beam_jones(int ntype, int nx, int ny, int nplane, const float *pixels, float fblank,
                       int hwidth, int projection, const double crval[2], const double crpix[2],
                       const double cdelt[2], double crota, const double *planeFreq, double refSizeFact,
                       double parAng, const float *pos, int ncomp, float *jones) {
  const int iwid = 2 * hwidth + 1;
  const size_t img = (size_t)nplane * ny * nx;
  for (int t = 0; t < ntype; t++)
    for (int c = 0; c < ncomp; c++) {
      float *Jc = jones + ((size_t)t * ncomp + c) * nplane * 8;
      double x = pos[2 * c], y = pos[2 * c + 1];
      double l, m;
      const int ok = grid_offsets(projection, crval, cdelt, crota, x, y, &l, &m);
      const double lr = l * cos(parAng) + m * sin(parAng), mr = m * cos(parAng) - l * sin(parAng);
      const double px = lr / cdelt[0] + crpix[0], py = mr / cdelt[1] + crpix[1];
      if (!ok || !(px >= 1.0 && px <= nx && py >= 1.0 && py <= ny)) { /* NaN is off the grid */
        for (int k = 0; k < nplane; k++) {
          float *J = Jc + 8 * k;
          for (int e = 0; e < 8; e++) J[e] = (e == 0 || e == 6) ? 1.0f : 0.0f;
        }
        continue;
      }
      /* Lagrange taps on each axis: nodes 1..iwid counted from the first tap */
      double w[2][9];
      int start[2];
      const double pix[2] = {px, py};
      const int n[2] = {nx, ny};
      for (int a = 0; a < 2; a++) {
        int cen = (int)(pix[a] + 0.5) - hwidth;
        if (cen > n[a] - iwid + 1) cen = n[a] - iwid + 1;
        if (cen < 1) cen = 1;
        start[a] = cen - 1;
        const double xx = pix[a] - (double)(cen - 1);
        for (int j = 0; j < iwid; j++) {
          double prod = 1.0, den = 1.0;
          for (int i = 0; i < iwid; i++)
            if (i != j) {
              prod *= xx - (i + 1);
              den *= (double)(j - i);
            }
          w[a][j] = prod / den;
        }
      }
      const double ang = sqrt(x * x + y * y);
      for (int k = 0; k < nplane; k++) {
        double v[8];
        int blank = 0;
        for (int q = 0; q < 8; q++) {
          const float *d = pixels + ((size_t)t * 8 + q) * img + (size_t)k * ny * nx;
          double sum = 0.0, sumwt = 0.0;
          for (int j = 0; j < iwid; j++)
            for (int i = 0; i < iwid; i++) {
              const float val = d[(size_t)(start[1] + j) * nx + start[0] + i];
              if (val != fblank) {
                sumwt += w[0][i] * w[1][j];
                sum += val * w[0][i] * w[1][j];
              }
            }
          if (sumwt > 0.90) v[q] = sum / sumwt;
          else blank = 1;
        }
        const double arg = refSizeFact * planeFreq[k] * ang;
        const double g = (arg > 1.02) ? 100.0 : (1.0 - 4.0 * arg * arg) / cos(3.141592653589793 * arg);
        float *J = Jc + 8 * k;
        if (blank || !(g < 10.0) || !(fabs(g * v[0]) <= 1.3) || !(fabs(g * v[2]) <= 1.3)) {
          for (int e = 0; e < 8; e++) J[e] = (e == 0 || e == 6) ? 1.0f : 0.0f;
          continue;
        }
        const int src[8] = {0, 1, 4, 5, 6, 7, 2, 3};
        for (int e = 0; e < 8; e++) J[e] = (float)(g * v[src[e]]);
      }
    }
}
