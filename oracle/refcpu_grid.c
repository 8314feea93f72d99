/*
 * Test infrastructure: the reference's per-visibility loop of the gridded
 * model, restated in C in single precision -- ThreadSkyModelFTGrid
 * (ObitSystem/Obit/src/ObitSkyModel.c:2970-3232) with ObitCInterpolateOffset,
 * ObitCInterpolatePixel and SetConvKernal (ObitCInterpolate.c:557-580,
 * 359-455, 699-745) -- threaded over records as ObitSkyModelFTGrid
 * (ObitSkyModel.c:2878-2943) divides them.  It reads the interpolator's plane
 * and kernel table built by the oracle (oracle_grid.py) and times the
 * reference's CPU algorithm for the CPU baseline; tests also compare it with
 * the GPU.  Every operation rounds as the reference's C does (no
 * contraction: compiled without FMA).  The product never links this file.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>

#include "oracle_dft.h"

#define HW 12
#define IWID (2 * HW + 1)

static void conv_setup(float pixel, int naxis, int ntab, int *start, int *k0, int *nterm, int *itab) {
  int ipos = (int)((double)pixel + 0.5);
  int cen = ipos - HW;
  if (cen > naxis - IWID) cen = naxis - IWID;
  if (cen < 1) cen = 1;
  float off = pixel - (float)cen;
  off = off - (float)HW;
  int ioff = off > 0.0f ? (int)((double)off + 0.5) : (int)((double)off - 0.5);
  off -= (float)ioff;
  int it = (int)(((0.5 + (double)off) * ntab) + 0.5);
  if (it < 0) it = 0;
  if (it > ntab) it = ntab;
  *itab = it;
  *start = cen - 1;
  *k0 = ioff < 0 ? -ioff : ioff;
  *nterm = IWID - *k0;
}

/* ObitCInterpolatePixel on the plane (no blanked plane values); returns 0
 * when the reference returns its blank. */
static int interp_pixel(const RefGridJob *j, float px, float py, float out[2]) {
  if (px < 1.0f || px > (float)j->nxp || py < 1.0f || py > (float)j->ny) return 0;
  int sx, k0x, ntx, tx, sy, k0y, nty, ty;
  conv_setup(px, j->nxp, j->ntab, &sx, &k0x, &ntx, &tx);
  conv_setup(py, j->ny, j->ntab, &sy, &k0y, &nty, &ty);
  const float *kx = j->table + (size_t)tx * IWID + k0x;
  const float *ky = j->table + (size_t)ty * IWID + k0y;
  float sumR = 0.0f, sumI = 0.0f, sumwt = 0.0f;
  for (int b = 0; b < nty; b++) {
    const float wty = ky[b];
    const float *row = j->plane + 2 * ((size_t)(sy + b) * j->nxp + sx);
    for (int a = 0; a < ntx; a++) {
      const float wt = kx[a] * wty;
      sumwt += wt;
      sumR += row[2 * a] * wt;
      sumI += row[2 * a + 1] * wt;
    }
  }
  if (!(sumwt > 0.5f)) return 0;
  out[0] = sumR / sumwt;
  out[1] = sumI / sumwt;
  return 1;
}

static void apply_rows(const RefGridJob *j, float *vis, long lo, long hi) {
  for (long iv = lo; iv < hi; iv++) {
    float *rec = vis + (size_t)iv * j->lrec;
    for (int iIF = j->ifb; iIF < j->ifb + j->nif; iIF++) {
      for (int ich = j->chanb; ich < j->chanb + j->nchan; ich++) {
        const float ff = j->fscale[iIF * j->kincif + ich * j->kincf];
        float u = ff * rec[j->ilocu], v = ff * rec[j->ilocv], w = ff * rec[j->ilocw];
        if (j->do3Dmul) {
          const float *m = j->umat;
          const float ut = u * m[0] + v * m[1] + w * m[2];
          const float vt = u * m[3] + v * m[4] + w * m[5];
          const float wt = u * m[6] + v * m[7] + w * m[8];
          u = ut;
          v = vt;
          w = wt;
        } else if (j->doRot) {
          const float ut = j->ccrot * u - j->ssrot * v;
          const float vt = j->ccrot * v + j->ssrot * u;
          u = ut;
          v = vt;
        }
        const int conj = j->flip * u < 0.0f;
        if (conj) {
          u = -u;
          v = -v;
          w = -w;
        }
        float val[2] = {0.0f, 0.0f};
        const float px = j->crpix0 + (u / j->cdelt0);
        const float py = j->crpix1 + (v / j->cdelt1);
        const int good = interp_pixel(j, px, py, val);
        if (good && j->doPC) {
          const float pc = u * j->dxyzc[0] + v * j->dxyzc[1] + w * j->dxyzc[2];
          const float c = (float)cos((double)pc), s = (float)sin((double)pc);
          const float rt = c * val[0] - s * val[1];
          const float it = c * val[1] + s * val[0];
          val[0] = rt;
          val[1] = it;
        }
        float mr = val[0], mi = conj ? -val[1] : val[1];
        if (j->doFlip) {
          const float t = mr;
          mr = -mi;
          mi = t;
        }
        float wtf = 1.0f;
        if (j->doDivide && good) {
          const float wt = mr * mr + mi * mi;
          mr /= wt;
          mi /= wt;
          wtf = (float)sqrt((double)wt);
        }
        float *base = rec + j->nrparm + iIF * j->incif + ich * j->incf;
        for (int s = j->stokb; s < j->stokb + j->nstok; s++) {
          float *c = base + s * j->incs;
          if (c[2] <= 0.0f && !j->doReplace) continue;
          if (!good) {
            c[0] = c[1] = c[2] = 0.0f;
          } else if (j->doDivide) {
            const float t = mr * c[0] + mi * c[1];
            c[1] = mr * c[1] - mi * c[0];
            c[0] = t;
            c[2] *= wtf;
          } else if (j->doReplace) {
            c[0] = mr;
            c[1] = mi;
          } else {
            c[0] -= mr;
            c[1] -= mi;
          }
          mr *= j->stokFactor;
          mi *= j->stokFactor;
        }
      }
    }
  }
}

typedef struct {
  const RefGridJob *j;
  float *vis;
  long lo, hi;
} Slice;

static void *slice_main(void *arg) {
  Slice *s = (Slice *)arg;
  apply_rows(s->j, s->vis, s->lo, s->hi);
  return NULL;
}

int refcpu_grid_apply(const RefGridJob *job, float *vis, long nvis, int nthreads) {
  if (!job || (nvis > 0 && !vis)) return 1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (nvis < 1000) nthreads = 1; /* as ObitSkyModelFTGrid */
  pthread_t th[256];
  Slice sl[256];
  int running[256];
  const long per = nvis / nthreads > 0 ? nvis / nthreads : 1;
  for (int t = 0; t < nthreads; t++) {
    running[t] = 0;
    const long lo = (long)t * per;
    const long hi = t == nthreads - 1 ? nvis : (lo + per < nvis ? lo + per : nvis);
    sl[t] = (Slice){job, vis, lo, hi};
    if (lo >= hi) continue;
    if (nthreads > 1 && pthread_create(&th[t], NULL, slice_main, &sl[t]) == 0)
      running[t] = 1;
    else
      slice_main(&sl[t]);
  }
  for (int t = 0; t < nthreads; t++)
    if (running[t]) pthread_join(th[t], NULL);
  return 0;
}
