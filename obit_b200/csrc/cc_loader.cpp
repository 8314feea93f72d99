// CLEAN-component tables to the DFT component table (include/obit_dft_comps.h).
//
// Restates, on the host, ObitTableCCUtilMergeSel (ObitTableCCUtil.c:1238-1361:
// position sort, merge of equal positions, sort by decreasing |flux|) and
// ObitSkyModelLoadComps (ObitSkyModel.c:1682-2121: selection, factor, field
// offsets, re-projection, Gaussian and spectral terms), keeping the
// reference's single- and double-precision rounding points so that the
// resulting table is the one the reference would hand to its DFT.  The file is
// compiled without floating-point contraction: every single-precision
// operation rounds where the reference's does.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "abi_internal.h"
#include "obit_dft.h"
#include "obit_dft_comps.h"
#include "sky_geom.h"

namespace {

using obit::set_last_error;
using obit::geom::shift_sin;
using obit::geom::shift_sin_d;
using obit::geom::urot3d;

constexpr double kPi = 3.14159265358979323846;
// ObitSkyModelCompType numbering (ObitSkyModel.h)
constexpr int kPointMod = 0, kGaussMod = 1, kPointSpec = 10, kGaussSpec = 11;

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

bool is_spec(int t) { return t == kPointSpec || t == kGaussSpec; }
bool is_gauss(int t) { return t == kGaussMod || t == kGaussSpec; }

// Merged CC entry: position, flux, deltaZ and spectral terms.
struct Entry {
  float dx, dy, flux, dz;
  std::vector<float> spec;
};

// Model type of a field: the first selected row's PARMS[3] (ObitSkyModel.c:1767-1790).
int field_type(const ObitDFTCCField& f, int start) {
  if (f.nparms < 4 || !f.parms || f.nrow <= 0) return kPointMod;
  const int row = std::min(std::max(start, 1), f.nrow) - 1;
  return (int)(f.parms[(size_t)row * f.nparms + 3] + 0.5f);
}

// ObitTableCCUtilMergeSel (ObitTableCCUtil.c:1238-1361) on one field's selected
// rows: sort by position, merge rows at the same (DeltaX, DeltaY) -- summing
// the flux, and for tabulated spectra each plane's flux (CCMergeSpec,
// :3189-3240); polynomial spectra are not merged -- then sort by decreasing
// |flux|.  parms receives the first selected row's PARMS[0..3].
std::vector<Entry> merge_field(const ObitDFTCCField& f, int start, int end, float parms[4]) {
  const int nspec = std::max(0, f.nparms - 4);
  std::vector<Entry> ent;
  bool first = true;
  for (int r = start; r <= end; r++) {
    const size_t k = (size_t)r - 1;
    if (f.status && f.status[k] < 0) continue;
    Entry e{f.deltaX[k], f.deltaY[k], f.flux[k], f.deltaZ ? f.deltaZ[k] : 0.0f, {}};
    if (nspec) e.spec.assign(f.parms + k * f.nparms + 4, f.parms + k * f.nparms + 4 + nspec);
    if (first && f.nparms > 0)
      for (int j = 0; j < std::min(4, f.nparms); j++) parms[j] = f.parms[k * f.nparms + j];
    first = false;
    ent.push_back(std::move(e));
  }
  std::stable_sort(ent.begin(), ent.end(), [](const Entry& a, const Entry& b) {
    return a.dx < b.dx || (a.dx == b.dx && a.dy < b.dy);
  });
  // polynomial spectra are not merged (ObitTableCCUtil.c:3215-3216)
  const bool doSpec = parms[3] >= 9.9f && parms[3] <= 19.0f;
  const bool doTSpec = parms[3] >= 19.9f && parms[3] <= 29.0f;
  std::vector<Entry> merged;
  if (doSpec) {
    merged = std::move(ent);
  } else {
    for (size_t a = 0; a < ent.size();) {
      size_t b = a + 1;
      Entry m = ent[a];
      while (b < ent.size() && ent[b].dx == m.dx && ent[b].dy == m.dy) {
        if (doTSpec)
          for (size_t t = 0; t < m.spec.size() && t < ent[b].spec.size(); t++) m.spec[t] += ent[b].spec[t];
        m.flux += ent[b++].flux;
      }
      merged.push_back(std::move(m));
      a = b;
    }
  }
  std::stable_sort(merged.begin(), merged.end(),
                   [](const Entry& a, const Entry& b) { return std::fabs(a.flux) > std::fabs(b.flux); });
  return merged;
}

// Field geometry of ObitSkyModelLoadComps (ObitSkyModel.c:1898-1928) and
// ObitSkyModelMFLoadComps (ObitSkyModelMF.c:1362-1395): the phase-centre
// shift, map / uv rotation and 3-D re-projection, in FP32 at the reference's
// rounding points and, for FP64 positions, in FP64.
struct FieldGeom {
  float ssrot = 0.f, ccrot = 1.f, xpoff = 0.f, ypoff = 0.f, xxoff = 0.f, yyoff = 0.f, zzoff = 0.f;
  bool do3Dmul = false;
  float U[3][3];
  double Ud[3][3], xxoffd = 0.0, yyoffd = 0.0, zzoffd = 0.0, ssd = 0.0, ccd = 1.0, xpoffd = 0.0, ypoffd = 0.0;
  bool deltaZ = false;
};

int field_geom(const ObitDFTCCField& f, int i, const ObitDFTCCModel* model, bool wantD, FieldGeom* g) {
  const float maprot = f.rotation, uvrot = model->uvRotation;
  g->ssrot = (float)std::sin(kPi / 180.0 * (double)(uvrot - maprot));
  g->ccrot = (float)std::cos(kPi / 180.0 * (double)(uvrot - maprot));
  g->do3Dmul = maprot != 0.0f || uvrot != 0.0f || std::fabs(f.crvalRA - model->uvRA) > 1.0e-10 ||
               std::fabs(f.crvalDec - model->uvDec) > 1.0e-10 || std::fabs(f.xPxOff) > 1.0e-20f ||
               std::fabs(f.yPxOff) > 1.0e-20f;
  if (!f.do3D && (f.xShift != 0.0f || f.yShift != 0.0f || g->do3Dmul))
    return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) +
                                           ": 2-D image with a shift, rotation or offset centre");
  float dxyzc[3];
  shift_sin(model->uvRA, model->uvDec, maprot, f.crvalRA, f.crvalDec, dxyzc);
  if (!model->do3D) {
    g->xpoff = f.xPxOff * f.cdeltX;
    g->ypoff = f.yPxOff * f.cdeltY;
  }
  g->xxoff = dxyzc[0] * g->ccrot + dxyzc[1] * g->ssrot;
  g->yyoff = dxyzc[1] * g->ccrot - dxyzc[0] * g->ssrot;
  g->zzoff = dxyzc[2];
  if (g->do3Dmul) urot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, g->U);
  g->deltaZ = f.deltaZ != nullptr;
  if (wantD) {  // FP64 positions: the same geometry with every step in double
    double dxyzd[3];
    g->ssd = std::sin(kPi / 180.0 * ((double)uvrot - (double)maprot));
    g->ccd = std::cos(kPi / 180.0 * ((double)uvrot - (double)maprot));
    shift_sin_d(model->uvRA, model->uvDec, maprot, f.crvalRA, f.crvalDec, dxyzd);
    g->xxoffd = dxyzd[0] * g->ccd + dxyzd[1] * g->ssd;
    g->yyoffd = dxyzd[1] * g->ccd - dxyzd[0] * g->ssd;
    g->zzoffd = dxyzd[2];
    if (!model->do3D) {
      g->xpoffd = (double)f.xPxOff * (double)f.cdeltX;
      g->ypoffd = (double)f.yPxOff * (double)f.cdeltY;
    }
    if (g->do3Dmul) urot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, g->Ud);
  }
  return OBIT_DFT_OK;
}

// Fields 1-3 of a component row (and its FP64 X, Y, Z when xyz is given).
void place(const FieldGeom& g, const Entry& e, float* row, double* xyz) {
  const float konst = (float)(kPi / 180.0 * 2.0 * kPi);
  const float xp0 = (e.dx + g.xpoff) * konst;
  const float xp1 = (e.dy + g.ypoff) * konst;
  const float xp2 = g.deltaZ ? e.dz * konst : 0.0f;
  float v[3];
  if (g.do3Dmul) {
    v[0] = xp0 * g.U[0][0] + xp1 * g.U[1][0];
    v[1] = xp0 * g.U[0][1] + xp1 * g.U[1][1];
    v[2] = xp0 * g.U[0][2] + xp1 * g.U[1][2];
  } else {
    v[0] = g.ccrot * xp0 + g.ssrot * xp1;
    v[1] = g.ccrot * xp1 - g.ssrot * xp0;
    v[2] = xp2;
  }
  row[1] = v[0] + g.xxoff;
  row[2] = v[1] + g.yyoff;
  row[3] = v[2] + g.zzoff;
  if (xyz) {
    const double konstd = kPi / 180.0 * 2.0 * kPi;
    const double q0 = ((double)e.dx + g.xpoffd) * konstd;
    const double q1 = ((double)e.dy + g.ypoffd) * konstd;
    const double q2 = g.deltaZ ? (double)e.dz * konstd : 0.0;
    if (g.do3Dmul) {
      xyz[0] = q0 * g.Ud[0][0] + q1 * g.Ud[1][0] + g.xxoffd;
      xyz[1] = q0 * g.Ud[0][1] + q1 * g.Ud[1][1] + g.yyoffd;
      xyz[2] = q0 * g.Ud[0][2] + q1 * g.Ud[1][2] + g.zzoffd;
    } else {
      xyz[0] = g.ccd * q0 + g.ssd * q1 + g.xxoffd;
      xyz[1] = g.ccd * q1 - g.ssd * q0 + g.yyoffd;
      xyz[2] = q2 + g.zzoffd;
    }
  }
}

// Gaussian terms from a field's FWHM and PA (ObitSkyModel.c:1938-1947,
// ObitSkyModelMF.c:1403-1411).
void gauss_terms(const float parms[4], float* gp) {
  const float konst2 = (float)(kPi / 180.0 * std::sqrt(2.0) * kPi / 2.35482044);
  const float cpa = (float)std::cos(kPi / 180.0 * (double)parms[2]);
  const float spa = (float)std::sin(kPi / 180.0 * (double)parms[2]);
  const float xmaj = parms[0] * konst2, xmin = parms[1] * konst2;
  gp[0] = -(((cpa * xmaj) * (cpa * xmaj)) + (spa * xmin) * (spa * xmin));
  gp[1] = -(((spa * xmaj) * (spa * xmaj)) + (cpa * xmin) * (cpa * xmin));
  gp[2] = (float)(-2.0 * (double)cpa * (double)spa * (double)(xmaj * xmaj - xmin * xmin));
}

// Spectral index of one component's plane fluxes: ObitSpectrumFitSingleArg
// with two terms (ObitSpectrumFit.c:1362-1412) and the control flow of NLFit
// (:2044-2250, whose post-processing after its `done` label is skipped by an
// early return).  The reference solves the least squares with GSL's lmder
// (MINPACK Levenberg-Marquardt, GNU Scientific Library, the version on the
// build host; not in this image) to |dx| < 1e-5 + 1e-5 |x|; restated here as a
// Levenberg-Marquardt iteration with Marquardt scaling and the same test, which
// converges to the same minimum.  L: ln(nu / nu_0) per plane (FP32, as the
// reference stores it); obs: plane fluxes; isig: 1/sigma (0 leaves a plane
// out).  Returns alpha (0 when the fit is not kept).
float fit_spectral_index(int n, const float* L, const float* obs, const double* isig) {
  double sum = 0.0, sumwt = 0.0, sumSig = 0.0;
  int nvalid = 0;
  bool hasNeg = false;
  for (int i = 0; i < n; i++)
    if (isig[i] > 0.0) {
      const double w = isig[i] * isig[i];
      sum += w * obs[i];
      sumwt += w;
      sumSig += isig[i];
      nvalid++;
      hasNeg = hasNeg || obs[i] < 0.0f;
    }
  if (nvalid <= 0) return 0.0f;
  const float avg = (float)(sum / sumwt);
  if (nvalid == 1) return 0.0f;  // blanked index, zeroed by the loader's sanity range
  double chi = 0.0, snr = 0.0;
  for (int i = 0; i < n; i++)
    if (isig[i] > 0.0) {
      const float d = obs[i] - avg;
      chi += isig[i] * isig[i] * (double)d * d;
      snr += std::fabs(obs[i]) * isig[i];
    }
  const float chiSq = (float)(chi / (nvalid - 1));
  const float meanSNR = (float)(snr / nvalid);
  bool isDone = hasNeg || chiSq < 0.0f || 0.0f > avg;  // minFlux 0
  if (meanSNR > 1.0f && 0.0f < avg) isDone = false;
  if (isDone) return 0.0f;
  // two-term fit S0 exp(alpha L) from (avg, 0)
  double x[2] = {avg, 0.0};
  auto cost = [&](const double* y) {
    double c = 0.0;
    for (int i = 0; i < n; i++)
      if (isig[i] > 0.0) {
        const double r = (y[0] * std::exp(y[1] * (double)L[i]) - obs[i]) * isig[i];
        c += r * r;
      }
    return c;
  };
  double c0 = cost(x), lambda = 1e-3;
  for (int iter = 0; iter < 100; iter++) {
    double A[2][2] = {{0, 0}, {0, 0}}, gr[2] = {0, 0};
    for (int i = 0; i < n; i++)
      if (isig[i] > 0.0) {
        const double e = std::exp(x[1] * (double)L[i]);
        const double r = (x[0] * e - obs[i]) * isig[i];
        const double j0 = e * isig[i], j1 = x[0] * (double)L[i] * e * isig[i];
        A[0][0] += j0 * j0;
        A[0][1] += j0 * j1;
        A[1][1] += j1 * j1;
        gr[0] += j0 * r;
        gr[1] += j1 * r;
      }
    double dx[2] = {0.0, 0.0}, c1 = c0;
    bool stepped = false;
    for (int tries = 0; tries < 30 && !stepped; tries++) {
      const double a = A[0][0] * (1.0 + lambda), d = A[1][1] * (1.0 + lambda), b = A[0][1];
      const double det = a * d - b * b;
      if (!(det > 0.0)) {
        lambda *= 10.0;
        continue;
      }
      dx[0] = -(d * gr[0] - b * gr[1]) / det;
      dx[1] = -(a * gr[1] - b * gr[0]) / det;
      const double y[2] = {x[0] + dx[0], x[1] + dx[1]};
      c1 = cost(y);
      if (c1 <= c0) {
        stepped = true;
        lambda = std::max(lambda * 0.1, 1e-12);
      } else {
        lambda *= 10.0;
      }
    }
    if (!stepped) break;  // no decrease at any damping: at the minimum
    x[0] += dx[0];
    x[1] += dx[1];
    c0 = c1;
    if (std::fabs(dx[0]) < 1e-5 + 1e-5 * std::fabs(x[0]) && std::fabs(dx[1]) < 1e-5 + 1e-5 * std::fabs(x[1]))
      break;
  }
  // reduced chi^2 of the fit; kept if not much worse than the constant's
  const float chi2Test = (nvalid > 2) ? (float)(c0 / (nvalid - 2)) : -1.0f;
  if (!(chi2Test < 1.5f * chiSq)) return 0.0f;
  return (float)x[1];
}

}  // namespace

extern "C" int obit_dft_load_comps(const ObitDFTCCField* fields, int nfield, const ObitDFTCCModel* model,
                                   float* table, long long capacity, int* nrowOut, int* ncompOut,
                                   int* lcompOut, int* modTypeOut, int* ntermOut) {
  return obit_dft_load_comps_d(fields, nfield, model, table, capacity, nrowOut, ncompOut, lcompOut,
                               modTypeOut, ntermOut, nullptr);
}

extern "C" int obit_dft_load_comps_d(const ObitDFTCCField* fields, int nfield, const ObitDFTCCModel* model,
                                     float* table, long long capacity, int* nrowOut, int* ncompOut,
                                     int* lcompOut, int* modTypeOut, int* ntermOut, double* xyzOut) {
  set_last_error("");
  if (nfield < 0 || (nfield > 0 && !fields) || !model || !nrowOut || !lcompOut)
    return fail(OBIT_DFT_EBADARG, "NULL or negative argument");
  // ---- counting pass: rows, model type, spectral terms (ObitSkyModel.c:1727-1816)
  long long count = 0;
  int maxType = kPointMod, maxTerm = 1;
  for (int i = 0; i < nfield; i++) {
    const ObitDFTCCField& f = fields[i];
    if (f.nrow < 0 || (f.nrow > 0 && (!f.flux || !f.deltaX || !f.deltaY)) || f.nparms < 0 ||
        (f.nparms > 0 && !f.parms))
      return fail(OBIT_DFT_EBADARG, "field " + std::to_string(i) + ": bad CC columns");
    const int start = std::max(1, f.startComp);
    const int end = f.endComp > 0 ? std::min(f.endComp, f.nrow) : f.nrow;
    if (end < start) continue;
    count += end - start + 1;
    const int t = field_type(f, start);
    if (t != kPointMod && t != kGaussMod && t != kPointSpec && t != kGaussSpec)
      return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) + ": component type " +
                                             std::to_string(t) + " is not a DFT model type here");
    maxType = std::max(maxType, t);
    if (is_spec(maxType)) maxTerm = std::max(maxTerm, f.nparms - 3);
  }
  const int nterm = std::max(0, maxTerm - 1);
  const int lcomp = 4 + (is_gauss(maxType) ? 3 : 0) + (is_spec(maxType) ? nterm : 0);
  *nrowOut = (int)count;
  *lcompOut = lcomp;
  if (modTypeOut) *modTypeOut = maxType;
  if (ntermOut) *ntermOut = is_spec(maxType) ? nterm : 0;
  if (ncompOut) *ncompOut = 0;
  if (!table) return OBIT_DFT_OK;
  if (capacity < count * lcomp)
    return fail(OBIT_DFT_EBADARG, "table capacity below rows x floats per row");
  std::fill(table, table + count * lcomp, 0.0f);

  long long ncomp = 0;
  float* row = table;
  for (int i = 0; i < nfield; i++) {
    const ObitDFTCCField& f = fields[i];
    const int start = std::max(1, f.startComp);
    const int end = f.endComp > 0 ? std::min(f.endComp, f.nrow) : f.nrow;
    if (end < start) continue;
    if (f.ncpProjection) return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) + ": -NCP projection");
    // ---- ObitTableCCUtilMergeSel: selected rows, model parameters of the first
    const int ftype = field_type(f, start);
    // type combinations the reference accepts (ObitSkyModel.c:2047-2083)
    if (!(ftype == maxType || (ftype == kPointMod && maxType == kGaussMod) ||
          (ftype == kPointSpec && maxType == kGaussSpec) || (ftype == kPointMod && maxType == kPointSpec)))
      return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) + ": component type " +
                                             std::to_string(ftype) + " cannot be mixed into type " +
                                             std::to_string(maxType));
    float parms[4] = {0, 0, 0, 0};
    const std::vector<Entry> merged = merge_field(f, start, end, parms);
    FieldGeom g;
    if (int rc = field_geom(f, i, model, xyzOut != nullptr, &g)) return rc;
    float gp[3] = {0.f, 0.f, 0.f};
    if (is_gauss(ftype)) gauss_terms(parms, gp);
    for (const Entry& e : merged) {
      if (model->noNeg && e.flux <= 0.0f) break;
      const bool want = std::fabs(e.flux) > model->minDFT && std::fabs(e.flux) > model->minFlux &&
                        ncomp < count;
      if (!want) continue;
      row[0] = e.flux * model->factor;
      place(g, e, row, xyzOut ? xyzOut + 3 * (size_t)ncomp : nullptr);
      // type-specific terms, mixed types zero what a field lacks (ObitSkyModel.c:1990-2083)
      const int g0 = 4, s0 = is_gauss(maxType) ? 7 : 4;
      if (is_gauss(maxType) && is_gauss(ftype)) {
        row[g0] = gp[0];
        row[g0 + 1] = gp[1];
        row[g0 + 2] = gp[2];
      }
      if (is_spec(maxType) && is_spec(ftype))
        for (int t = 0; t < nterm && t < (int)e.spec.size(); t++) row[s0 + t] = e.spec[t];
      row += lcomp;
      ncomp++;
    }
  }
  if (ncompOut) *ncompOut = (int)ncomp;
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_load_comps_mf(const ObitDFTCCField* fields, int nfield, const ObitDFTCCModel* model,
                                      const ObitDFTCCModelMF* mf, float* table, long long capacity,
                                      int* nrowOut, int* ncompOut, int* lcompOut, int* modTypeOut) {
  set_last_error("");
  if (nfield < 0 || (nfield > 0 && !fields) || !model || !mf || !nrowOut || !lcompOut)
    return fail(OBIT_DFT_EBADARG, "NULL or negative argument");
  const int nSpec = mf->nSpec;
  if (nSpec < 1 || !mf->specFreq) return fail(OBIT_DFT_EBADARG, "tabulated spectra need nSpec >= 1 plane frequencies");
  for (int k = 0; k < nSpec; k++)
    if (!(mf->specFreq[k] > 0.0)) return fail(OBIT_DFT_EBADARG, "plane frequencies must be positive");
  constexpr int kPointTSpec = 20, kGaussTSpec = 21;
  // ---- counting pass (ObitSkyModelMF.c:1178-1268)
  long long count = 0;
  int mtype = -1;
  for (int i = 0; i < nfield; i++) {
    const ObitDFTCCField& f = fields[i];
    if (f.nrow < 0 || (f.nrow > 0 && (!f.flux || !f.deltaX || !f.deltaY)) || f.nparms < 0 ||
        (f.nparms > 0 && !f.parms))
      return fail(OBIT_DFT_EBADARG, "field " + std::to_string(i) + ": bad CC columns");
    const int start = std::max(1, f.startComp);
    const int end = f.endComp > 0 ? std::min(f.endComp, f.nrow) : f.nrow;
    if (end < start) continue;
    count += end - start + 1;
    const int t = field_type(f, start);
    if (t != kPointTSpec && t != kGaussTSpec)
      return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) + ": component type " + std::to_string(t) +
                                             " is not a tabulated-spectrum type");
    if (mtype >= 0 && t != mtype)
      return fail(OBIT_DFT_EUNSUPPORTED, "fields of both tabulated-spectrum types");
    mtype = t;
    if (f.nparms < 4 + nSpec)
      return fail(OBIT_DFT_EBADARG, "field " + std::to_string(i) + ": PARMS shorter than 4 + nSpec");
  }
  if (mtype < 0) mtype = kPointTSpec;
  const bool gauss = (mtype == kGaussTSpec);
  const int lcomp = 4 + (gauss ? 3 : 0) + nSpec + 1;
  *nrowOut = (int)count;
  *lcompOut = lcomp;
  if (modTypeOut) *modTypeOut = mtype;
  if (ncompOut) *ncompOut = 0;
  if (!table) return OBIT_DFT_OK;
  if (capacity < count * lcomp) return fail(OBIT_DFT_EBADARG, "table capacity below rows x floats per row");
  std::fill(table, table + count * lcomp, 0.0f);
  // the fit's planes and the prior-alpha correction times Factor (ObitSkyModelMF.c:1293-1318)
  const bool doFit = !mf->noSIfit && nSpec > 1;
  std::vector<float> L(nSpec), specCorr(nSpec);
  for (int k = 0; k < nSpec; k++) {
    L[k] = (float)std::log(mf->specFreq[k] / mf->specFreq[0]);
    specCorr[k] = (mf->doAlphaCorr && mf->priorAlpha != 0.0f)
                      ? (float)((double)model->factor * std::pow(mf->specFreq[k] / mf->priorAlphaRefF,
                                                                 (double)mf->priorAlpha))
                      : model->factor;
  }
  std::vector<float> obs(nSpec);
  std::vector<double> isig(nSpec);
  long long ncomp = 0;
  float* row = table;
  const int s0 = gauss ? 7 : 4;  // spectral index, then the planes
  for (int i = 0; i < nfield; i++) {
    const ObitDFTCCField& f = fields[i];
    const int start = std::max(1, f.startComp);
    const int end = f.endComp > 0 ? std::min(f.endComp, f.nrow) : f.nrow;
    if (end < start) continue;
    if (f.ncpProjection) return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) + ": -NCP projection");
    float parms[4] = {0, 0, 0, 0};
    const std::vector<Entry> merged = merge_field(f, start, end, parms);
    FieldGeom g;
    if (int rc = field_geom(f, i, model, false, &g)) return rc;
    float gp[3] = {0.f, 0.f, 0.f};
    if (gauss) gauss_terms(parms, gp);
    for (const Entry& e : merged) {
      if (model->noNeg && e.flux <= 0.0f) break;
      const bool want = std::fabs(e.flux) > model->minDFT && std::fabs(e.flux) > model->minFlux &&
                        ncomp < count;
      if (!want) continue;
      float alpha = 0.0f;
      if (doFit) {
        for (int k = 0; k < nSpec; k++) {
          const float v = k < (int)e.spec.size() ? e.spec[k] : 0.0f;
          obs[k] = v * specCorr[k];
          isig[k] = (v == 0.0f) ? 0.0 : 1.0 / 1.0e-4;  // exactly-zero planes left out
        }
        alpha = fit_spectral_index(nSpec, L.data(), obs.data(), isig.data());
        if (alpha < -2.0f || alpha > 2.0f) alpha = 0.0f;  // sanity range (ObitSkyModelMF.c:1432-1433)
      }
      row[0] = e.flux * model->factor;
      place(g, e, row, nullptr);
      if (gauss) {
        row[4] = gp[0];
        row[5] = gp[1];
        row[6] = gp[2];
      }
      row[s0] = alpha;
      for (int k = 0; k < nSpec; k++) row[s0 + 1 + k] = (k < (int)e.spec.size() ? e.spec[k] : 0.0f) * specCorr[k];
      row += lcomp;
      ncomp++;
    }
  }
  if (ncompOut) *ncompOut = (int)ncomp;
  return OBIT_DFT_OK;
}
