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

namespace {

using obit::set_last_error;

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

// ObitSkyGeomShiftSIN (ObitSkyGeom.c:177-205): FP64 direction cosines of the
// field centre in the map frame, FP32 phase-shift terms 2 pi (l, m, n - 1).
void shift_sin(double ra, double dec, float rotate, double xra, double xdec, float dxyzc[3]) {
  // the reference's DG2RAD macro expands unparenthesized: rotate * pi / 180
  const float maprr = (float)(rotate * kPi / 180.0);
  const double d2r = kPi / 180.0;
  const double xxshft = std::cos(d2r * xdec) * std::sin(d2r * (xra - ra));
  const double yyshft = std::sin(d2r * xdec) * std::cos(d2r * dec) -
                        std::cos(d2r * xdec) * std::sin(d2r * dec) * std::cos(d2r * (xra - ra));
  const float xshift = (float)(std::cos((double)maprr) * xxshft + std::sin((double)maprr) * yyshft);
  const float yshift = (float)(-std::sin((double)maprr) * xxshft + std::cos((double)maprr) * yyshft);
  const float x2 = xshift * xshift, y2 = yshift * yshift;  // single-precision squares
  const double dz = std::sqrt(1.0 - (double)x2 - (double)y2);
  dxyzc[0] = (float)(2.0 * kPi * (double)xshift);
  dxyzc[1] = (float)(2.0 * kPi * (double)yshift);
  dxyzc[2] = (float)(2.0 * kPi * (dz - 1.0));
}

// The same shift terms with no single-precision rounding (FP64 positions).
void shift_sin_d(double ra, double dec, float rotate, double xra, double xdec, double dxyzc[3]) {
  const double maprr = (double)rotate * kPi / 180.0;
  const double d2r = kPi / 180.0;
  const double xxshft = std::cos(d2r * xdec) * std::sin(d2r * (xra - ra));
  const double yyshft = std::sin(d2r * xdec) * std::cos(d2r * dec) -
                        std::cos(d2r * xdec) * std::sin(d2r * dec) * std::cos(d2r * (xra - ra));
  const double xshift = std::cos(maprr) * xxshft + std::sin(maprr) * yyshft;
  const double yshift = -std::sin(maprr) * xxshft + std::cos(maprr) * yyshft;
  const double dz = std::sqrt(1.0 - xshift * xshift - yshift * yshift);
  dxyzc[0] = 2.0 * kPi * xshift;
  dxyzc[1] = 2.0 * kPi * yshift;
  dxyzc[2] = 2.0 * kPi * (dz - 1.0);
}

// ObitUVDescShift3DMatrix, 3-D image branch (ObitUVDesc.c:913-978): the uv
// re-projection matrix R(map +) X R(uv -), FP64 products in the reference's
// summation order, FP32 result.
template <typename T>
void urot3d(double ra, double dec, double xra, double xdec, float mrot, float urot, T U[3][3]) {
  const double d2r = kPi / 180.0;
  const double sa = std::sin(d2r * (xra - ra)), ca = std::cos(d2r * (xra - ra));
  const double sd = std::sin(d2r * xdec), cd = std::cos(d2r * xdec);
  const double sd0 = std::sin(d2r * dec), cd0 = std::cos(d2r * dec);
  double rm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 1.0}};
  double r = d2r * (double)mrot;
  rm[0][0] = std::cos(r);
  rm[1][1] = rm[0][0];
  rm[1][0] = -std::sin(r);
  rm[0][1] = std::sin(r);
  double x[3][3];
  x[0][0] = ca;
  x[1][0] = -sd * sa;
  x[2][0] = cd * sa;
  x[0][1] = sd0 * sa;
  x[1][1] = cd * cd0 + sd * sd0 * ca;
  x[2][1] = sd * cd0 - cd * sd0 * ca;
  x[0][2] = -cd0 * sa;
  x[1][2] = cd * sd0 - sd * cd0 * ca;
  x[2][2] = sd * sd0 + cd * cd0 * ca;
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      t[j][i] = 0.0;
      for (int k = 0; k < 3; k++) t[j][i] += x[k][i] * rm[j][k];
    }
  r = d2r * (double)urot;
  rm[0][0] = std::cos(r);
  rm[1][1] = rm[0][0];
  rm[1][0] = std::sin(r);
  rm[0][1] = -std::sin(r);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++) s += rm[k][i] * t[j][k];
      U[j][i] = (T)s;
    }
}

// Model type of a field: the first selected row's PARMS[3] (ObitSkyModel.c:1767-1790).
int field_type(const ObitDFTCCField& f, int start) {
  if (f.nparms < 4 || !f.parms || f.nrow <= 0) return kPointMod;
  const int row = std::min(std::max(start, 1), f.nrow) - 1;
  return (int)(f.parms[(size_t)row * f.nparms + 3] + 0.5f);
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

  const float konst = (float)(kPi / 180.0 * 2.0 * kPi);
  const float konst2 = (float)(kPi / 180.0 * std::sqrt(2.0) * kPi / 2.35482044);
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
    const int nspec = std::max(0, f.nparms - 4);
    float parms[4] = {0, 0, 0, 0};
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
    std::vector<Entry> merged;
    if (doSpec) {
      merged = std::move(ent);
    } else {
      for (size_t a = 0; a < ent.size();) {
        size_t b = a + 1;
        Entry m = ent[a];
        while (b < ent.size() && ent[b].dx == m.dx && ent[b].dy == m.dy) m.flux += ent[b++].flux;
        merged.push_back(std::move(m));
        a = b;
      }
    }
    std::stable_sort(merged.begin(), merged.end(),
                     [](const Entry& a, const Entry& b) { return std::fabs(a.flux) > std::fabs(b.flux); });

    // ---- ObitSkyModelLoadComps: field geometry (ObitSkyModel.c:1898-1928)
    const float maprot = f.rotation, uvrot = model->uvRotation;
    const float ssrot = (float)std::sin(kPi / 180.0 * (double)(uvrot - maprot));
    const float ccrot = (float)std::cos(kPi / 180.0 * (double)(uvrot - maprot));
    const bool do3Dmul = maprot != 0.0f || uvrot != 0.0f || std::fabs(f.crvalRA - model->uvRA) > 1.0e-10 ||
                         std::fabs(f.crvalDec - model->uvDec) > 1.0e-10 ||
                         std::fabs(f.xPxOff) > 1.0e-20f || std::fabs(f.yPxOff) > 1.0e-20f;
    if (!f.do3D && (f.xShift != 0.0f || f.yShift != 0.0f || do3Dmul))
      return fail(OBIT_DFT_EUNSUPPORTED, "field " + std::to_string(i) +
                                             ": 2-D image with a shift, rotation or offset centre");
    float dxyzc[3];
    shift_sin(model->uvRA, model->uvDec, maprot, f.crvalRA, f.crvalDec, dxyzc);
    float xpoff = 0.0f, ypoff = 0.0f;
    if (!model->do3D) {
      xpoff = f.xPxOff * f.cdeltX;
      ypoff = f.yPxOff * f.cdeltY;
    }
    const float xxoff = dxyzc[0] * ccrot + dxyzc[1] * ssrot;
    const float yyoff = dxyzc[1] * ccrot - dxyzc[0] * ssrot;
    const float zzoff = dxyzc[2];
    float U[3][3];
    if (do3Dmul) urot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, U);
    // FP64 positions: the same geometry with every step in double
    double Ud[3][3], dxyzd[3], xxoffd = 0.0, yyoffd = 0.0, zzoffd = 0.0, ssd = 0.0, ccd = 1.0;
    double xpoffd = 0.0, ypoffd = 0.0;
    const double konstd = kPi / 180.0 * 2.0 * kPi;
    if (xyzOut) {
      ssd = std::sin(kPi / 180.0 * ((double)uvrot - (double)maprot));
      ccd = std::cos(kPi / 180.0 * ((double)uvrot - (double)maprot));
      shift_sin_d(model->uvRA, model->uvDec, maprot, f.crvalRA, f.crvalDec, dxyzd);
      xxoffd = dxyzd[0] * ccd + dxyzd[1] * ssd;
      yyoffd = dxyzd[1] * ccd - dxyzd[0] * ssd;
      zzoffd = dxyzd[2];
      if (!model->do3D) {
        xpoffd = (double)f.xPxOff * (double)f.cdeltX;
        ypoffd = (double)f.yPxOff * (double)f.cdeltY;
      }
      if (do3Dmul) urot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, Ud);
    }
    // Gaussian terms from the first row's FWHM and PA (ObitSkyModel.c:1938-1947)
    float gp1 = 0.f, gp2 = 0.f, gp3 = 0.f;
    if (is_gauss(ftype)) {
      const float cpa = (float)std::cos(kPi / 180.0 * (double)parms[2]);
      const float spa = (float)std::sin(kPi / 180.0 * (double)parms[2]);
      const float xmaj = parms[0] * konst2, xmin = parms[1] * konst2;
      gp1 = -(((cpa * xmaj) * (cpa * xmaj)) + (spa * xmin) * (spa * xmin));
      gp2 = -(((spa * xmaj) * (spa * xmaj)) + (cpa * xmin) * (cpa * xmin));
      gp3 = (float)(-2.0 * (double)cpa * (double)spa * (double)(xmaj * xmaj - xmin * xmin));
    }
    for (const Entry& e : merged) {
      if (model->noNeg && e.flux <= 0.0f) break;
      const bool want = std::fabs(e.flux) > model->minDFT && std::fabs(e.flux) > model->minFlux &&
                        ncomp < count;
      if (!want) continue;
      row[0] = e.flux * model->factor;
      const float xp0 = (e.dx + xpoff) * konst;
      const float xp1 = (e.dy + ypoff) * konst;
      const float xp2 = f.deltaZ ? e.dz * konst : 0.0f;
      float xyz[3];
      if (do3Dmul) {
        xyz[0] = xp0 * U[0][0] + xp1 * U[1][0];
        xyz[1] = xp0 * U[0][1] + xp1 * U[1][1];
        xyz[2] = xp0 * U[0][2] + xp1 * U[1][2];
      } else {
        xyz[0] = ccrot * xp0 + ssrot * xp1;
        xyz[1] = ccrot * xp1 - ssrot * xp0;
        xyz[2] = xp2;
      }
      row[1] = xyz[0] + xxoff;
      row[2] = xyz[1] + yyoff;
      row[3] = xyz[2] + zzoff;
      if (xyzOut) {
        const double q0 = ((double)e.dx + xpoffd) * konstd;
        const double q1 = ((double)e.dy + ypoffd) * konstd;
        const double q2 = f.deltaZ ? (double)e.dz * konstd : 0.0;
        double* o = xyzOut + 3 * (size_t)ncomp;
        if (do3Dmul) {
          o[0] = q0 * Ud[0][0] + q1 * Ud[1][0] + xxoffd;
          o[1] = q0 * Ud[0][1] + q1 * Ud[1][1] + yyoffd;
          o[2] = q0 * Ud[0][2] + q1 * Ud[1][2] + zzoffd;
        } else {
          o[0] = ccd * q0 + ssd * q1 + xxoffd;
          o[1] = ccd * q1 - ssd * q0 + yyoffd;
          o[2] = q2 + zzoffd;
        }
      }
      // type-specific terms, mixed types zero what a field lacks (ObitSkyModel.c:1990-2083)
      const int g0 = 4, s0 = is_gauss(maxType) ? 7 : 4;
      if (is_gauss(maxType) && is_gauss(ftype)) {
        row[g0] = gp1;
        row[g0 + 1] = gp2;
        row[g0 + 2] = gp3;
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
