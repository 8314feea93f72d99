// Host half of the gridded model (include/obit_dft_grid.h): the component
// selection and gridding of ObitTableCCUtilGrid, the taper constants and
// interpolator set-up of ObitSkyModelGridFTComps / newObitCInterpolateCreate,
// the kernel table of InitConvKernal, the per-field geometry of
// ThreadSkyModelFTGrid, and the mode choice of ObitSkyModelChose.  Compiled
// without floating-point contraction: every single-precision step rounds where
// the reference's does, so that the grid cells, sums, table and constants are
// the reference's own.
#include "grid_host.h"

#include <cmath>
#include <string>

#include "abi_internal.h"
#include "sky_geom.h"

namespace obit {

namespace {

constexpr double kPi = geom::kGeomPi;
constexpr int kOverSample = 2;  // ObitSkyModel.c:71

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

bool gauss_type(int t) { return t == 1 || t == 2 || t == 11 || t == 12 || t == 21 || t == 22; }
bool disk_or_sphere(int t) { return t == 3 || t == 4 || t == 13 || t == 14 || t == 23 || t == 24; }

}  // namespace

// InitConvKernal / CalcConvKernal (ObitCInterpolate.c:747-830): Lagrange
// weights of 2 hwidth + 1 taps for 201 fractional positions, single precision.
void grid_kernel_table(std::vector<float>* tab) {
  constexpr int iwid = kGridTaps;
  float denom[iwid];
  for (int j = 1; j <= iwid; j++) {
    float prod = 1.0f;
    for (int i = 1; i <= iwid; i++)
      if (i != j) prod = prod * (float)(j - i);
    denom[j - 1] = (float)(1.0 / (double)prod);
  }
  const float ks = 0.005f;
  const int num = (int)(1 + (1.0 / (double)ks) + 0.5);
  tab->assign((size_t)num * iwid, 0.0f);
  for (int k = 0; k < num; k++) {
    const float xx = (float)((double)((float)kGridHalfWidth + ks * (float)(k - 1)) + 0.5);
    const int ipos = (int)((double)xx + 0.5);
    int cen = ipos - kGridHalfWidth;
    cen = std::max(1, std::min(cen, 1024 - iwid));
    cen--;
    const float x = (float)((double)(xx - (float)cen) + 1.0);
    for (int j = 0; j < iwid; j++) {
      float prod = denom[j];
      for (int i = 0; i < iwid; i++)
        if (i != j) prod = prod * (x - (float)(i + 1));
      (*tab)[(size_t)k * iwid + j] = prod;
    }
  }
}

namespace {

// The plan of a field: with components (ObitSkyModelGridFTComps) or, for an
// image model (ObitSkyModelLoadImage), everything but the gridding.
int plan_field(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
               float maxGrid, bool withComps, GridHostPlan* g) {
  if (!field || !image || !model || !g) return fail(OBIT_DFT_EBADARG, "grid: null argument");
  const ObitDFTCCField& f = *field;
  // the conjugate columns of row 0 read columns up to 2 HWIDTH of the half plane
  if (image->nx < 2 * kGridHalfWidth || image->ny < 2 * kGridHalfWidth)
    return fail(OBIT_DFT_EBADARG, "grid: image smaller than the interpolation kernel");
  if ((long long)image->nx * image->ny > (1LL << 28))
    return fail(OBIT_DFT_EBADARG, "grid: image larger than 2^28 pixels");
  if (withComps && (f.nrow < 0 || (f.nrow > 0 && (!f.flux || !f.deltaX || !f.deltaY))))
    return fail(OBIT_DFT_EBADARG, "grid: missing CC columns");
  if (f.ncpProjection) return fail(OBIT_DFT_EUNSUPPORTED, "grid: -NCP fields are not supported");
  const float maprot = f.rotation, uvrot = model->uvRotation;
  const bool off3d = maprot != 0.0f || uvrot != 0.0f || std::fabs(f.crvalRA - model->uvRA) > 1.0e-10 ||
                     std::fabs(f.crvalDec - model->uvDec) > 1.0e-10 || std::fabs(f.xPxOff) > 1.0e-20f ||
                     std::fabs(f.yPxOff) > 1.0e-20f;
  if (!f.do3D && (f.xShift != 0.0f || f.yShift != 0.0f || off3d))
    return fail(OBIT_DFT_EUNSUPPORTED, "grid: 2-D image with a shift, rotation or offset centre");

  // ---- ObitTableCCUtilGrid (ObitTableCCUtil.c:106-302) ----
  const int nx = kOverSample * image->nx, ny = kOverSample * image->ny;
  g->nx = nx;
  g->ny = ny;
  const float cdx = f.cdeltX, cdy = f.cdeltY;
  const float fNx = (float)nx, fNy = (float)ny;
  const float minX = (float)((-fNx / 2.0) * std::fabs((double)cdx));
  const float maxX = (float)(((fNx / 2.0) - 1.0) * std::fabs((double)cdx));
  const float minY = (float)((-fNy / 2.0) * std::fabs((double)cdy));
  const float maxY = (float)(((fNy / 2.0) - 1.0) * std::fabs((double)cdy));
  const float iCellX = cdx != 0.0f ? (float)(1.0 / (double)cdx) : 1.0f;
  const float iCellY = cdy != 0.0f ? (float)(1.0 / (double)cdy) : 1.0f;
  const float xpoff = (image->crpixX - (float)(image->nx / 2) - 1.0f) * cdx;
  const float ypoff = (image->crpixY - (float)(image->ny / 2) - 1.0f) * cdy;
  int first = f.startComp > 0 ? f.startComp : 1;
  int last = f.endComp > 0 ? f.endComp : f.nrow;
  last = std::min(last, f.nrow);
  g->gparm[0] = g->gparm[1] = g->gparm[2] = -1.0f;
  bool isGauss = false;
  g->ncomp = g->bad = 0;
  if (!withComps) last = first - 1;  // image model: no rows
  // The reference's row loop up to the point where each row's cell is found:
  // the model type of the first row, one Gaussian size for all, and the stop
  // at the first negative flux (noNeg).  The rows' cells and sums are formed
  // on the device (grid_rows_kernel) with the constants below.
  int stop = last;
  for (int j = first; j <= last; j++) {
    const size_t k = (size_t)j - 1;
    const float* pr = (f.parms && f.nparms > 0) ? f.parms + k * f.nparms : nullptr;
    if (j == first) {
      if (pr && f.nparms >= 4) {
        const int mtype = (int)pr[3];  // (ObitCCCompType)PARMS[3] + 0.5 truncates twice
        if (disk_or_sphere(mtype))
          return fail(OBIT_DFT_EUNSUPPORTED, "grid: exponential disks and uniform spheres are not supported");
        if (gauss_type(mtype)) {
          g->gparm[0] = pr[0];
          g->gparm[1] = pr[1];
          g->gparm[2] = pr[2];
          isGauss = true;
        }
      }
    } else if (isGauss && (pr[0] != g->gparm[0] || pr[1] != g->gparm[1] || pr[2] != g->gparm[2])) {
      return fail(OBIT_DFT_EBADARG, "grid: all Gaussians of a field must have the same size");
    }
    if (model->noNeg && f.flux[k] < 0.0f) {
      stop = j - 1;
      break;
    }
  }
  GridRows& r = g->rowsDesc;
  r.first = first - 1;
  r.count = std::max(0, stop - first + 1);
  r.factor = model->factor;
  r.minFlux = model->minFlux;
  r.maxGrid = maxGrid;
  r.xpoff = xpoff;
  r.ypoff = ypoff;
  r.minX = minX;
  r.maxX = maxX;
  r.minY = minY;
  r.maxY = maxY;
  r.iCellX = iCellX;
  r.iCellY = iCellY;
  r.nx = nx;
  r.ny = ny;

  // ---- taper constants (ObitSkyModel.c:4291-4310) ----
  g->doGaus = g->gparm[0] > 0.0f || g->gparm[1] > 0.0f;
  g->UU.clear();
  if (g->doGaus) {
    const double d2r = kPi / 180.0, r2d = 180.0 / kPi;
    g->dV = (float)(r2d / ((double)ny * std::fabs((double)cdy)));
    const float dU = (float)(r2d / ((double)nx * std::fabs((double)cdx)));
    const float konst = (float)(d2r * kPi * std::sqrt(0.5) / 1.17741022);
    const float xmaj = g->gparm[0] * konst, xmin = g->gparm[1] * konst;
    const float cpa = (float)std::cos(d2r * (90.0 + (double)g->gparm[2]));
    const float spa = (float)std::sin(d2r * (90.0 + (double)g->gparm[2]));
    g->b1 = -(((cpa * xmaj) * (cpa * xmaj)) + ((spa * xmin) * (spa * xmin)));
    g->b2 = -(((spa * xmaj) * (spa * xmaj)) + ((cpa * xmin) * (cpa * xmin)));
    g->b3 = (float)(-2.0 * (double)spa * (double)cpa * (double)(xmaj * xmaj - xmin * xmin));
    // UU advances by repeated single-precision addition along each row
    float uu = 0.0f;
    for (int j = 0; j < nx / 2 + 1; j++) {
      g->UU.push_back(uu);
      uu = uu + dU;
    }
  }

  // ---- interpolator (ObitCInterpolate.c:128-206 with ObitSkyModel.c:4354-4358) ----
  g->nxp = nx / 2 + 1 + kGridHalfWidth;
  // even (16-byte rows for pair loads), with zero columns past the last one for
  // the apply kernel's window unions, which may reach 7 columns beyond it
  g->pitch = (g->nxp + 8) & ~1;
  g->rows = ny + kGridPadRows;
  g->crpix0 = (float)kGridHalfWidth;
  g->crpix1 = (float)(ny / 2);
  g->cdelt0 = (float)(1.0 / ((-kPi / 180.0) * (double)(float)kOverSample * (double)cdx * (double)image->nx));
  g->cdelt1 = (float)(1.0 / ((-kPi / 180.0) * (double)(float)kOverSample * (double)cdy * (double)image->ny));
  grid_kernel_table(&g->table);

  // ---- geometry of ThreadSkyModelFTGrid (ObitSkyModel.c:3037-3101) ----
  g->ssrot = (float)std::sin(kPi / 180.0 * (double)(uvrot - maprot));
  g->ccrot = (float)std::cos(kPi / 180.0 * (double)(uvrot - maprot));
  g->flip = cdx > 0.0f ? -1.0f : 1.0f;
  // ObitUVDescShiftPhase: 3-D fields from their reference position; the
  // supported 2-D fields sit on the phase centre, so the shift is zero
  geom::shift_sin(model->uvRA, model->uvDec, maprot, f.do3D ? f.crvalRA : model->uvRA,
                  f.do3D ? f.crvalDec : model->uvDec, g->dxyzc);
  g->doPC = std::fabs(g->dxyzc[0]) > 1.0e-12f || std::fabs(g->dxyzc[1]) > 1.0e-12f ||
            std::fabs(g->dxyzc[2]) > 1.0e-12f;
  g->do3Dmul = false;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g->umat[i][j] = i == j ? 1.0f : 0.0f;
  if (model->do3D) {
    g->do3Dmul = off3d;
    float pmat[3][3];
    geom::urot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, g->umat);
    geom::prot3d(model->uvRA, model->uvDec, f.crvalRA, f.crvalDec, maprot, uvrot, pmat);
    if (g->doPC) {
      // rmat[0][0] = cc, rmat[1][0] = ss, rmat[0][1] = -ss, rmat[1][1] = cc (ObitSkyModel.c:3066-3068)
      const float rmat[3][3] = {{g->ccrot, -g->ssrot, 0.0f}, {g->ssrot, g->ccrot, 0.0f}, {0.0f, 0.0f, 1.0f}};
      float dmat[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          dmat[j][i] = 0.0f;
          for (int k = 0; k < 3; k++) dmat[j][i] += pmat[k][i] * rmat[j][k];
        }
      const float* d = g->dxyzc;
      float r[3];
      for (int c = 0; c < 3; c++) r[c] = d[0] * dmat[0][c] + d[1] * dmat[1][c] + d[2] * dmat[2][c];
      for (int c = 0; c < 3; c++) g->dxyzc[c] = r[c];
    }
  }
  g->doRot = std::fabs((double)g->ssrot) > 1.0e-10 || std::fabs((double)g->ccrot - 1.0) > 1.0e-4;
  return OBIT_DFT_OK;
}

}  // namespace

int grid_host_plan(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
                   float maxGrid, GridHostPlan* g) {
  return plan_field(field, image, model, maxGrid, true, g);
}

int grid_host_plan_image(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
                         GridHostPlan* g) {
  if (image && image->nx != image->ny)
    return fail(OBIT_DFT_EUNSUPPORTED, "grid: image models must be square (the reference sizes the FFT "
                                       "output from the transposed axes)");
  const int rc = plan_field(field, image, model, 1e20f, false, g);
  if (rc) return rc;
  g->ncomp = image->nx * image->ny;  // the reference always models an image field
  g->rowsDesc.count = 0;
  return OBIT_DFT_OK;
}

}  // namespace obit

// ObitSkyModelChose (ObitSkyModel.c:3560-3620).
extern "C" int obit_dft_choose_mode(int modelMode, int modelType, const int* ncc, const int* nx, const int* ny,
                                    int nfield, long long nvis, int nchan) {
  if (modelMode != 0) return modelMode;
  if (modelType == 2) return 1;
  const float tpvgrd = 1.0e-5f, tfft = 0.8e-6f, tpcgrd = 1.0e-4f, tpvpc = 6.6e-7f;
  long long sumcc = 0, t1 = 0, t2 = 0, t3 = 0;
  for (int i = 0; i < nfield; i++) {
    const int n = ncc ? ncc[i] : 0;
    if (n > 0) {
      const int x = (nx[i] > 2048 || ny[i] > 2048) ? 2 : 4;
      sumcc += n;
      t1 += nvis;
      t2 += (long long)x * nx[i] * ny[i];
      t3 += n;
    }
  }
  float timfft = ((float)t1 * tpvgrd + (float)t2 * tfft + (float)t3 * tpcgrd) * (float)nchan;
  timfft *= 0.50f;
  const float timdft = tpvpc * (float)nvis * (float)sumcc * (float)nchan;
  int mode = timdft <= timfft ? 1 : 2;
  if (modelType == 1) mode = 2;
  return mode;
}

extern "C" int obit_dft_choose_mode_measured(int modelType, const int* ncc, const int* nx, const int* ny,
                                             int nfield, long long nvis, int nchan, double dftRate,
                                             double gridRate, double gridSetup) {
  (void)nx;
  (void)ny;
  if (modelType == 1) return 2;
  if (modelType == 2) return 1;
  if (dftRate <= 0.0) dftRate = 4.5e12;
  if (gridRate <= 0.0) gridRate = 3.5e9;
  if (gridSetup <= 0.0) gridSetup = 0.01;
  double tdft = 0.0, tgrid = 0.0;
  const double vis = (double)nvis * (double)nchan;
  for (int i = 0; i < nfield; i++) {
    const int n = ncc ? ncc[i] : 0;
    if (n <= 0) continue;
    tdft += (double)n * vis / dftRate;
    tgrid += vis / gridRate + gridSetup;
  }
  return tdft <= tgrid ? 1 : 2;
}
