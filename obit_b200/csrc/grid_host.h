// Host-side plan of a gridded-model field (grid_host.cpp), consumed by the
// device half (grid_model.cu).
#pragma once
#include <vector>

#include "obit_dft_grid.h"

namespace obit {

constexpr int kGridHalfWidth = 12;                 // HWIDTH, ObitSkyModel.c:75
constexpr int kGridTaps = 2 * kGridHalfWidth + 1;  // taps per axis
constexpr int kGridTableRows = 201;                // 1 + 1 / 0.005, ObitCInterpolate.c:760
constexpr int kGridPadRows = 6;                    // zero rows after the plane (window unions)

// ObitTableCCUtilGrid's per-row constants (ObitTableCCUtil.c:140-176) for the
// device pass over a field's rows first .. first + count - 1 (0-relative, after
// the noNeg stop).
struct GridRows {
  int first = 0, count = 0;
  float factor = 1.f, minFlux = 0.f, maxGrid = 1e20f;
  float xpoff = 0.f, ypoff = 0.f, minX = 0.f, maxX = 0.f, minY = 0.f, maxY = 0.f;
  float iCellX = 1.f, iCellY = 1.f;
  int nx = 0, ny = 0;
};

struct GridHostPlan {
  int nx = 0, ny = 0;        // grid: OverSample x the image
  int nxp = 0;               // plane columns: nx / 2 + 1 + HWIDTH conjugate columns
  int pitch = 0;             // complex values per plane row in device memory (even, > nxp + 6)
  int rows = 0;              // plane rows in device memory: ny, then kGridPadRows zero rows
  GridRows rowsDesc;         // the component rows, gridded on the device
  int ncomp = 0, bad = 0;    // components gridded, off-cell warnings (set by the device pass)
  float gparm[3] = {-1.f, -1.f, -1.f};
  bool doGaus = false;
  float b1 = 0.f, b2 = 0.f, b3 = 0.f, dV = 0.f;
  std::vector<float> UU;     // u of each half-plane column, as the taper loop accumulates it
  float crpix0 = 0.f, crpix1 = 0.f, cdelt0 = 0.f, cdelt1 = 0.f;
  std::vector<float> table;  // kGridTableRows x kGridTaps
  float flip = 1.f;
  bool do3Dmul = false, doRot = false, doPC = false;
  float umat[3][3];
  float ccrot = 1.f, ssrot = 0.f;
  float dxyzc[3] = {0.f, 0.f, 0.f};
};

// The reference's Lagrange kernel table (kGridTableRows x kGridTaps).
void grid_kernel_table(std::vector<float>* tab);

// Everything of a field that is computed on the host.  Returns OBIT_DFT_OK or
// an error code with the last error set.
int grid_host_plan(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
                   float maxGrid, GridHostPlan* g);

// The same for an image model (no components: the field's rows are not read;
// the geometry, interpolator and table as for components; ncomp = pixels).
int grid_host_plan_image(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
                         GridHostPlan* g);

}  // namespace obit
