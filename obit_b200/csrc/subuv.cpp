// ObitSkyModelSubUV's pass structure (ObitSkyModel.c:850-1087) over this
// library's GPU paths: the mode choice, one DFT pass over every field's
// components, a gridded pass per field, or both per field (Mixed).  Host code
// over the C ABI; see include/obit_dft_subuv.h.
#include "obit_dft_subuv.h"

#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

namespace {

int set_err(ObitDFTErr* err, int code, const char* fmt, ...) {
  if (err) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err->message, sizeof(err->message), fmt, ap);
    va_end(ap);
    err->error = 1;
  }
  return code;
}

// The library's own message for a failed call, or the mirror's.
int lib_err(ObitDFTErr* err, int code, const char* what) {
  return set_err(err, code, "obit_dft_sub_uv: %s: %s", what, obit_dft_last_error());
}

struct MirrorDeleter {
  void operator()(ObitDFTGPUSkyModel* in) const {
    if (in) {
      ObitDFTErr e{};
      obit_gpu_skymodel_dft_shutdown(in, &e);
      obit_gpu_skymodel_unref(in);
    }
  }
};
using Mirror = std::unique_ptr<ObitDFTGPUSkyModel, MirrorDeleter>;

struct GridDeleter {
  void operator()(ObitDFTGrid* g) const {
    if (g) obit_dft_grid_destroy(g);
  }
};

// One DFT pass over the components of `fields` (one table, the ObitGPUSkyModel
// mirror); *ncomp receives the merged component rows.
int dft_pass(const ObitDFTCCField* fields, int nfield, const ObitDFTCCModel* model, const ObitDFTSkyModel* sky,
             ObitDFTUVData* uv, int* ncompOut, ObitDFTErr* err) {
  int nrow = 0, ncomp = 0, lcomp = 0, modType = 0, nterm = 0;
  int rc = obit_dft_load_comps(fields, nfield, model, nullptr, 0, &nrow, &ncomp, &lcomp, &modType, &nterm);
  if (rc) return lib_err(err, rc, "component table");
  std::vector<float> table((size_t)std::max(1, nrow) * std::max(1, lcomp));
  rc = obit_dft_load_comps(fields, nfield, model, table.data(), (long long)table.size(), &nrow, &ncomp, &lcomp,
                           &modType, &nterm);
  if (rc) return lib_err(err, rc, "component table");
  *ncompOut = ncomp;
  const int nvis = uv->numVisBuff;
  if (ncomp <= 0 || nvis <= 0) return OBIT_DFT_OK;
  ObitDFTSkyModel s = *sky;
  s.modType = modType;
  s.nSpecTerm = nterm;
  s.nVisPIO = std::max(1, nvis);
  Mirror in(obit_gpu_skymodel_create("subuv"));
  if (!in) return set_err(err, OBIT_DFT_ECUDA, "obit_dft_sub_uv: cannot create the GPU sky model");
  if (obit_gpu_skymodel_dft_init(in.get(), &s, uv, err)) return OBIT_DFT_EBADARG;
  if (obit_gpu_skymodel_dft_setmod(in.get(), &s, table.data(), lcomp, ncomp, err)) return OBIT_DFT_EBADARG;
  if (obit_gpu_skymodel_dft_calc(in.get(), uv, err)) return OBIT_DFT_EKERNEL;
  return OBIT_DFT_OK;
}

// The records' layout and selection as a GPUVisInfo, from a mirror instance
// (held by `in` while the descriptor is used).
int grid_descriptor(const ObitDFTSkyModel* sky, ObitDFTUVData* uv, Mirror* in, const GPUVisInfo** vi,
                    ObitDFTErr* err) {
  ObitDFTSkyModel s = *sky;
  s.modType = 0;
  s.nSpecTerm = 0;
  s.nVisPIO = 1;
  in->reset(obit_gpu_skymodel_create("subuv-grid"));
  if (!*in) return set_err(err, OBIT_DFT_ECUDA, "obit_dft_sub_uv: cannot create the GPU sky model");
  if (obit_gpu_skymodel_dft_init(in->get(), &s, uv, err)) return OBIT_DFT_EBADARG;
  *vi = obit_gpu_skymodel_info(in->get())->h_visInfo;
  return OBIT_DFT_OK;
}

// One gridded pass of a field: its components of at most maxGrid, or, with
// pixels, its model image; *nrow receives the rows (pixels) gridded.
int grid_pass(const ObitDFTCCField* field, const ObitDFTGridImage* image, const ObitDFTCCModel* model,
              float maxGrid, int kernel, const GPUVisInfo* vi, const ObitDFTSkyModel* sky, ObitDFTUVData* uv,
              long long* nrow, ObitDFTErr* err, const float* pixels = nullptr, float fblank = 0.0f) {
  ObitDFTGrid* raw = nullptr;
  int rc = pixels ? obit_dft_grid_create_image(pixels, fblank, field, image, model, kernel, nullptr, &raw)
                  : obit_dft_grid_create(field, image, model, maxGrid, kernel, nullptr, &raw);
  if (rc) return lib_err(err, rc, "gridded field");
  std::unique_ptr<ObitDFTGrid, GridDeleter> grid(raw);
  long long info[1] = {0};
  if ((rc = obit_dft_grid_info(grid.get(), info, 1))) return lib_err(err, rc, "gridded field");
  *nrow = info[0];
  if (info[0] <= 0) return OBIT_DFT_OK;
  const int opType = sky->doReplace ? 2 : (sky->doDivide ? 1 : 0);
  rc = obit_dft_grid_apply_host(grid.get(), vi, opType, sky->stokFactor, sky->doFlip, uv->buffer,
                                uv->numVisBuff, nullptr);
  if (rc) return lib_err(err, rc, "gridded pass");
  return OBIT_DFT_OK;
}

}  // namespace

extern "C" int obit_dft_sub_uv(const ObitDFTCCField* fields, int nfield, const ObitDFTGridImage* images,
                               const ObitDFTCCModel* model, const ObitDFTSkyModel* sky, ObitDFTUVData* uv,
                               int mode, int measured, float maxGrid, int kernel, int* modeUsed,
                               int* ncompUsed, ObitDFTErr* err) {
  if (!fields || nfield < 1 || !model || !sky || !uv || !uv->buffer)
    return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv: NULL argument or no fields");
  if (uv->jlocf < 0 || uv->jlocf > 6 || (uv->jlocif > 6))
    return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv: uv descriptor without a frequency axis");
  if (mode < 0 || mode > 3)
    return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv: mode %d is not 0, 1, 2 or 3", mode);
  const int nvis = uv->numVisBuff;
  const int nchan = uv->inaxes[uv->jlocf] * (uv->jlocif >= 0 ? uv->inaxes[uv->jlocif] : 1);
  // components per field (the selected CC rows) and image sizes for the choice
  std::vector<int> ncc(nfield), nx(nfield, 0), ny(nfield, 0);
  for (int f = 0; f < nfield; f++) {
    const int first = fields[f].startComp > 0 ? fields[f].startComp : 1;
    const int last = fields[f].endComp > 0 ? fields[f].endComp : fields[f].nrow;
    ncc[f] = std::max(0, last - first + 1);
    if (images) {
      nx[f] = images[f].nx;
      ny[f] = images[f].ny;
    }
  }
  int use = mode;
  if (mode == 0) {
    if (!images) return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv: choosing a mode needs the images");
    use = measured ? obit_dft_choose_mode_measured(0, ncc.data(), nx.data(), ny.data(), nfield, nvis, nchan,
                                                   0.0, 0.0, 0.0)
                   : obit_dft_choose_mode(0, 0, ncc.data(), nx.data(), ny.data(), nfield, nvis, nchan);
  }
  if (modeUsed) *modeUsed = use;
  if (ncompUsed) *ncompUsed = 0;

  if (use == 1) {  // DFT: all fields' components in one table, one pass
    int n = 0;
    const int rc = dft_pass(fields, nfield, model, sky, uv, &n, err);
    if (ncompUsed) *ncompUsed = n;
    return rc;
  }
  if (use != 2 && use != 3)
    return set_err(err, OBIT_DFT_EUNSUPPORTED, "obit_dft_sub_uv: mode %d is not supported", use);
  if (!images) return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv: the gridded model needs the images");
  if (nvis <= 0) return OBIT_DFT_OK;
  Mirror in;
  const GPUVisInfo* vi = nullptr;
  if (int rc = grid_descriptor(sky, uv, &in, &vi, err)) return rc;
  long long total = 0;
  for (int f = 0; f < nfield; f++) {  // a pass per field, in field order
    if (use == 3) {  // Mixed: the field's components above minDFT by the DFT first
      int n = 0;
      if (int rc = dft_pass(&fields[f], 1, model, sky, uv, &n, err)) return rc;
      total += n;
    }
    long long n = 0;
    if (int rc = grid_pass(&fields[f], &images[f], model, maxGrid, kernel, vi, sky, uv, &n, err)) return rc;
    total += n;
  }
  if (ncompUsed) *ncompUsed = (int)total;
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_sub_uv_image(const float* const* pixels, float fblank, const ObitDFTCCField* fields,
                                     int nfield, const ObitDFTGridImage* images, const ObitDFTCCModel* model,
                                     const ObitDFTSkyModel* sky, ObitDFTUVData* uv, int kernel,
                                     long long* npixUsed, ObitDFTErr* err) {
  if (!pixels || !fields || !images || nfield < 1 || !model || !sky || !uv || !uv->buffer)
    return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv_image: NULL argument or no fields");
  if (npixUsed) *npixUsed = 0;
  for (int f = 0; f < nfield; f++)
    if (!pixels[f]) return set_err(err, OBIT_DFT_EBADARG, "obit_dft_sub_uv_image: field %d has no pixels", f);
  if (uv->numVisBuff <= 0) return OBIT_DFT_OK;
  Mirror in;
  const GPUVisInfo* vi = nullptr;
  if (int rc = grid_descriptor(sky, uv, &in, &vi, err)) return rc;
  long long total = 0;
  for (int f = 0; f < nfield; f++) {  // a pass per field, in field order
    long long n = 0;
    if (int rc = grid_pass(&fields[f], &images[f], model, 1e20f, kernel, vi, sky, uv, &n, err, pixels[f], fblank))
      return rc;
    total += n;
  }
  if (npixUsed) *npixUsed = total;
  return OBIT_DFT_OK;
}
