// Translation of the reference-layout descriptors into planner descriptions
// (see abi_internal.h).
#include <algorithm>
#include <cmath>

#include "abi_internal.h"

namespace obit {

namespace {
thread_local std::string g_last_error;

int bad(std::string* err, int code, const std::string& msg) {
  *err = msg;
  return code;
}

// Device -> host copy, blocking on the legacy default stream, or ordered on
// *order and then synchronized with it.
cudaError_t read_device(void* dst, const void* src, size_t bytes, const cudaStream_t* order) {
  if (!order) return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
  cudaError_t ce = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, *order);
  return ce == cudaSuccess ? cudaStreamSynchronize(*order) : ce;
}
}  // namespace

int kernel_flag_status(int flag, std::string* msg) {
  if (!flag) return OBIT_DFT_OK;
  const char* what = flag == 2   ? ": a component-tile copy did not complete within the wait limit"
                     : flag == 3 ? ": a record's antenna number is outside the beam's antenna table"
                     : flag == 5 ? ": a component-tile copy was still in flight when a CTA gave up; "
                                   "the CUDA context must be treated as unusable"
                                 : "";
  *msg = "kernel reported internal error code " + std::to_string(flag) + what;
  return flag == 5 ? OBIT_DFT_ECUDA : OBIT_DFT_EKERNEL;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

int model_from_info(const GPUModelInfo* m, int ncomp, int lcomp, const GPUVisInfo* v, ModelCfg* mc,
                    std::string* err, const cudaStream_t* order) {
  if (!m) return bad(err, OBIT_DFT_EBADARG, "GPUModelInfo is NULL");
  ModelDesc md;
  md.kind = (int)m->type;
  md.nterm = m->nterm;
  md.lcomp = lcomp;
  md.ncomp = ncomp;
  if (md.kind < kPoint || md.kind > kGaussTSpec)
    return bad(err, OBIT_DFT_EUNSUPPORTED, "model type " + std::to_string(md.kind) + " not supported");
  if (md.ncomp < 0) return bad(err, OBIT_DFT_EBADARG, "negative component count");
  const bool spec = (md.kind == kPointSpec || md.kind == kGaussSpec);
  const bool tspec = (md.kind == kPointTSpec || md.kind == kGaussTSpec);
  const bool gauss = (md.kind >= kGauss);
  int minLen = gauss ? 7 : 4;
  if (spec) minLen += md.nterm;
  if (tspec) minLen = (gauss ? 8 : 5) + 1;
  if (md.ncomp > 0 && md.lcomp < minLen)
    return bad(err, OBIT_DFT_EBADARG, "component record shorter than the model type needs");
  if (spec && (md.nterm < 1 || md.nterm > kMaxNTerm))
    return bad(err, OBIT_DFT_EUNSUPPORTED,
               "spectral term count must be 1.." + std::to_string(kMaxNTerm));
  md.nspec = tspec ? md.lcomp - (gauss ? 8 : 5) : 0;
  mc->model = md;
  mc->opType = (int)m->opType;
  mc->doSwap = m->doSwap;
  for (int i = 0; i < 4; i++) mc->stokFact[i] = m->stokFact[i];
  mc->specIndex.clear();
  if (tspec) {
    if (!v) return bad(err, OBIT_DFT_EBADARG, "GPUVisInfo is NULL");
    const int nfreq = v->nchan * std::max(1, v->nIF);
    if (m->specIndex) {
      mc->specIndex.assign(m->specIndex, m->specIndex + nfreq);
    } else if (m->d_specIndex) {
      mc->specIndex.resize(nfreq);
      cudaError_t ce = read_device(mc->specIndex.data(), m->d_specIndex, sizeof(int) * nfreq, order);
      if (ce != cudaSuccess)
        return bad(err, OBIT_DFT_ECUDA, std::string("specIndex copy: ") + cudaGetErrorString(ce));
    } else {
      return bad(err, OBIT_DFT_EBADARG, "tabulated spectra need specIndex");
    }
  }
  return OBIT_DFT_OK;
}

int layout_from_info(const GPUVisInfo* v, const ModelCfg& mc, const FreqSide& fs, LayoutDesc* L,
                     std::string* err, const cudaStream_t* order) {
  if (!v) return bad(err, OBIT_DFT_EBADARG, "GPUVisInfo is NULL");
  L->lrec = v->lenvis;
  L->nrparm = v->nrparm;
  L->ilocu = v->ilocu;
  L->ilocv = v->ilocv;
  L->ilocw = v->ilocw;
  L->nchan = v->nchan;
  L->nif = std::max(1, v->nIF);
  L->nstok = v->nstok;
  L->incs = 3 * v->incs;
  L->incf = 3 * v->incf;
  L->incif = 3 * v->incif;
  L->kincf = v->kincf;
  L->kincif = v->kincif;
  L->chanb = v->chanb;
  L->chane = v->chane;
  L->ifb = v->IFb;
  L->ife = v->IFe;
  L->stokb = v->stokb;
  L->stoke = v->stoke;
  if (L->lrec <= 0 || L->nchan <= 0 || L->nstok <= 0)
    return bad(err, OBIT_DFT_EBADARG,
               "record length, channel and polarization counts must be positive");
  if (L->chanb < 0 || L->chane < L->chanb || L->chane >= L->nchan || L->ifb < 0 || L->ife < L->ifb ||
      L->ife >= L->nif || L->stokb < 0 || L->stoke < L->stokb || L->stoke >= L->nstok)
    return bad(err, OBIT_DFT_EBADARG, "channel, IF or polarization selection outside the data");
  const int nfreq = L->nchan * L->nif;
  // every selected product must lie inside the record
  const long long lastOff = (long long)L->nrparm + (long long)L->ife * L->incif +
                            (long long)L->chane * L->incf + (long long)L->stoke * L->incs + 2;
  if (lastOff >= L->lrec) return bad(err, OBIT_DFT_EBADARG, "selected products extend past the record");
  if (L->ilocu < 0 || L->ilocu >= L->nrparm || L->ilocv < 0 || L->ilocv >= L->nrparm ||
      L->ilocw < 0 || L->ilocw >= L->nrparm)
    return bad(err, OBIT_DFT_EBADARG, "u/v/w offsets must index random parameters");
  L->fscale.assign(nfreq, 1.0);
  if (fs.have) {
    if ((int)fs.freqArr.size() < nfreq) return bad(err, OBIT_DFT_EBADARG, "FP64 frequency table too short");
    for (int i = 0; i < nfreq; i++) L->fscale[i] = fs.freqArr[i] / fs.uvRef;
  } else {
    if (!v->freqScale) return bad(err, OBIT_DFT_EBADARG, "GPUVisInfo.freqScale is NULL");
    std::vector<float> f32(nfreq);
    cudaError_t ce = read_device(f32.data(), v->freqScale, sizeof(float) * nfreq, order);
    if (ce != cudaSuccess)
      return bad(err, OBIT_DFT_ECUDA, std::string("freqScale copy: ") + cudaGetErrorString(ce));
    for (int i = 0; i < nfreq; i++) L->fscale[i] = (double)f32[i];
  }
  const int kind = mc.model.kind;
  if (kind == kPointSpec || kind == kGaussSpec) {
    L->lnspec.assign(nfreq, 0.0);
    for (int i = 0; i < nfreq; i++) {
      double r;
      if (fs.have)
        r = fs.freqArr[i] / (fs.modelRef > 0 ? fs.modelRef : fs.uvRef);
      else
        r = L->fscale[i] * (v->freqRat ? (double)v->freqRat[0] : 1.0);
      L->lnspec[i] = std::log(r);
    }
  } else if (kind == kPointTSpec || kind == kGaussTSpec) {
    if ((int)mc.specIndex.size() < nfreq)
      return bad(err, OBIT_DFT_EBADARG, "tabulated spectra need GPUModelInfo.specIndex");
    L->specIndex = mc.specIndex;
    L->lnspec.assign(nfreq, 0.0);
    for (int i = 0; i < nfreq; i++) {
      const int pl = mc.specIndex[i];
      if (pl < 0 || pl >= mc.model.nspec)
        return bad(err, OBIT_DFT_EBADARG, "specIndex outside the component's plane table");
      double r;
      if (fs.have && (int)fs.specFreq.size() > pl)
        r = fs.freqArr[i] / fs.specFreq[pl];
      else if (v->freqRat)
        r = L->fscale[i] * (double)v->freqRat[pl];
      else
        return bad(err, OBIT_DFT_EBADARG, "tabulated spectra need freqRat or specFreq");
      L->lnspec[i] = std::log(r);
    }
  }
  return OBIT_DFT_OK;
}

int apply_from_info(const ModelCfg& mc, const PolnRules& pr, const LayoutDesc& L, ApplyDesc* A,
                    std::string* err) {
  A->op = mc.opType;
  if (A->op < 0 || A->op > 2) return bad(err, OBIT_DFT_EBADARG, "unknown operation type");
  if (pr.cpuRules) {
    A->cumulative = 1;
    A->stokFactor = pr.stokFactor;
    for (int j = 0; j < kMaxPol; j++) A->polFact[j] = 1.0f;
    A->flipMask = pr.doFlip ? 0xF : 0;
  } else {
    // GPUModelInfo semantics: stokFact per polarization, doSwap on pol 3 only
    A->cumulative = 0;
    A->stokFactor = 1.0f;
    for (int j = 0; j < kMaxPol; j++) {
      const int ist = L.stokb + j;
      A->polFact[j] = (ist < 4) ? mc.stokFact[ist] : 1.0f;
    }
    A->flipMask = 0;
    if (mc.doSwap && L.stokb <= 3 && L.stoke >= 3) A->flipMask = 1 << (3 - L.stokb);
  }
  return OBIT_DFT_OK;
}

int copy_comps(float* dst, const float* src, const ModelDesc& md, cudaStream_t stream,
               std::string* err) {
  if (md.ncomp <= 0) return OBIT_DFT_OK;
  if (!src) return bad(err, OBIT_DFT_EBADARG, "device component table is NULL");
  const size_t stride = (size_t)comp_stride(md);
  cudaError_t ce = cudaMemsetAsync(dst, 0, (size_t)md.ncomp * stride * sizeof(float), stream);
  if (ce == cudaSuccess)
    ce = cudaMemcpy2DAsync(dst, stride * sizeof(float), src, (size_t)md.lcomp * sizeof(float),
                           (size_t)md.lcomp * sizeof(float), (size_t)md.ncomp,
                           cudaMemcpyDeviceToDevice, stream);
  if (ce != cudaSuccess)
    return bad(err, OBIT_DFT_ECUDA, std::string("component copy: ") + cudaGetErrorString(ce));
  return OBIT_DFT_OK;
}

}  // namespace obit
