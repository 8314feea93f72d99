// C ABI of libobit_dft.so (include/obit_dft.h): the reference's CUDA-layer
// entry points and their status-returning forms.
//
// Library state is kept per GPUInfo* in a registry; the GPUInfo itself is
// owned by the caller (ObitGPUSkyModel.c or the host mirror in this package),
// exactly as in the reference, and is only read here.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "obit_dft.h"
#include "dft_plan.h"

namespace {

using namespace obit;

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess)                                                          \
      return fail(OBIT_DFT_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)

struct State {
  int device = 0;
  // FP64 frequency side table
  bool haveFreqD = false;
  std::vector<double> freqArr, specFreq;
  double uvRef = 0.0, modelRef = 0.0;
  // CPU-reference polarization rules
  bool cpuRules = false;
  float stokFactor = 1.0f;
  int doFlip = 0;
  // kernel choice
  TuneDesc tune;
  // model
  ModelDesc model;
  int opType = 0, doSwap = 0;
  float stokFact[4] = {1.f, 1.f, 1.f, 1.f};
  std::vector<int> specIndex;
  float* d_comps = nullptr;
  size_t compBytes = 0;
  bool haveModel = false;
  // plan
  Plan plan;
  bool planValid = false;
  int planNvis = -1;
  // staging
  int bufRows = 0;                 // rows per device staging buffer
  std::vector<float*> ownBufs;     // used when the caller supplies none
  std::vector<cudaStream_t> ownStreams;
  int* d_err = nullptr;
};

std::mutex g_mu;
std::unordered_map<const GPUInfo*, std::unique_ptr<State>> g_states;

State* find_state(const GPUInfo* g) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_states.find(g);
  return it == g_states.end() ? nullptr : it->second.get();
}

int ensure_state(GPUInfo* g, State** out) {
  if (!g) return fail(OBIT_DFT_EBADARG, "NULL GPUInfo");
  State* s = find_state(g);
  if (!s) {
    std::unique_ptr<State> ns(new State());
    ns->device = g->cuda_device;
    CUDA_TRY(cudaSetDevice(ns->device));
    CUDA_TRY(cudaMalloc(&ns->d_err, sizeof(int)));
    CUDA_TRY(cudaMemset(ns->d_err, 0, sizeof(int)));
    ns->bufRows = 0;
    if (g->nstream > 0 && g->lenvis > 0 && g->nvis > 0)
      ns->bufRows = (int)(((long long)(g->nvis + 3) * g->lenvis / g->nstream) / g->lenvis);
    s = ns.get();
    std::lock_guard<std::mutex> lk(g_mu);
    g_states[g] = std::move(ns);
  } else {
    CUDA_TRY(cudaSetDevice(s->device));
  }
  *out = s;
  return OBIT_DFT_OK;
}

void release_state(State* s) {
  cudaSetDevice(s->device);
  free_plan(&s->plan);
  if (s->d_comps) cudaFree(s->d_comps);
  if (s->d_err) cudaFree(s->d_err);
  for (float* b : s->ownBufs) cudaFree(b);
  for (cudaStream_t st : s->ownStreams) cudaStreamDestroy(st);
}

// Build the layout description from the reference structures plus the
// optional FP64 side table.
int make_layout(GPUInfo* g, State* s, LayoutDesc* L) {
  const GPUVisInfo* v = g->h_visInfo;
  if (!v) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_visInfo is NULL");
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
    return fail(OBIT_DFT_EBADARG, "record length, channel and polarization counts must be positive");
  const int nfreq = L->nchan * L->nif;
  // the frequency table must stay inside the record for every selected product
  const long long lastOff = (long long)L->nrparm + (long long)L->ife * L->incif +
                            (long long)L->chane * L->incf + (long long)L->stoke * L->incs + 2;
  if (lastOff >= L->lrec) return fail(OBIT_DFT_EBADARG, "selected products extend past the record");
  if (L->ilocu < 0 || L->ilocu >= L->nrparm || L->ilocv < 0 || L->ilocv >= L->nrparm ||
      L->ilocw < 0 || L->ilocw >= L->nrparm)
    return fail(OBIT_DFT_EBADARG, "u/v/w offsets must index random parameters");
  L->fscale.assign(nfreq, 1.0);
  if (s->haveFreqD) {
    if ((int)s->freqArr.size() < nfreq) return fail(OBIT_DFT_EBADARG, "FP64 frequency table too short");
    for (int i = 0; i < nfreq; i++) L->fscale[i] = s->freqArr[i] / s->uvRef;
  } else {
    if (!v->freqScale) return fail(OBIT_DFT_EBADARG, "GPUVisInfo.freqScale is NULL");
    std::vector<float> fs(nfreq);
    CUDA_TRY(cudaMemcpy(fs.data(), v->freqScale, sizeof(float) * nfreq, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nfreq; i++) L->fscale[i] = (double)fs[i];
  }
  const int kind = s->model.kind;
  if (kind == kPointSpec || kind == kGaussSpec) {
    L->lnspec.assign(nfreq, 0.0);
    for (int i = 0; i < nfreq; i++) {
      double r;
      if (s->haveFreqD)
        r = s->freqArr[i] / (s->modelRef > 0 ? s->modelRef : s->uvRef);
      else
        r = L->fscale[i] * (v->freqRat ? (double)v->freqRat[0] : 1.0);
      L->lnspec[i] = std::log(r);
    }
  } else if (kind == kPointTSpec || kind == kGaussTSpec) {
    if ((int)s->specIndex.size() < nfreq)
      return fail(OBIT_DFT_EBADARG, "tabulated spectra need GPUModelInfo.specIndex");
    L->specIndex = s->specIndex;
    L->lnspec.assign(nfreq, 0.0);
    for (int i = 0; i < nfreq; i++) {
      const int pl = s->specIndex[i];
      if (pl < 0 || pl >= s->model.nspec)
        return fail(OBIT_DFT_EBADARG, "specIndex outside the component's plane table");
      double r;
      if (s->haveFreqD && (int)s->specFreq.size() > pl)
        r = s->freqArr[i] / s->specFreq[pl];
      else if (v->freqRat)
        r = L->fscale[i] * (double)v->freqRat[pl];
      else
        return fail(OBIT_DFT_EBADARG, "tabulated spectra need freqRat or specFreq");
      L->lnspec[i] = std::log(r);
    }
  }
  return OBIT_DFT_OK;
}

int make_apply(const GPUInfo* g, const State* s, const LayoutDesc& L, ApplyDesc* A) {
  A->op = s->opType;
  if (A->op < 0 || A->op > 2) return fail(OBIT_DFT_EBADARG, "unknown operation type");
  if (s->cpuRules) {
    A->cumulative = 1;
    A->stokFactor = s->stokFactor;
    for (int j = 0; j < kMaxPol; j++) A->polFact[j] = 1.0f;
    A->flipMask = s->doFlip ? 0xF : 0;
  } else {
    // GPUModelInfo semantics: stokFact per polarization, doSwap on pol 3 only
    A->cumulative = 0;
    A->stokFactor = 1.0f;
    for (int j = 0; j < kMaxPol; j++) {
      const int ist = L.stokb + j;
      A->polFact[j] = (ist < 4) ? s->stokFact[ist] : 1.0f;
    }
    A->flipMask = 0;
    if (s->doSwap && L.stokb <= 3 && L.stoke >= 3) A->flipMask = 1 << (3 - L.stokb);
  }
  (void)g;
  return OBIT_DFT_OK;
}

int ensure_plan(GPUInfo* g, State* s) {
  if (s->planValid) return OBIT_DFT_OK;
  if (!s->haveModel) return fail(OBIT_DFT_EBADARG, "no model set (call SetMod first)");
  LayoutDesc L;
  int rc = make_layout(g, s, &L);
  if (rc) return rc;
  ApplyDesc A;
  rc = make_apply(g, s, L, &A);
  if (rc) return rc;
  free_plan(&s->plan);
  std::string err;
  rc = build_plan(L, s->model, A, s->tune, &s->plan, &err);
  if (rc) return fail(rc, err);
  s->planValid = true;
  return OBIT_DFT_OK;
}

int read_err_flag(State* s) {
  int h = 0;
  CUDA_TRY(cudaMemcpy(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CUDA_TRY(cudaMemset(s->d_err, 0, sizeof(int)));
    return fail(OBIT_DFT_EKERNEL, "kernel reported internal error code " + std::to_string(h));
  }
  return OBIT_DFT_OK;
}

}  // namespace

extern "C" {

int obit_dft_version(void) { return 100; }

const char* obit_dft_last_error(void) { return g_last_error.c_str(); }

int obit_dft_init(GPUInfo* g) {
  g_last_error.clear();
  State* s;
  return ensure_state(g, &s);
}

int obit_dft_set_mod(GPUInfo* g) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  const GPUModelInfo* m = g->h_modelInfo;
  if (!m) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_modelInfo is NULL");
  ModelDesc md;
  md.kind = (int)m->type;
  md.nterm = m->nterm;
  md.lcomp = m->size > 0 ? m->size : g->modelSize;
  md.ncomp = g->nmodel[0] > 0 ? g->nmodel[0] : m->nmodel[0];
  if (md.kind < kPoint || md.kind > kGaussTSpec)
    return fail(OBIT_DFT_EUNSUPPORTED, "model type " + std::to_string(md.kind) + " not supported");
  if (md.ncomp < 0) return fail(OBIT_DFT_EBADARG, "negative component count");
  const bool spec = (md.kind == kPointSpec || md.kind == kGaussSpec);
  const bool tspec = (md.kind == kPointTSpec || md.kind == kGaussTSpec);
  const bool gauss = (md.kind >= kGauss);
  int minLen = 4;
  if (gauss) minLen = 7;
  if (spec) minLen += md.nterm;
  if (tspec) minLen = (gauss ? 8 : 5) + 1;
  if (md.ncomp > 0 && md.lcomp < minLen)
    return fail(OBIT_DFT_EBADARG, "component record shorter than the model type needs");
  if (spec && (md.nterm < 1 || md.nterm > kMaxNTerm))
    return fail(OBIT_DFT_EUNSUPPORTED, "spectral term count must be 1.." + std::to_string(kMaxNTerm));
  md.nspec = tspec ? md.lcomp - (gauss ? 8 : 5) : 0;
  // padded copy of the component table (16-byte aligned rows for bulk copies)
  const float* src = g->d_model[0] ? g->d_model[0] : m->model[0];
  const size_t stride = (size_t)comp_stride(md);
  const size_t bytes = std::max<size_t>(16, (size_t)md.ncomp * stride * sizeof(float));
  if (bytes > s->compBytes) {
    if (s->d_comps) cudaFree(s->d_comps);
    s->d_comps = nullptr;
    s->compBytes = 0;
    CUDA_TRY(cudaMalloc(&s->d_comps, bytes));
    s->compBytes = bytes;
  }
  if (md.ncomp > 0) {
    if (!src) return fail(OBIT_DFT_EBADARG, "device component table is NULL");
    CUDA_TRY(cudaMemset(s->d_comps, 0, (size_t)md.ncomp * stride * sizeof(float)));
    CUDA_TRY(cudaMemcpy2D(s->d_comps, stride * sizeof(float), src, (size_t)md.lcomp * sizeof(float),
                          (size_t)md.lcomp * sizeof(float), (size_t)md.ncomp, cudaMemcpyDeviceToDevice));
  }
  s->model = md;
  s->opType = (int)m->opType;
  s->doSwap = m->doSwap;
  for (int i = 0; i < 4; i++) s->stokFact[i] = m->stokFact[i];
  s->specIndex.clear();
  if (tspec) {
    const GPUVisInfo* v = g->h_visInfo;
    if (!v) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_visInfo is NULL");
    const int nfreq = v->nchan * std::max(1, v->nIF);
    if (m->specIndex) {
      s->specIndex.assign(m->specIndex, m->specIndex + nfreq);
    } else if (m->d_specIndex) {
      s->specIndex.resize(nfreq);
      CUDA_TRY(cudaMemcpy(s->specIndex.data(), m->d_specIndex, sizeof(int) * nfreq,
                          cudaMemcpyDeviceToHost));
    } else {
      return fail(OBIT_DFT_EBADARG, "tabulated spectra need specIndex");
    }
  }
  s->haveModel = true;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_freq(GPUInfo* g, const double* freqArr, int nfreq, double uvRefFreq,
                      double modelRefFreq, const double* specFreq, int nSpec) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!freqArr) {  // clear
    s->haveFreqD = false;
    s->planValid = false;
    return OBIT_DFT_OK;
  }
  if (nfreq <= 0 || !(uvRefFreq > 0.0)) return fail(OBIT_DFT_EBADARG, "bad FP64 frequency table");
  s->freqArr.assign(freqArr, freqArr + nfreq);
  s->uvRef = uvRefFreq;
  s->modelRef = modelRefFreq;
  s->specFreq.clear();
  if (specFreq && nSpec > 0) s->specFreq.assign(specFreq, specFreq + nSpec);
  s->haveFreqD = true;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_poln(GPUInfo* g, int cpuRules, float stokFactor, int doFlip) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  s->cpuRules = cpuRules != 0;
  s->stokFactor = stokFactor;
  s->doFlip = doFlip;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_kernel(GPUInfo* g, int flavor, int chanPerThread, int compsPerTile) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (flavor != OBIT_DFT_RECUR && flavor != OBIT_DFT_PLAIN)
    return fail(OBIT_DFT_EBADARG, "unknown kernel flavor");
  // 0 leaves the choice to the planner (also when switching flavor)
  const int K = chanPerThread ? chanPerThread : (flavor == s->tune.flavor ? s->tune.K : 0);
  if (flavor == OBIT_DFT_RECUR && !(K == 0 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32))
    return fail(OBIT_DFT_EBADARG, "recurrence kernel: channels per thread must be 2, 4, 8, 16 or 32");
  if (flavor == OBIT_DFT_PLAIN && !(K == 0 || K == 1 || K == 2 || K == 4 || K == 8 || K == 16))
    return fail(OBIT_DFT_EBADARG, "plain kernel: channels per thread must be 1, 2, 4, 8 or 16");
  if (compsPerTile < 0 || compsPerTile > 1024) return fail(OBIT_DFT_EBADARG, "bad components per tile");
  s->tune.flavor = flavor;
  s->tune.K = K;
  if (compsPerTile) s->tune.ct = compsPerTile;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_tile(GPUInfo* g, int blocksPerTile, int threadsPerCTA) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (blocksPerTile < 0 || blocksPerTile > kMaxBt || (blocksPerTile & (blocksPerTile - 1)))
    return fail(OBIT_DFT_EBADARG, "blocks per tile must be 0 or a power of two up to 32");
  if (threadsPerCTA != 0 && threadsPerCTA != 128 && threadsPerCTA != 256)
    return fail(OBIT_DFT_EBADARG, "threads per CTA must be 128 or 256");
  const int th = threadsPerCTA ? threadsPerCTA : 256;
  if (blocksPerTile && th / blocksPerTile < 8)
    return fail(OBIT_DFT_EBADARG, "a tile needs at least 8 rows (threads / blocks)");
  s->tune.Bt = blocksPerTile;
  s->tune.threads = th;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_calc_device(GPUInfo* g, float* d_vis, int nvis, void* stream) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (nvis < 0) return fail(OBIT_DFT_EBADARG, "negative record count");
  if (nvis > 0 && !d_vis) return fail(OBIT_DFT_EBADARG, "NULL visibility buffer");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  std::string err;
  rc = launch_plan(s->plan, d_vis, 0, nvis, s->d_comps, s->d_err, (cudaStream_t)stream, &err);
  if (rc) return fail(rc, err);
  return OBIT_DFT_OK;
}

int obit_dft_plan_info(GPUInfo* g, int* info, int n) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!info || n < 1) return fail(OBIT_DFT_EBADARG, "plan info needs an output array");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  const Plan& pl = s->plan;
  const int v[8] = {pl.tune.flavor, pl.tune.K, pl.kp.ct, pl.kp.Bt, pl.kp.R, pl.threads,
                    pl.kp.nblocks, pl.kp.ndf};
  for (int i = 0; i < n && i < 8; i++) info[i] = v[i];
  return OBIT_DFT_OK;
}

int obit_dft_check(GPUInfo* g) {
  g_last_error.clear();
  State* s = find_state(g);
  if (!s) return fail(OBIT_DFT_EBADARG, "GPUInfo not initialized");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  return read_err_flag(s);
}

int obit_dft_calc(GPUInfo* g) {
  g_last_error.clear();
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  const int nvis = g->nvis;
  if (nvis < 0) return fail(OBIT_DFT_EBADARG, "negative record count");
  if (nvis == 0) return OBIT_DFT_OK;
  if (!g->h_data) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_data is NULL");
  if (g->h_visInfo && g->h_visInfo->lenvis != g->lenvis)
    return fail(OBIT_DFT_EBADARG, "GPUInfo.lenvis and h_visInfo->lenvis differ");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  const int lenvis = g->lenvis;
  // staging buffers and streams: the caller's (reference layout) or our own
  int nbuf = g->nstream > 0 ? g->nstream : 0;
  std::vector<float*> bufs;
  std::vector<cudaStream_t> streams;
  int rowsPerBuf = s->bufRows;
  if (nbuf > 0 && g->d_data && rowsPerBuf > 0) {
    for (int i = 0; i < nbuf; i++) bufs.push_back(g->d_data[i]);
  } else {
    nbuf = 3;
    rowsPerBuf = std::max(1, std::min(nvis, (nvis + nbuf - 1) / nbuf));
    if ((int)s->ownBufs.size() != nbuf || s->bufRows < rowsPerBuf) {
      for (float* b : s->ownBufs) cudaFree(b);
      s->ownBufs.clear();
      for (int i = 0; i < nbuf; i++) {
        float* b = nullptr;
        CUDA_TRY(cudaMalloc(&b, sizeof(float) * (size_t)rowsPerBuf * lenvis));
        s->ownBufs.push_back(b);
      }
      s->bufRows = rowsPerBuf;
    }
    rowsPerBuf = s->bufRows;
    bufs = s->ownBufs;
  }
  for (int i = 0; i < nbuf; i++) {
    if (g->stream && g->stream[i]) {
      streams.push_back((cudaStream_t)g->stream[i]);
    } else {
      while ((int)s->ownStreams.size() <= i) {
        cudaStream_t st;
        CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        s->ownStreams.push_back(st);
      }
      streams.push_back(s->ownStreams[i]);
    }
  }
  // chunk i: upload, compute and download on stream i % nbuf, so that copies of
  // one chunk overlap the kernel of another
  std::string err;
  int chunk = 0;
  for (int r0 = 0; r0 < nvis; r0 += rowsPerBuf, chunk++) {
    const int nr = std::min(rowsPerBuf, nvis - r0);
    const int b = chunk % nbuf;
    const size_t bytes = sizeof(float) * (size_t)nr * lenvis;
    float* host = g->h_data + (size_t)r0 * lenvis;
    CUDA_TRY(cudaMemcpyAsync(bufs[b], host, bytes, cudaMemcpyHostToDevice, streams[b]));
    rc = launch_plan(s->plan, bufs[b], 0, nr, s->d_comps, s->d_err, streams[b], &err);
    if (rc) return fail(rc, err);
    CUDA_TRY(cudaMemcpyAsync(host, bufs[b], bytes, cudaMemcpyDeviceToHost, streams[b]));
  }
  for (int i = 0; i < nbuf; i++) CUDA_TRY(cudaStreamSynchronize(streams[i]));
  return read_err_flag(s);
}

int obit_dft_shutdown(GPUInfo* g) {
  g_last_error.clear();
  if (!g) return fail(OBIT_DFT_EBADARG, "NULL GPUInfo");
  std::unique_ptr<State> s;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_states.find(g);
    if (it == g_states.end()) return OBIT_DFT_OK;
    s = std::move(it->second);
    g_states.erase(it);
  }
  for (cudaStream_t st : s->ownStreams) cudaStreamSynchronize(st);
  release_state(s.get());
  return OBIT_DFT_OK;
}

// ---- the reference's void entry points ----------------------------------

static void report(const char* who, int rc) {
  if (rc) fprintf(stderr, "%s: error %d: %s\n", who, rc, g_last_error.c_str());
}

void ObitCUDASkyModelDFTInit(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTInit", obit_dft_init(gpuInfo));
}

void ObitCUDASkyModelDFTSetMod(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTSetMod", obit_dft_set_mod(gpuInfo));
}

void ObitCUDASkyModelDFTCalc(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTCalc", obit_dft_calc(gpuInfo));
}

void ObitCUDASkyModelDFTShutdown(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTShutdown", obit_dft_shutdown(gpuInfo));
}

}  // extern "C"
