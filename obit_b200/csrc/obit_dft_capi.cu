// C ABI of libobit_dft.so (include/obit_dft.h): the reference's CUDA-layer
// entry points and their status-returning forms.
//
// Library state is kept per GPUInfo* in a registry; the GPUInfo itself is
// owned by the caller (ObitGPUSkyModel.c or the host mirror in this package),
// exactly as in the reference, and is only read here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "obit_dft.h"
#include "abi_internal.h"
#include "dft_beam.h"
#include "dft_plan.h"

namespace {

using namespace obit;

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess)                                                          \
      return fail(OBIT_DFT_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)

// Beam-corrected DFT (obit_dft_set_beam): the caller's description, its
// per-antenna and per-(channel, IF) tables on the device, and the launch
// parameters built with the plan.
struct BeamState {
  bool on = false;
  int numAnt = 0, numAntType = 0, numJChan = 0, ilocb = -1, iloca1 = -1, iloca2 = -1;
  int jonesComps = 0, stokType = 1, circular = 0;
  float c2p = 1.f, s2p = 0.f;
  const float* jones = nullptr;
  int* d_antType = nullptr;
  int* d_jchan = nullptr;
  std::vector<int> jchan;  // host copy: the planner cuts blocks at Jones-plane changes
  double* d_fscale = nullptr;
  double* d_lnspec = nullptr;
  int* d_plane = nullptr;
  BlockDesc* d_blocks = nullptr;  // channel blocks of the beam plan
  BeamSeg* d_segs = nullptr;      // channel runs of the tensor-core form
  float4* d_coef = nullptr;       // its coefficient fragments (written per launch)
  float2* d_amp = nullptr;        // its spectral amplitudes (written per launch)
  BeamKParams kp{};
};

void free_beam_tables(BeamState& b) {
  for (void* q : {(void*)b.d_fscale, (void*)b.d_lnspec, (void*)b.d_plane, (void*)b.d_blocks, (void*)b.d_segs,
                  (void*)b.d_coef, (void*)b.d_amp})
    if (q) cudaFree(q);
  b.d_coef = nullptr;
  b.d_amp = nullptr;
  b.d_fscale = nullptr;
  b.d_lnspec = nullptr;
  b.d_plane = nullptr;
  b.d_blocks = nullptr;
  b.d_segs = nullptr;
}

// Runs of the tensor-core beam form from a plan of kBeamMmaRows-channel
// blocks: consecutive full blocks of one IF, one channel-increment class and
// one Jones plane, at most kBeamMmaMaxChan channels each.
std::vector<BeamSeg> beam_segments(const Plan& plan, const LayoutDesc& L, const std::vector<int>& jchan) {
  std::vector<BeamSeg> segs;
  const std::vector<BlockDesc>& bl = plan.blocks;
  for (size_t i = 0; i < bl.size(); i++) {
    const BlockDesc& b = bl[i];
    const int jp = jchan[b.ifq0];
    bool extend = false;
    if (!segs.empty()) {
      const BeamSeg& sg = segs.back();
      const BlockDesc& pb = bl[i - 1];
      extend = pb.len == kBeamMmaRows && sg.nch % kBeamMmaRows == 0 && sg.nch + b.len <= kBeamMmaMaxChan &&
               b.ifq0 == pb.ifq0 + kBeamMmaRows * L.kincf && b.off0 == pb.off0 + kBeamMmaRows * L.incf &&
               b.dfc == sg.dfc && jp == sg.jplane;
    }
    if (extend) {
      segs.back().nch += b.len;
    } else {
      BeamSeg sg{};
      sg.f0_hi = b.f0_hi;
      sg.f0_lo = b.f0_lo;
      sg.dfc = b.dfc;
      sg.off0 = b.off0;
      sg.ifq0 = b.ifq0;
      sg.nch = b.len;
      sg.jplane = jp;
      segs.push_back(sg);
    }
  }
  return segs;
}

struct State {
  int device = 0;
  FreqSide fs;   // FP64 frequency side table
  PolnRules pr;  // CPU-reference polarization rules
  TuneDesc tune; // kernel choice
  ModelCfg mc;   // model description
  float* d_comps = nullptr;
  size_t compBytes = 0;
  bool haveModel = false;
  float* d_lo = nullptr;  // low parts of FP64 positions (obit_dft_set_mod_d)
  size_t loBytes = 0;
  bool haveLo = false;
  // The recurrence kernels' copy of the table (and of the low parts) ordered by
  // spectral index, for point families with one index (spectral-factored
  // form); the beam kernel and the FP64 side table keep the caller's order.
  float* d_sorted = nullptr;
  float* d_sortedLo = nullptr;
  size_t sortedBytes = 0, sortedLoBytes = 0;
  const float* runComps = nullptr;  // table the plan's launches read
  // plan
  Plan plan;
  bool planValid = false;
  // staging
  int bufRows = 0;                 // rows per device staging buffer
  std::vector<float*> ownBufs;     // used when the caller supplies none
  std::vector<cudaStream_t> ownStreams;
  int* d_err = nullptr;
  int waitPolls = kDefaultWaitPolls;  // obit_dft_set_wait_limit
  BeamState beam;
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
  if (s->d_lo) cudaFree(s->d_lo);
  if (s->d_sorted) cudaFree(s->d_sorted);
  if (s->d_sortedLo) cudaFree(s->d_sortedLo);
  if (s->d_err) cudaFree(s->d_err);
  free_beam_tables(s->beam);
  if (s->beam.d_antType) cudaFree(s->beam.d_antType);
  if (s->beam.d_jchan) cudaFree(s->beam.d_jchan);
  for (float* b : s->ownBufs) cudaFree(b);
  for (cudaStream_t st : s->ownStreams) cudaStreamDestroy(st);
}

// The recurrence kernels' copy of the model table, in s->d_sorted:
//  - point families with one spectral index: the padded table (and, with FP64
//    positions, its low parts in s->d_sortedLo) stably ordered by index;
//  - Gaussian families with one spectral index (no FP64 positions): the
//    untapered components (g1 = g2 = g3 = 0, the reference's encoding of
//    points in a Gaussian table, ObitSkyModel.c:2044-2063) re-encoded in the
//    matching point family's field order and ordered by index, followed by
//    the Gaussian components.  *md becomes that point family when no Gaussian
//    is left, else a mixed model (md->ncompPt point rows, md->ncomp Gaussian).
// *index receives the ordered spectral indices of the point rows; left empty
// (no copy made, *md unchanged) when an index is not finite or no component
// qualifies.
int prepare_run_table(State* s, ModelDesc* md, std::vector<float>* index) {
  index->clear();
  const bool gauss = md->kind == kGaussSpec || md->kind == kGaussTSpec;
  const size_t stride = (size_t)comp_stride(*md), n = (size_t)md->ncomp;
  // spectral index: field 7 of a Gaussian record, 4 of a point record
  const int aField = gauss ? 7 : kSpecIndexField;
  std::vector<float> tab(n * stride), lo;
  CUDA_TRY(cudaMemcpy(tab.data(), s->d_comps, sizeof(float) * tab.size(), cudaMemcpyDeviceToHost));
  const bool withLo = s->haveLo && !gauss;
  if (withLo) {
    lo.resize(n * 4);
    CUDA_TRY(cudaMemcpy(lo.data(), s->d_lo, sizeof(float) * lo.size(), cudaMemcpyDeviceToHost));
  }
  std::vector<int> pts, gs;
  for (size_t i = 0; i < n; i++) {
    const float* r = tab.data() + i * stride;
    if (!std::isfinite(r[aField])) return OBIT_DFT_OK;
    if (!gauss || (r[4] == 0.0f && r[5] == 0.0f && r[6] == 0.0f)) pts.push_back((int)i);
    else gs.push_back((int)i);
  }
  if (pts.empty()) return OBIT_DFT_OK;
  std::stable_sort(pts.begin(), pts.end(), [&](int a, int b) {
    return tab[(size_t)a * stride + aField] < tab[(size_t)b * stride + aField];
  });
  std::vector<float> out(tab.size(), 0.0f), outLo(lo.size());
  index->resize(pts.size());
  for (size_t k = 0; k < pts.size(); k++) {
    const float* src = tab.data() + (size_t)pts[k] * stride;
    float* dst = out.data() + k * stride;
    if (!gauss) {
      std::copy(src, src + stride, dst);
      if (withLo) std::copy(lo.begin() + (size_t)pts[k] * 4, lo.begin() + (size_t)pts[k] * 4 + 4,
                            outLo.begin() + k * 4);
    } else {
      // [A, X, Y, Z, g1, g2, g3, alpha (, planes)] -> [A, X, Y, Z, alpha (, planes)]
      std::copy(src, src + 4, dst);
      dst[4] = src[7];
      if (md->kind == kGaussTSpec)
        for (int q = 0; q < md->nspec; q++) dst[5 + q] = src[8 + q];
    }
    (*index)[k] = src[aField];
  }
  for (size_t k = 0; k < gs.size(); k++)
    std::copy(tab.begin() + (size_t)gs[k] * stride, tab.begin() + (size_t)(gs[k] + 1) * stride,
              out.begin() + (pts.size() + k) * stride);
  auto upload = [&](const std::vector<float>& h, float** d, size_t* cap) -> int {
    const size_t bytes = std::max<size_t>(16, sizeof(float) * h.size());
    if (bytes > *cap) {
      if (*d) cudaFree(*d);
      *d = nullptr;
      *cap = 0;
      CUDA_TRY(cudaMalloc(d, bytes));
      *cap = bytes;
    }
    CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
    return OBIT_DFT_OK;
  };
  int rc = upload(out, &s->d_sorted, &s->sortedBytes);
  if (!rc && withLo) rc = upload(outLo, &s->d_sortedLo, &s->sortedLoBytes);
  if (rc) {
    index->clear();
    return rc;
  }
  if (gauss) {
    if (gs.empty()) {
      md->kind = (md->kind == kGaussTSpec) ? kPointTSpec : kPointSpec;
    } else {
      md->ncompPt = (int)pts.size();
      md->ncomp = (int)gs.size();
    }
  }
  return OBIT_DFT_OK;
}

int ensure_plan(GPUInfo* g, State* s) {
  if (s->planValid) return OBIT_DFT_OK;
  if (!s->haveModel) return fail(OBIT_DFT_EBADARG, "no model set (call SetMod first)");
  LayoutDesc L;
  ApplyDesc A;
  std::string err;
  int rc = layout_from_info(g->h_visInfo, s->mc, s->fs, &L, &err);
  if (!rc) rc = apply_from_info(s->mc, s->pr, L, &A, &err);
  if (rc) return fail(rc, err);
  free_plan(&s->plan);
  // Point families with one spectral index: the recurrence kernels read a copy
  // ordered by the index, which lets the planner choose the spectral-factored
  // form (the wait-limit diagnostic has a chain-form instance only).
  TuneDesc T = s->tune;
  if (s->waitPolls != kDefaultWaitPolls) T.specFactor = 0;
  ModelDesc md = s->mc.model;
  std::vector<float> index;
  s->runComps = s->d_comps;
  const float* runLo = s->haveLo ? s->d_lo : nullptr;
  const bool ptOne = md.kind == kPointTSpec || (md.kind == kPointSpec && md.nterm == 1);
  const bool gsOne = md.kind == kGaussTSpec || (md.kind == kGaussSpec && md.nterm == 1);
  if (T.flavor == kFlavorRecur && T.specFactor && md.ncomp > 1 && (ptOne || (gsOne && !s->haveLo))) {
    ModelDesc m2 = md;
    if ((rc = prepare_run_table(s, &m2, &index))) return rc;
    if (!index.empty()) {
      m2.specIndex = index.data();
      Plan trial;
      rc = plan_layout(L, m2, A, T, &trial, &err);
      if (rc == 0) {  // the ordered (and, for Gaussian families, split) copy
        md = m2;
        s->runComps = s->d_sorted;
        if (s->haveLo) runLo = s->d_sortedLo;
      } else if (rc != 4) {
        return fail(rc, err);
      }  // 4: the split table cannot run mixed on this layout; keep the caller's table
    }
  }
  rc = plan_layout(L, md, A, T, &s->plan, &err);
  s->plan.kp.waitPolls = s->waitPolls;  // chooses the diagnostic instance when lowered
  s->plan.kp.compsLo = runLo;
  if (!rc) rc = finalize_plan(&s->plan, nullptr, 0, &err);
  if (rc) return fail(rc, err);
  if (s->beam.on) {  // launch parameters and per-(channel, IF) tables of the beam kernel
    BeamState& b = s->beam;
    if (b.jonesComps < s->mc.model.ncomp)
      return fail(OBIT_DFT_EBADARG, "the Jones table holds fewer components than the model");
    free_beam_tables(b);
    const int nfreq = L.nchan * L.nif;
    auto upload = [&](const void* h, size_t bytes, void** d) -> int {
      CUDA_TRY(cudaMalloc(d, std::max<size_t>(bytes, 8)));
      CUDA_TRY(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
      return OBIT_DFT_OK;
    };
    if ((rc = upload(L.fscale.data(), sizeof(double) * nfreq, (void**)&b.d_fscale))) return rc;
    if ((int)L.lnspec.size() >= nfreq &&
        (rc = upload(L.lnspec.data(), sizeof(double) * nfreq, (void**)&b.d_lnspec)))
      return rc;
    if ((int)L.specIndex.size() >= nfreq &&
        (rc = upload(L.specIndex.data(), sizeof(int) * nfreq, (void**)&b.d_plane)))
      return rc;
    // Channel blocks that never span a change of Jones plane, from the same
    // planner: 16-channel blocks joined into runs for the tensor-core form
    // (uniformly spaced channels, runs of 4 channels or more
    // on average), else blocks of at most kBeamK channels for the block form.
    LayoutDesc LB = L;
    LB.blockKey = b.jchan;
    TuneDesc TB;
    TB.flavor = kFlavorRecur;
    TB.threads = kThreads;
    TB.specFactor = 0;
    Plan mplan, bplan;
    std::vector<BeamSeg> segs;
    bool mma = false;
    if (s->tune.flavor == kFlavorRecur && s->tune.specFactor && beam_mma_supported(s->mc.model.kind)) {
      TB.K = kBeamMmaRows;
      rc = plan_layout(LB, s->mc.model, A, TB, &mplan, &err);
      if (rc) return fail(rc, err);
      if (mplan.linear) {
        segs = beam_segments(mplan, L, b.jchan);
        long long nch = 0;
        for (const BeamSeg& sg : segs) nch += sg.nch;
        mma = !segs.empty() && nch >= 4LL * (long long)segs.size();
      }
      if (mma) {  // the tile must fit shared memory with this many antenna types, and
                  // the per-launch tables stay within 4 GiB
        BeamKParams trial{};
        trial.k = mplan.kp;
        trial.mode = s->mc.model.kind;
        trial.numAntType = b.numAntType;
        trial.numJChan = b.numJChan;
        trial.nseg = (int)segs.size();
        mma = beam_mma_fit_tile(&trial) > 0;
        if (mma) {
          trial.ncompPad = (trial.k.ncomp + trial.k.ct - 1) / trial.k.ct * trial.k.ct;
          mma = beam_mma_coef_bytes(trial) + beam_mma_amp_bytes(trial) <= (size_t(4) << 30);
        }
      }
    }
    if (!mma) {
      TB.K = kBeamK;
      rc = plan_layout(LB, s->mc.model, A, TB, &bplan, &err);
      if (rc) return fail(rc, err);
    }
    const Plan& used = mma ? mplan : bplan;
    BeamKParams& k = b.kp;
    k = BeamKParams{};
    k.k = used.kp;
    if (mma) {
      CUDA_TRY(cudaMalloc(&b.d_segs, sizeof(BeamSeg) * segs.size()));
      CUDA_TRY(cudaMemcpy(b.d_segs, segs.data(), sizeof(BeamSeg) * segs.size(), cudaMemcpyHostToDevice));
      k.segs = b.d_segs;
      k.nseg = (int)segs.size();
      k.mma = 1;
      k.k.blocks = nullptr;
      k.k.R = kBeamMmaWarps;
    } else {
      const int nb = (int)bplan.blocks.size();
      CUDA_TRY(cudaMalloc(&b.d_blocks, sizeof(BlockDesc) * (size_t)std::max(1, nb)));
      if (nb)
        CUDA_TRY(cudaMemcpy(b.d_blocks, bplan.blocks.data(), sizeof(BlockDesc) * (size_t)nb,
                            cudaMemcpyHostToDevice));
      k.k.blocks = b.d_blocks;
    }
    k.k.comps = s->d_comps;
    k.k.compsLo = s->haveLo ? s->d_lo : nullptr;  // FP64 positions, the caller's order as d_comps
    k.k.ncomp = s->mc.model.ncomp;
    k.k.errFlag = s->d_err;
    k.k.rowBase = 0;
    k.k.waitPolls = kDefaultWaitPolls;
    k.nrparm = L.nrparm;
    k.ilocb = b.ilocb;
    k.iloca1 = b.iloca1;
    k.iloca2 = b.iloca2;
    k.incif = L.incif;
    k.ncorr = L.nstok >= 4 ? 4 : std::min(2, L.nstok);
    if ((long long)L.nrparm + (long long)L.ife * L.incif + (long long)L.chane * L.incf +
            (long long)(k.ncorr - 1) * L.incs + 2 >= L.lrec)
      return fail(OBIT_DFT_EBADARG, "modelled correlations extend past the record");
    for (int q = 0; q < 4; q++) k.polFact[q] = s->mc.stokFact[q];
    k.chanb = L.chanb;
    k.nchanSel = L.chane - L.chanb + 1;
    k.ifb = L.ifb;
    k.nifSel = L.ife - L.ifb + 1;
    k.kincf = L.kincf;
    k.kincif = L.kincif;
    k.fscale = b.d_fscale;
    k.lnspec = b.d_lnspec;
    k.plane = b.d_plane;
    k.jchan = b.d_jchan;
    k.antType = b.d_antType;
    k.numAnt = b.numAnt;
    k.numAntType = b.numAntType;
    k.numJChan = b.numJChan;
    k.jones = b.jones;
    k.jonesComps = b.jonesComps;
    k.mode = s->mc.model.kind;
    k.stokType = b.stokType;
    k.circular = b.circular;
    k.c2p = b.c2p;
    k.s2p = b.s2p;
    k.flavor = (s->tune.flavor == kFlavorPlain) ? kFlavorPlain : kFlavorRecur;
    if (k.mma) {
      beam_mma_fit_tile(&k);
      k.ncompPad = (k.k.ncomp + k.k.ct - 1) / k.k.ct * k.k.ct;
      CUDA_TRY(cudaMalloc(&b.d_coef, std::max<size_t>(16, beam_mma_coef_bytes(k))));
      k.coefTab = b.d_coef;
      if (const size_t ab = beam_mma_amp_bytes(k)) {
        CUDA_TRY(cudaMalloc(&b.d_amp, ab));
        k.ampTab = b.d_amp;
      }
    } else if ((rc = beam_fit_tile(&k, &err))) {
      return fail(rc, err);
    }
  }
  s->planValid = true;
  return OBIT_DFT_OK;
}

int read_err_flag(State* s) {
  int h = 0;
  CUDA_TRY(cudaMemcpy(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CUDA_TRY(cudaMemset(s->d_err, 0, sizeof(int)));
    std::string msg;
    const int rc = kernel_flag_status(h, &msg);
    return fail(rc, msg);
  }
  return OBIT_DFT_OK;
}

}  // namespace

extern "C" {

int obit_dft_version(void) { return 100; }

const char* obit_dft_last_error(void) { return last_error(); }

int obit_dft_init(GPUInfo* g) {
  set_last_error("");
  State* s;
  return ensure_state(g, &s);
}

int obit_dft_set_mod(GPUInfo* g) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  const GPUModelInfo* m = g->h_modelInfo;
  if (!m) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_modelInfo is NULL");
  std::string err;
  const int lcomp = m->size > 0 ? m->size : g->modelSize;
  const int ncomp = g->nmodel[0] > 0 ? g->nmodel[0] : m->nmodel[0];
  ModelCfg mc;
  rc = model_from_info(m, ncomp, lcomp, g->h_visInfo, &mc, &err);
  if (rc) return fail(rc, err);
  // padded copy of the component table (16-byte aligned rows for bulk copies)
  const ModelDesc& md = mc.model;
  const size_t bytes = std::max<size_t>(16, (size_t)md.ncomp * comp_stride(md) * sizeof(float));
  if (bytes > s->compBytes) {
    if (s->d_comps) cudaFree(s->d_comps);
    s->d_comps = nullptr;
    s->compBytes = 0;
    CUDA_TRY(cudaMalloc(&s->d_comps, bytes));
    s->compBytes = bytes;
  }
  rc = copy_comps(s->d_comps, g->d_model[0] ? g->d_model[0] : m->model[0], md, 0, &err);
  if (rc) return fail(rc, err);
  CUDA_TRY(cudaStreamSynchronize(0));
  s->mc = mc;
  s->haveModel = true;
  s->haveLo = false;  // FP64 positions belong to the previous model
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_mod_d(GPUInfo* g, const double* xyz, int ncomp) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!xyz) {  // back to the FP32 fields as they now stand
    s->haveLo = false;
    s->planValid = false;
    return OBIT_DFT_OK;
  }
  if (!s->haveModel) return fail(OBIT_DFT_EBADARG, "no model set (call SetMod first)");
  const ModelDesc& md = s->mc.model;
  if (ncomp < md.ncomp)
    return fail(OBIT_DFT_EBADARG, "FP64 positions for " + std::to_string(ncomp) + " components, the model has " +
                                      std::to_string(md.ncomp));
  // X, Y, Z = hi + lo: hi the nearest float (it replaces fields 1-3 of the
  // device table), lo the float of the remainder (a side table of 4 floats per
  // component, staged beside each component tile)
  std::vector<float> hi(3 * (size_t)md.ncomp), lo(4 * (size_t)md.ncomp, 0.0f);
  for (int i = 0; i < md.ncomp; i++) {
    for (int k = 0; k < 3; k++) {
      const double x = xyz[3 * (size_t)i + k];
      if (!std::isfinite(x)) return fail(OBIT_DFT_EBADARG, "non-finite FP64 position");
      const float h = (float)x;
      hi[3 * (size_t)i + k] = h;
      lo[4 * (size_t)i + k] = (float)(x - (double)h);
    }
  }
  if (md.ncomp > 0) {
    const size_t bytes = lo.size() * sizeof(float);
    if (bytes > s->loBytes) {
      if (s->d_lo) cudaFree(s->d_lo);
      s->d_lo = nullptr;
      s->loBytes = 0;
      CUDA_TRY(cudaMalloc(&s->d_lo, bytes));
      s->loBytes = bytes;
    }
    CUDA_TRY(cudaMemcpy(s->d_lo, lo.data(), bytes, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy2D(s->d_comps + 1, sizeof(float) * comp_stride(md), hi.data(), 3 * sizeof(float),
                          3 * sizeof(float), (size_t)md.ncomp, cudaMemcpyHostToDevice));
  }
  s->haveLo = true;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_beam(GPUInfo* g, const ObitDFTBeam* beam) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  BeamState& b = s->beam;
  if (!beam) {
    b.on = false;
    s->planValid = false;
    return OBIT_DFT_OK;
  }
  const GPUVisInfo* v = g->h_visInfo;
  if (!v) return fail(OBIT_DFT_EBADARG, "GPUInfo.h_visInfo is NULL (call Init first)");
  if (beam->stokType < 1 || beam->stokType > 4)
    return fail(OBIT_DFT_EUNSUPPORTED, "Stokes type must be 1..4 (I, Q, U, V)");
  if (beam->numAnt < 1 || beam->numAntType < 1 || beam->numJChan < 1 || !beam->antType || !beam->jchan ||
      !beam->jones || beam->jonesComps < 1)
    return fail(OBIT_DFT_EBADARG, "incomplete beam description");
  if (((uintptr_t)beam->jones & 15u) != 0) return fail(OBIT_DFT_EBADARG, "Jones table not 16-byte aligned");
  const int nrparm = v->nrparm;
  if (beam->ilocb >= 0 ? beam->ilocb >= nrparm
                       : (beam->iloca1 < 0 || beam->iloca1 >= nrparm || beam->iloca2 < 0 || beam->iloca2 >= nrparm))
    return fail(OBIT_DFT_EBADARG, "antenna random parameters outside the record's random parameters");
  for (int i = 0; i < beam->numAnt; i++)
    if (beam->antType[i] < 0 || beam->antType[i] >= beam->numAntType)
      return fail(OBIT_DFT_EBADARG, "antenna type outside 0..numAntType-1");
  const int nfreq = v->nchan * std::max(1, v->nIF);
  for (int i = 0; i < nfreq; i++)
    if (beam->jchan[i] < 0 || beam->jchan[i] >= beam->numJChan)
      return fail(OBIT_DFT_EBADARG, "Jones plane outside 0..numJChan-1");
  if (b.d_antType) cudaFree(b.d_antType);
  if (b.d_jchan) cudaFree(b.d_jchan);
  b.d_antType = nullptr;
  b.d_jchan = nullptr;
  CUDA_TRY(cudaMalloc(&b.d_antType, sizeof(int) * beam->numAnt));
  CUDA_TRY(cudaMemcpy(b.d_antType, beam->antType, sizeof(int) * beam->numAnt, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&b.d_jchan, sizeof(int) * nfreq));
  CUDA_TRY(cudaMemcpy(b.d_jchan, beam->jchan, sizeof(int) * nfreq, cudaMemcpyHostToDevice));
  b.jchan.assign(beam->jchan, beam->jchan + nfreq);
  b.numAnt = beam->numAnt;
  b.numAntType = beam->numAntType;
  b.numJChan = beam->numJChan;
  b.ilocb = beam->ilocb;
  b.iloca1 = beam->iloca1;
  b.iloca2 = beam->iloca2;
  b.jones = beam->jones;
  b.jonesComps = beam->jonesComps;
  b.stokType = beam->stokType;
  b.circular = beam->circular ? 1 : 0;
  b.c2p = (float)std::cos(2.0 * (double)beam->parAng);
  b.s2p = (float)std::sin(2.0 * (double)beam->parAng);
  b.on = true;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_freq(GPUInfo* g, const double* freqArr, int nfreq, double uvRefFreq,
                      double modelRefFreq, const double* specFreq, int nSpec) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!freqArr) {  // clear
    s->fs.have = false;
    s->planValid = false;
    return OBIT_DFT_OK;
  }
  if (nfreq <= 0 || !(uvRefFreq > 0.0)) return fail(OBIT_DFT_EBADARG, "bad FP64 frequency table");
  s->fs.freqArr.assign(freqArr, freqArr + nfreq);
  s->fs.uvRef = uvRefFreq;
  s->fs.modelRef = modelRefFreq;
  s->fs.specFreq.clear();
  if (specFreq && nSpec > 0) s->fs.specFreq.assign(specFreq, specFreq + nSpec);
  s->fs.have = true;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_poln(GPUInfo* g, int cpuRules, float stokFactor, int doFlip) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  s->pr.cpuRules = cpuRules != 0;
  s->pr.stokFactor = stokFactor;
  s->pr.doFlip = doFlip;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_kernel(GPUInfo* g, int flavor, int chanPerThread, int compsPerTile) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (flavor != OBIT_DFT_RECUR && flavor != OBIT_DFT_PLAIN && flavor != OBIT_DFT_RECUR_CHAIN)
    return fail(OBIT_DFT_EBADARG, "unknown kernel flavor");
  const int specFactor = (flavor == OBIT_DFT_RECUR_CHAIN) ? 0 : 1;
  if (flavor == OBIT_DFT_RECUR_CHAIN) flavor = OBIT_DFT_RECUR;
  // 0 leaves the choice to the planner (also when switching flavor)
  const int K = chanPerThread ? chanPerThread : (flavor == s->tune.flavor ? s->tune.K : 0);
  if (flavor == OBIT_DFT_RECUR && !(K == 0 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32))
    return fail(OBIT_DFT_EBADARG, "recurrence kernel: channels per thread must be 2, 4, 8, 16 or 32");
  if (flavor == OBIT_DFT_PLAIN && !(K == 0 || K == 1 || K == 2 || K == 4 || K == 8 || K == 16))
    return fail(OBIT_DFT_EBADARG, "plain kernel: channels per thread must be 1, 2, 4, 8 or 16");
  if (compsPerTile < 0 || compsPerTile > 1024) return fail(OBIT_DFT_EBADARG, "bad components per tile");
  s->tune.flavor = flavor;
  s->tune.specFactor = specFactor;
  s->tune.K = K;
  if (compsPerTile) s->tune.ct = compsPerTile;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_tile(GPUInfo* g, int blocksPerTile, int threadsPerCTA) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (blocksPerTile < 0 || blocksPerTile > kMaxBt || (blocksPerTile & (blocksPerTile - 1)))
    return fail(OBIT_DFT_EBADARG, "blocks per tile must be 0 or a power of two up to 32");
  if (threadsPerCTA != 0 && threadsPerCTA != 128 && threadsPerCTA != 256)
    return fail(OBIT_DFT_EBADARG, "threads per CTA must be 128 or 256");
  if (blocksPerTile && (threadsPerCTA ? threadsPerCTA : 256) / blocksPerTile < 8)
    return fail(OBIT_DFT_EBADARG, "a tile needs at least 8 rows (threads / blocks)");
  s->tune.Bt = blocksPerTile;
  s->tune.threads = threadsPerCTA;
  s->planValid = false;
  return OBIT_DFT_OK;
}

int obit_dft_set_wait_limit(GPUInfo* g, int polls) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  s->waitPolls = polls < 0 ? kDefaultWaitPolls : polls;
  s->planValid = false;  // re-planned (and re-finalized) at the next calc
  return OBIT_DFT_OK;
}

int obit_dft_calc_device(GPUInfo* g, float* d_vis, int nvis, void* stream) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (nvis < 0) return fail(OBIT_DFT_EBADARG, "negative record count");
  if (nvis > 0 && !d_vis) return fail(OBIT_DFT_EBADARG, "NULL visibility buffer");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  std::string err;
  if (s->beam.on) {
    BeamKParams k = s->beam.kp;
    k.k.vis = d_vis;
    k.k.nvis = nvis;
    rc = launch_beam(k, (cudaStream_t)stream, &err);
  } else {
    rc = launch_plan(s->plan, d_vis, 0, nvis, s->runComps, s->d_err, (cudaStream_t)stream, &err);
  }
  if (rc) return fail(rc, err);
  return OBIT_DFT_OK;
}

int obit_dft_plan_info(GPUInfo* g, int* info, int n) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!info || n < 1) return fail(OBIT_DFT_EBADARG, "plan info needs an output array");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  const Plan& pl = s->plan;
  const int v[11] = {pl.tune.flavor, pl.tune.K, pl.kp.ct, pl.kp.Bt, pl.kp.R, pl.threads,
                     pl.kp.nblocks, pl.kp.ndf, pl.specFactored ? 1 : 0, pl.mixed ? 1 : 0,
                     pl.mixed ? pl.model.ncompPt : 0};
  for (int i = 0; i < n && i < 11; i++) info[i] = v[i];
  return OBIT_DFT_OK;
}

int obit_dft_beam_info(GPUInfo* g, int* info, int n) {
  set_last_error("");
  State* s;
  int rc = ensure_state(g, &s);
  if (rc) return rc;
  if (!info || n < 1) return fail(OBIT_DFT_EBADARG, "beam info needs an output array");
  if (!s->beam.on) return fail(OBIT_DFT_EBADARG, "no beam is set");
  rc = ensure_plan(g, s);
  if (rc) return rc;
  const BeamKParams& k = s->beam.kp;
  const int v[3] = {k.mma ? 1 : (k.flavor == kFlavorPlain ? 2 : 0), k.k.ct, k.mma ? k.nseg : k.k.nblocks};
  for (int i = 0; i < n && i < 3; i++) info[i] = v[i];
  return OBIT_DFT_OK;
}

int obit_dft_check(GPUInfo* g) {
  set_last_error("");
  State* s = find_state(g);
  if (!s) return fail(OBIT_DFT_EBADARG, "GPUInfo not initialized");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  return read_err_flag(s);
}

int obit_dft_calc(GPUInfo* g) {
  set_last_error("");
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
  // one chunk overlap the kernel of another.  Large buffers are cut into
  // quarter-buffer chunks: only the first upload and the last download are not
  // hidden behind a kernel, and they shrink with the chunk.
  std::string err;
  // The beam's tensor-core form writes its coefficient and amplitude tables
  // once per call, on the first stream; the other streams wait for them.
  const bool beamPrologue = s->beam.on && s->beam.kp.mma;
  struct EventGuard {
    cudaEvent_t e = nullptr;
    ~EventGuard() {
      if (e) cudaEventDestroy(e);
    }
  } ready;
  if (beamPrologue) {
    if ((rc = launch_beam_prologue(s->beam.kp, streams[0], &err))) return fail(rc, err);
    CUDA_TRY(cudaEventCreateWithFlags(&ready.e, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(ready.e, streams[0]));
    for (int i = 1; i < nbuf; i++) CUDA_TRY(cudaStreamWaitEvent(streams[i], ready.e, 0));
  }
  const int step = rowsPerBuf >= 8192 ? (rowsPerBuf + 3) / 4 : rowsPerBuf;
  int chunk = 0;
  for (int r0 = 0; r0 < nvis; r0 += step, chunk++) {
    const int nr = std::min(step, nvis - r0);
    const int b = chunk % nbuf;
    const size_t bytes = sizeof(float) * (size_t)nr * lenvis;
    float* host = g->h_data + (size_t)r0 * lenvis;
    CUDA_TRY(cudaMemcpyAsync(bufs[b], host, bytes, cudaMemcpyHostToDevice, streams[b]));
    if (s->beam.on) {
      BeamKParams k = s->beam.kp;
      k.k.vis = bufs[b];
      k.k.nvis = nr;
      rc = launch_beam(k, streams[b], &err, !beamPrologue);
    } else {
      rc = launch_plan(s->plan, bufs[b], 0, nr, s->runComps, s->d_err, streams[b], &err);
    }
    if (rc) return fail(rc, err);
    CUDA_TRY(cudaMemcpyAsync(host, bufs[b], bytes, cudaMemcpyDeviceToHost, streams[b]));
  }
  for (int i = 0; i < nbuf; i++) CUDA_TRY(cudaStreamSynchronize(streams[i]));
  return read_err_flag(s);
}

int obit_dft_shutdown(GPUInfo* g) {
  set_last_error("");
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
  if (rc) fprintf(stderr, "%s: error %d: %s\n", who, rc, last_error());
}

void ObitCUDASkyModelDFTInit(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTInit", obit_dft_init(gpuInfo));
}

void ObitCUDASkyModelDFTSetMod(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTSetMod", obit_dft_set_mod(gpuInfo));
}

void ObitCUDASkyModelDFTSetModD(GPUInfo* gpuInfo, const double* xyz, int ncomp) {
  report("ObitCUDASkyModelDFTSetModD", obit_dft_set_mod_d(gpuInfo, xyz, ncomp));
}

void ObitCUDASkyModelDFTCalc(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTCalc", obit_dft_calc(gpuInfo));
}

void ObitCUDASkyModelDFTShutdown(GPUInfo* gpuInfo) {
  report("ObitCUDASkyModelDFTShutdown", obit_dft_shutdown(gpuInfo));
}

}  // extern "C"
