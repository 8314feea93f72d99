// Multi-facet batch of the DFT subtract (include/obit_dft.h, obit_dft_batch_*):
// many facets with uneven row and component counts applied by one persistent
// kernel launch per model family, captured in a CUDA graph, with a tile shape
// per family chosen by timing candidates on a row sample.
//
// The reference applies such a model field by field and buffer by buffer
// (ObitSkyModel's per-image loop around ObitGPUSkyModelDFTCalc,
// ObitSystem/Obit/src/ObitGPUSkyModel.c:502-518); each call there is a separate
// kernel launch whose tail leaves SMs idle.  Here the work items (rows x
// channel-block tiles) of all facets form one list, ordered by decreasing cost
// per item, that persistent CTAs drain through a device counter.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "abi_internal.h"
#include "dft_plan.h"
#include "obit_dft.h"

using namespace obit;

namespace {

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

size_t round_up(size_t n, size_t a) { return (n + a - 1) / a * a; }

struct Facet {
  ModelCfg mc;
  LayoutDesc L;
  ApplyDesc A;
  float* d_vis = nullptr;
  int nvis = 0;
  size_t compOff = 0;        // float offset in the batch's padded component buffer
  long long evalsPerRow = 0; // selected (channel, IF) pairs x components
  // planner-default single-facet plans for the per-facet comparator
  Plan single[2];
  bool haveSingle[2] = {false, false};
};

// One model family: its facets in work order and its device work list.
struct Group {
  int kind = kPoint;
  std::vector<int> order;  // facet indices, decreasing cost per item
  TuneDesc tune;           // requested shape (0 fields: planner's choice)
  // resolved
  int K = 0, ct = 0, Bt = 0, R = 0, threads = 0, grid = 0;
  size_t smemBytes = 0;
  int cap = 0;                // CTAs resident across the device
  long long items = 0, evals = 0;
  std::vector<KParams> hkps;  // host copies of the facets' parameter blocks (group order)
  KParams* d_params = nullptr;
  int* d_itemStart = nullptr;
  int* d_counter = nullptr;
  BlockDesc* d_blocks = nullptr;
  bool built = false;
};

void free_group(Group& g) {
  if (g.d_params) cudaFree(g.d_params);
  if (g.d_itemStart) cudaFree(g.d_itemStart);
  if (g.d_counter) cudaFree(g.d_counter);
  if (g.d_blocks) cudaFree(g.d_blocks);
  g.d_params = nullptr;
  g.d_itemStart = g.d_counter = nullptr;
  g.d_blocks = nullptr;
  g.built = false;
}

// The streamed form (obit_dft_batch_run_host): waves of rows through a
// two-half device staging area, captured once as H2D -> batch kernels -> D2H.
struct HostRun {
  std::vector<float*> h;       // the facets' host records the graph reads and writes
  long long stagingBytes = 0;
  float* d_stage = nullptr;
  KParams* d_params = nullptr; // per (wave, group): the pieces' parameter blocks
  int* d_starts = nullptr;
  int* d_counters = nullptr;
  cudaStream_t copyStream = nullptr;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int waves = 0;
  long long h2dBytes = 0;
};

void free_host_run(HostRun& r) {
  if (r.exec) cudaGraphExecDestroy(r.exec);
  if (r.graph) cudaGraphDestroy(r.graph);
  for (cudaEvent_t e : r.events) cudaEventDestroy(e);
  for (void* q : {(void*)r.d_stage, (void*)r.d_params, (void*)r.d_starts, (void*)r.d_counters})
    if (q) cudaFree(q);
  if (r.copyStream) cudaStreamDestroy(r.copyStream);
  r = HostRun();
}

}  // namespace

struct ObitDFTBatch {
  int device = 0;
  std::vector<Facet> facets;
  float* d_comps = nullptr;
  int* d_err = nullptr;
  std::vector<Group> groups;
  cudaStream_t capStream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  HostRun host;
};

namespace {

void drop_graph(ObitDFTBatch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  free_host_run(b->host);  // its graph holds the groups' parameter blocks too
}

// Plan every facet of group g with one tile shape and upload its work list.
// Facets are read from `fs` (the batch's own, or a row sample's).
int build_group(Group& g, std::vector<Facet>& fs, const float* d_comps, int* d_err, std::string* err) {
  free_group(g);
  if (g.order.empty()) return 0;
  // the tile shape: requested fields, else the planner's choice for the
  // facet of the most work
  TuneDesc T = g.tune;
  T.flavor = kFlavorRecur;
  if (T.threads != 128) T.threads = 256;
  if (T.ct == 0) T.ct = 128;  // the batch's default tile: every facet is planned with the lead's
  {
    int lead = g.order[0];
    long long best = -1;
    for (int f : g.order) {
      const long long w = (long long)fs[f].nvis * fs[f].evalsPerRow;
      if (w > best) best = w, lead = f;
    }
    Plan p;
    int rc = plan_layout(fs[lead].L, fs[lead].mc.model, fs[lead].A, T, &p, err);
    if (rc) return rc;
    T.K = p.tune.K;
    T.Bt = p.kp.Bt;
    T.ct = p.kp.ct;
  }
  if (!batch_kernel_exists(T.K)) {
    *err = "no batched kernel for K=" + std::to_string(T.K);
    return OBIT_DFT_EUNSUPPORTED;
  }
  // plan all facets; the component tile is the smallest any facet allows
  std::vector<Plan> plans(fs.size());
  for (int pass = 0; pass < 2; pass++) {
    int ctMin = T.ct;
    for (int f : g.order) {
      int rc = plan_layout(fs[f].L, fs[f].mc.model, fs[f].A, T, &plans[f], err);
      if (rc) return rc;
      if (plans[f].tune.K != T.K || plans[f].kp.Bt != T.Bt) {
        *err = "facets of one model family need one tile shape";
        return OBIT_DFT_EUNSUPPORTED;
      }
      ctMin = std::min(ctMin, plans[f].kp.ct);
    }
    if (ctMin == T.ct) break;
    T.ct = ctMin;
  }
  // work order: decreasing cost per item (components), then caller order
  std::stable_sort(g.order.begin(), g.order.end(), [&](int a, int b) {
    return fs[a].mc.model.ncomp > fs[b].mc.model.ncomp;
  });
  std::vector<KParams> kps;
  std::vector<int> starts(1, 0);
  std::vector<BlockDesc> blocks;
  std::vector<size_t> blkOff;
  size_t smem = 0;
  long long items = 0, evals = 0;
  for (int f : g.order) {
    const Plan& p = plans[f];
    blkOff.push_back(blocks.size());
    blocks.insert(blocks.end(), p.blocks.begin(), p.blocks.end());
    smem = std::max(smem, p.smemBytes);
    long long n = 0;
    if (fs[f].nvis > 0 && fs[f].mc.model.ncomp > 0 && p.kp.nblocks > 0)
      n = (long long)((fs[f].nvis + p.kp.R - 1) / p.kp.R) * p.kp.nBlockTiles;
    items += n;
    if (items > (long long)INT32_MAX - 1) {
      *err = "batch has more than 2^31 work items";
      return OBIT_DFT_EUNSUPPORTED;
    }
    evals += (long long)fs[f].nvis * fs[f].evalsPerRow;
    starts.push_back((int)items);
  }
  CUDA_TRY(cudaMalloc(&g.d_blocks, sizeof(BlockDesc) * std::max<size_t>(1, blocks.size())));
  CUDA_TRY(cudaMalloc(&g.d_params, sizeof(KParams) * g.order.size()));
  CUDA_TRY(cudaMalloc(&g.d_itemStart, sizeof(int) * starts.size()));
  CUDA_TRY(cudaMalloc(&g.d_counter, sizeof(int)));
  if (!blocks.empty())
    CUDA_TRY(cudaMemcpy(g.d_blocks, blocks.data(), sizeof(BlockDesc) * blocks.size(),
                        cudaMemcpyHostToDevice));
  for (size_t i = 0; i < g.order.size(); i++) {
    const int f = g.order[i];
    KParams kp = plans[f].kp;
    kp.vis = fs[f].d_vis;
    kp.nvis = fs[f].nvis;
    kp.rowBase = 0;
    kp.comps = d_comps + fs[f].compOff;
    kp.ncomp = fs[f].mc.model.ncomp;
    kp.errFlag = d_err;
    kp.blocks = g.d_blocks + blkOff[i];
    kp.ct = T.ct;
    kps.push_back(kp);
  }
  CUDA_TRY(cudaMemcpy(g.d_params, kps.data(), sizeof(KParams) * kps.size(), cudaMemcpyHostToDevice));
  g.hkps = kps;
  CUDA_TRY(cudaMemcpy(g.d_itemStart, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(g.d_counter, 0, sizeof(int)));
  int cap = 0;
  int rc = batch_prepare(T.K, g.kind, T.threads, smem, &cap, err);
  if (rc) return rc;
  g.K = T.K;
  g.ct = T.ct;
  g.Bt = T.Bt;
  g.threads = T.threads;
  g.R = T.threads / T.Bt;
  g.smemBytes = smem;
  g.cap = cap;
  g.items = items;
  g.evals = evals;
  g.grid = (int)std::min<long long>(items, cap);
  g.built = true;
  return 0;
}

int launch_group(const Group& g, cudaStream_t st, std::string* err) {
  if (!g.built || g.items <= 0) return 0;
  cudaError_t ce = cudaMemsetAsync(g.d_counter, 0, sizeof(int), st);
  if (ce != cudaSuccess) {
    *err = std::string("counter reset: ") + cudaGetErrorString(ce);
    return OBIT_DFT_ECUDA;
  }
  BatchParams bp{};
  bp.facets = g.d_params;
  bp.itemStart = g.d_itemStart;
  bp.nfacet = (int)g.order.size();
  bp.counter = g.d_counter;
  return launch_batch(g.K, g.kind, bp, g.grid, g.threads, g.smemBytes, st, err);
}

int ensure_built(ObitDFTBatch* b) {
  std::string err;
  for (Group& g : b->groups)
    if (!g.built) {
      int rc = build_group(g, b->facets, b->d_comps, b->d_err, &err);
      if (rc) return fail(rc, err);
    }
  return 0;
}

const Group* main_group(const ObitDFTBatch* b) {
  const Group* m = nullptr;
  for (const Group& g : b->groups)
    if (!m || g.evals > m->evals) m = &g;
  return m;
}

// Streamed run: build the waves, their parameter blocks and the captured graph
// for host records h (one pointer per facet) and a staging area of
// stagingBytes, unless the current graph was built for the same.
int build_host_run(ObitDFTBatch* b, float* const* h, long long stagingBytes) {
  HostRun& r = b->host;
  const size_t nf = b->facets.size();
  if (r.exec && r.stagingBytes == stagingBytes && r.h.size() == nf && std::equal(r.h.begin(), r.h.end(), h))
    return OBIT_DFT_OK;
  free_host_run(r);
  // two halves, each a multiple of 64 floats
  const size_t half = (size_t)(stagingBytes / (long long)sizeof(float) / 2) / 64 * 64;
  // facet -> (group, position in the group's work order)
  std::vector<int> grp(nf, -1), pos(nf, -1);
  for (size_t gi = 0; gi < b->groups.size(); gi++)
    for (size_t k = 0; k < b->groups[gi].order.size(); k++) {
      grp[b->groups[gi].order[k]] = (int)gi;
      pos[b->groups[gi].order[k]] = (int)k;
    }
  // waves: consecutive pieces of rows, facet after facet, each wave within half
  struct Piece {
    int f, r0, n;
    size_t off;  // floats into the wave's half
  };
  std::vector<std::vector<Piece>> waves(1);
  size_t used = 0;
  for (size_t f = 0; f < nf; f++) {
    const Facet& fc = b->facets[f];
    const size_t lrec = (size_t)fc.L.lrec;
    if (fc.nvis > 0 && lrec > half)
      return fail(OBIT_DFT_EBADARG, "staging area smaller than two records of facet " + std::to_string(f));
    int r0 = 0;
    while (r0 < fc.nvis) {
      size_t fit = (half - used) / lrec;
      if (fit == 0) {
        waves.emplace_back();
        used = 0;
        continue;
      }
      const int n = (int)std::min<size_t>(fit, (size_t)(fc.nvis - r0));
      waves.back().push_back({(int)f, r0, n, used});
      used += (size_t)n * lrec;
      r0 += n;
    }
  }
  if (waves.back().empty()) waves.pop_back();
  // per (wave, group): parameter blocks of the pieces in the group's work order
  const size_t ng = b->groups.size();
  std::vector<KParams> kps;
  std::vector<int> starts;
  struct Launch {
    size_t wave, group, params, start, pieces;
    long long items;
  };
  std::vector<Launch> launches;
  CUDA_TRY(cudaMalloc(&r.d_stage, sizeof(float) * std::max<size_t>(64, 2 * half)));
  for (size_t w = 0; w < waves.size(); w++) {
    for (size_t gi = 0; gi < ng; gi++) {
      const Group& g = b->groups[gi];
      std::vector<Piece> ps;
      for (const Piece& pc : waves[w])
        if (grp[pc.f] == (int)gi) ps.push_back(pc);
      std::stable_sort(ps.begin(), ps.end(), [&](const Piece& a, const Piece& c) { return pos[a.f] < pos[c.f]; });
      if (ps.empty() || !g.built) continue;
      Launch L{w, gi, kps.size(), starts.size(), ps.size(), 0};
      starts.push_back(0);
      for (const Piece& pc : ps) {
        KParams kp = g.hkps[pos[pc.f]];
        kp.vis = r.d_stage + (w % 2) * half + pc.off;
        kp.nvis = pc.n;
        kp.rowBase = 0;
        if (kp.ncomp > 0 && kp.nblocks > 0) L.items += (long long)((pc.n + kp.R - 1) / kp.R) * kp.nBlockTiles;
        kps.push_back(kp);
        starts.push_back((int)L.items);
      }
      if (L.items > (long long)INT32_MAX - 1) return fail(OBIT_DFT_EUNSUPPORTED, "wave has more than 2^31 work items");
      launches.push_back(L);
    }
  }
  CUDA_TRY(cudaMalloc(&r.d_params, sizeof(KParams) * std::max<size_t>(1, kps.size())));
  CUDA_TRY(cudaMalloc(&r.d_starts, sizeof(int) * std::max<size_t>(1, starts.size())));
  CUDA_TRY(cudaMalloc(&r.d_counters, sizeof(int) * std::max<size_t>(1, launches.size())));
  if (!kps.empty())
    CUDA_TRY(cudaMemcpy(r.d_params, kps.data(), sizeof(KParams) * kps.size(), cudaMemcpyHostToDevice));
  if (!starts.empty())
    CUDA_TRY(cudaMemcpy(r.d_starts, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaStreamCreateWithFlags(&r.copyStream, cudaStreamNonBlocking));
  // events: fork, per wave "uploaded" and "applied", join
  const size_t nw = waves.size();
  r.events.resize(2 * nw + 2);
  for (cudaEvent_t& e : r.events) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t fork = r.events[0], join = r.events[1];
  auto up = [&](size_t w) { return r.events[2 + 2 * w]; };
  auto done = [&](size_t w) { return r.events[3 + 2 * w]; };
  // capture: copies in order on the copy stream (H2D of wave w after the D2H
  // of wave w - 2, which used the same half), kernels on the capture stream
  std::string err;
  int rc = 0;
  CUDA_TRY(cudaStreamBeginCapture(b->capStream, cudaStreamCaptureModeThreadLocal));
  cudaStream_t cs = b->capStream, cp = r.copyStream;
  auto copy_wave = [&](size_t w, bool toDevice) -> cudaError_t {
    for (const Piece& pc : waves[w]) {
      const Facet& fc = b->facets[pc.f];
      float* dev = r.d_stage + (w % 2) * half + pc.off;
      float* host = h[pc.f] + (size_t)pc.r0 * fc.L.lrec;
      const size_t bytes = sizeof(float) * (size_t)pc.n * fc.L.lrec;
      cudaError_t ce = toDevice ? cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, cp)
                                : cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, cp);
      if (ce != cudaSuccess) return ce;
      if (toDevice) r.h2dBytes += (long long)bytes;
    }
    return cudaSuccess;
  };
  cudaError_t ce = cudaEventRecord(fork, cs);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cp, fork, 0);
  size_t li = 0;
  for (size_t w = 0; w < nw && ce == cudaSuccess && !rc; w++) {
    if (w >= 2) {  // the half of wave w is free once wave w - 2 is back on the host
      ce = cudaStreamWaitEvent(cp, done(w - 2), 0);
      if (ce == cudaSuccess) ce = copy_wave(w - 2, false);
    }
    if (ce == cudaSuccess) ce = copy_wave(w, true);
    if (ce == cudaSuccess) ce = cudaEventRecord(up(w), cp);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cs, up(w), 0);
    for (; li < launches.size() && launches[li].wave == w && ce == cudaSuccess && !rc; li++) {
      const Launch& L = launches[li];
      const Group& g = b->groups[L.group];
      if (L.items <= 0) continue;
      ce = cudaMemsetAsync(r.d_counters + li, 0, sizeof(int), cs);
      if (ce != cudaSuccess) break;
      BatchParams bp{};
      bp.facets = r.d_params + L.params;
      bp.itemStart = r.d_starts + L.start;
      bp.nfacet = (int)L.pieces;
      bp.counter = r.d_counters + li;
      rc = launch_batch(g.K, g.kind, bp, (int)std::min<long long>(L.items, g.cap), g.threads, g.smemBytes, cs, &err);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(done(w), cs);
  }
  for (size_t w = (nw >= 2 ? nw - 2 : 0); w < nw && ce == cudaSuccess; w++) {
    ce = cudaStreamWaitEvent(cp, done(w), 0);
    if (ce == cudaSuccess) ce = copy_wave(w, false);
  }
  if (ce == cudaSuccess) ce = cudaEventRecord(join, cp);
  if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cs, join, 0);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce2 = cudaStreamEndCapture(cs, &graph);
  if (rc || ce != cudaSuccess || ce2 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    free_host_run(r);
    if (rc) return fail(rc, err);
    return fail(OBIT_DFT_ECUDA, std::string("streamed batch capture: ") +
                                    cudaGetErrorString(ce != cudaSuccess ? ce : ce2));
  }
  r.graph = graph;
  ce = cudaGraphInstantiate(&r.exec, r.graph, 0);
  if (ce != cudaSuccess) {
    free_host_run(r);
    return fail(OBIT_DFT_ECUDA, std::string("streamed batch instantiate: ") + cudaGetErrorString(ce));
  }
  r.h.assign(h, h + nf);
  r.stagingBytes = stagingBytes;
  r.waves = (int)nw;
  return OBIT_DFT_OK;
}

}  // namespace

extern "C" int obit_dft_batch_create(const ObitDFTFacet* in, int nfacet, ObitDFTBatch** out) {
  set_last_error("");
  if (!out) return fail(OBIT_DFT_EBADARG, "NULL output handle");
  *out = nullptr;
  if (nfacet < 0 || (nfacet > 0 && !in)) return fail(OBIT_DFT_EBADARG, "bad facet array");
  std::unique_ptr<ObitDFTBatch> b(new ObitDFTBatch());
  CUDA_TRY(cudaGetDevice(&b->device));
  std::string err;
  size_t compFloats = 0;
  b->facets.resize(nfacet);
  for (int i = 0; i < nfacet; i++) {
    const ObitDFTFacet& s = in[i];
    Facet& f = b->facets[i];
    if (!s.visInfo || !s.modelInfo) return fail(OBIT_DFT_EBADARG, "facet " + std::to_string(i) + ": NULL descriptor");
    if (s.nvis < 0 || (s.nvis > 0 && !s.d_vis))
      return fail(OBIT_DFT_EBADARG, "facet " + std::to_string(i) + ": bad record buffer");
    int rc = model_from_info(s.modelInfo, s.modelInfo->nmodel[0], s.modelInfo->size, s.visInfo, &f.mc, &err);
    FreqSide fs;
    if (!rc && s.freqArr) {
      if (!(s.uvRefFreq > 0.0)) return fail(OBIT_DFT_EBADARG, "facet " + std::to_string(i) + ": bad reference frequency");
      const int nfreq = s.visInfo->nchan * std::max(1, s.visInfo->nIF);
      fs.have = true;
      fs.freqArr.assign(s.freqArr, s.freqArr + nfreq);
      fs.uvRef = s.uvRefFreq;
      fs.modelRef = s.modelRefFreq;
      if (s.specFreq && s.nSpec > 0) fs.specFreq.assign(s.specFreq, s.specFreq + s.nSpec);
    }
    PolnRules pr;
    pr.cpuRules = s.cpuRules != 0;
    pr.stokFactor = s.stokFactor;
    pr.doFlip = s.doFlip;
    if (!rc) rc = layout_from_info(s.visInfo, f.mc, fs, &f.L, &err);
    if (!rc) rc = apply_from_info(f.mc, pr, f.L, &f.A, &err);
    if (rc) return fail(rc, "facet " + std::to_string(i) + ": " + err);
    f.d_vis = s.d_vis;
    f.nvis = s.nvis;
    f.compOff = compFloats;
    compFloats += round_up((size_t)f.mc.model.ncomp * comp_stride(f.mc.model), 64);
    f.evalsPerRow = (long long)(f.L.chane - f.L.chanb + 1) * (f.L.ife - f.L.ifb + 1) * f.mc.model.ncomp;
  }
  CUDA_TRY(cudaMalloc(&b->d_err, sizeof(int)));
  CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(int)));
  CUDA_TRY(cudaMalloc(&b->d_comps, sizeof(float) * std::max<size_t>(64, compFloats)));
  for (int i = 0; i < nfacet; i++) {
    int rc = copy_comps(b->d_comps + b->facets[i].compOff, in[i].modelInfo->model[0],
                        b->facets[i].mc.model, 0, &err);
    if (rc) return fail(rc, "facet " + std::to_string(i) + ": " + err);
  }
  CUDA_TRY(cudaDeviceSynchronize());
  // one group per model family, in order of first appearance
  for (int i = 0; i < nfacet; i++) {
    const int kind = b->facets[i].mc.model.kind;
    auto it = std::find_if(b->groups.begin(), b->groups.end(), [&](const Group& g) { return g.kind == kind; });
    if (it == b->groups.end()) {
      b->groups.emplace_back();
      b->groups.back().kind = kind;
      it = b->groups.end() - 1;
    }
    it->order.push_back(i);
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&b->capStream, cudaStreamNonBlocking));
  int rc = ensure_built(b.get());
  if (rc) {
    obit_dft_batch_destroy(b.release());
    return rc;
  }
  *out = b.release();
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_set_tile(ObitDFTBatch* b, int K, int ct, int Bt, int threads) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  if (K && !batch_kernel_exists(K)) return fail(OBIT_DFT_EBADARG, "unsupported channels per thread");
  if (ct < 0 || Bt < 0 || (Bt & (Bt - 1)) || (threads && threads != 128 && threads != 256))
    return fail(OBIT_DFT_EBADARG, "bad tile shape");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaDeviceSynchronize());
  drop_graph(b);
  for (Group& g : b->groups) {
    g.tune.K = K;
    g.tune.ct = ct ? ct : 128;
    g.tune.Bt = Bt;
    g.tune.threads = threads ? threads : 256;
    free_group(g);
  }
  return ensure_built(b);
}

extern "C" int obit_dft_batch_run(ObitDFTBatch* b, void* stream) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  CUDA_TRY(cudaSetDevice(b->device));
  int rc = ensure_built(b);
  if (rc) return rc;
  if (!b->exec) {
    std::string err;
    CUDA_TRY(cudaStreamBeginCapture(b->capStream, cudaStreamCaptureModeThreadLocal));
    for (const Group& g : b->groups) {
      rc = launch_group(g, b->capStream, &err);
      if (rc) break;
    }
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->capStream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return fail(rc, err);
    }
    if (ce != cudaSuccess) return fail(OBIT_DFT_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    b->graph = graph;
    ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (ce != cudaSuccess) {
      drop_graph(b);
      return fail(OBIT_DFT_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
  }
  CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_run_host(ObitDFTBatch* b, float* const* h_vis, long long stagingBytes,
                                       void* stream, long long* info) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  if (!h_vis && !b->facets.empty()) return fail(OBIT_DFT_EBADARG, "NULL host record pointers");
  for (size_t f = 0; f < b->facets.size(); f++)
    if (b->facets[f].nvis > 0 && !h_vis[f])
      return fail(OBIT_DFT_EBADARG, "facet " + std::to_string(f) + ": NULL host records");
  if (stagingBytes < 2 * 64 * (long long)sizeof(float)) return fail(OBIT_DFT_EBADARG, "staging area too small");
  CUDA_TRY(cudaSetDevice(b->device));
  int rc = ensure_built(b);
  if (rc) return rc;
  rc = build_host_run(b, h_vis, stagingBytes);
  if (rc) return rc;
  if (info) {
    info[0] = b->host.waves;
    info[1] = b->host.h2dBytes;
  }
  CUDA_TRY(cudaGraphLaunch(b->host.exec, (cudaStream_t)stream));
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_run_per_facet(ObitDFTBatch* b, int flavor, void* stream) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  if (flavor != kFlavorRecur && flavor != kFlavorPlain) return fail(OBIT_DFT_EBADARG, "unknown flavor");
  CUDA_TRY(cudaSetDevice(b->device));
  std::string err;
  for (size_t i = 0; i < b->facets.size(); i++) {
    Facet& f = b->facets[i];
    if (!f.haveSingle[flavor]) {
      TuneDesc T;
      T.flavor = flavor;
      int rc = build_plan(f.L, f.mc.model, f.A, T, &f.single[flavor], &err);
      if (rc) return fail(rc, "facet " + std::to_string(i) + ": " + err);
      f.haveSingle[flavor] = true;
    }
    int rc = launch_plan(f.single[flavor], f.d_vis, 0, f.nvis, b->d_comps + f.compOff, b->d_err,
                         (cudaStream_t)stream, &err);
    if (rc) return fail(rc, "facet " + std::to_string(i) + ": " + err);
  }
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_autotune(ObitDFTBatch* b, void* stream, int* best) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  CUDA_TRY(cudaSetDevice(b->device));
  cudaStream_t st = (cudaStream_t)stream;
  std::string err;
  // Row samples of the facets (at least one 64-row tile each), copied into
  // scratch so the candidates leave the records alone: every candidate is timed
  // on a sample of about 1e11 evaluations, then the three fastest again, twice
  // each, on one four times larger, where the choice between near-equal shapes
  // is no longer decided by timing noise and sample-sized tails.
  long long total = 0;
  for (const Facet& f : b->facets) total += (long long)f.nvis * f.evalsPerRow;
  std::vector<float*> scratches;
  auto make_sample = [&](double evals, std::vector<Facet>* sample) -> int {
    const double frac = total > 0 ? std::min(1.0, evals / (double)total) : 1.0;
    sample->assign(b->facets.size(), Facet());
    std::vector<size_t> off(b->facets.size());
    size_t floats = 0;
    for (size_t i = 0; i < b->facets.size(); i++) {
      const Facet& f = b->facets[i];
      Facet& s = (*sample)[i];
      s.mc = f.mc;
      s.L = f.L;
      s.A = f.A;
      s.compOff = f.compOff;
      s.evalsPerRow = f.evalsPerRow;
      s.nvis = (int)std::min<long long>(f.nvis, std::max<long long>(64, (long long)std::ceil(f.nvis * frac)));
      off[i] = floats;
      floats += round_up((size_t)s.nvis * f.L.lrec, 64);
    }
    float* scratch = nullptr;
    cudaError_t ce = cudaMalloc(&scratch, sizeof(float) * std::max<size_t>(64, floats));
    if (ce != cudaSuccess) return fail(OBIT_DFT_ECUDA, std::string("sample buffer: ") + cudaGetErrorString(ce));
    scratches.push_back(scratch);
    for (size_t i = 0; i < sample->size(); i++) {
      Facet& s = (*sample)[i];
      s.d_vis = scratch + off[i];
      if (s.nvis > 0) {
        ce = cudaMemcpyAsync(s.d_vis, b->facets[i].d_vis, sizeof(float) * (size_t)s.nvis * b->facets[i].L.lrec,
                             cudaMemcpyDeviceToDevice, st);
        if (ce != cudaSuccess) return fail(OBIT_DFT_ECUDA, std::string("sample copy: ") + cudaGetErrorString(ce));
      }
    }
    return OBIT_DFT_OK;
  };
  auto free_samples = [&]() {
    cudaStreamSynchronize(st);
    for (float* p : scratches) cudaFree(p);
    scratches.clear();
  };
  std::vector<Facet> small, large;
  int rcAll = make_sample(1.0e11, &small);
  if (!rcAll) rcAll = make_sample(4.0e11, &large);
  if (rcAll) {
    free_samples();
    return rcAll;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int tried = 0;
  for (Group& g : b->groups) {
    if (g.order.empty()) continue;
    struct Cand { int K, threads, Bt, ct; double rate; };
    std::vector<Cand> cands;
    for (int K : {16, 32})
      for (int threads : {256, 128})
        for (int Bt = 1; Bt <= kMaxBt && threads / Bt >= 8; Bt *= 2)
          for (int ct : {64, 128})
            if (Bt >= 4) cands.push_back({K, threads, Bt, ct, -1.0});
    // evaluations per millisecond of the best of `reps` timed launches (after
    // one warm-up) of a candidate on a sample; 0 if the shape does not plan,
    // -1 on a launch failure
    auto time_cand = [&](const Cand& c, std::vector<Facet>& sample, int reps, TuneDesc* chosen) {
      Group t;
      t.kind = g.kind;
      t.order = g.order;
      t.tune.K = c.K;
      t.tune.threads = c.threads;
      t.tune.Bt = c.Bt;
      t.tune.ct = c.ct;
      if (build_group(t, sample, b->d_comps, b->d_err, &err) || t.items <= 0) {
        free_group(t);
        return 0.0;
      }
      bool ok = launch_group(t, st, &err) == 0;  // warm-up
      float best = 0.f;
      for (int r = 0; r < reps && ok; r++) {
        float ms = 0.f;
        ok = ok && cudaEventRecord(e0, st) == cudaSuccess;
        ok = ok && launch_group(t, st, &err) == 0;
        ok = ok && cudaEventRecord(e1, st) == cudaSuccess;
        ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
        ok = ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
        if (ok && ms > 0.f && (best == 0.f || ms < best)) best = ms;
      }
      double rate = (ok && best > 0.f) ? (double)t.evals / best : (ok ? 0.0 : -1.0);
      if (chosen) {
        *chosen = t.tune;
        chosen->K = t.K;
        chosen->Bt = t.Bt;
        chosen->ct = t.ct;
        chosen->threads = t.threads;
      }
      free_group(t);
      return rate;
    };
    for (Cand& c : cands) {
      c.rate = time_cand(c, small, 1, nullptr);
      if (c.rate < 0) {
        rcAll = fail(OBIT_DFT_ECUDA, "autotune launch failed: " + err);
        break;
      }
      if (c.rate > 0) tried++;
    }
    if (rcAll) break;
    std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& c) { return a.rate > c.rate; });
    double bestRate = -1.0;
    TuneDesc bestT = g.tune;
    for (size_t i = 0; i < cands.size() && i < 3 && cands[i].rate > 0; i++) {
      TuneDesc t;
      const double rate = time_cand(cands[i], large, 2, &t);
      if (rate < 0) {
        rcAll = fail(OBIT_DFT_ECUDA, "autotune launch failed: " + err);
        break;
      }
      if (rate > bestRate) {
        bestRate = rate;
        bestT = t;
      }
    }
    if (rcAll) break;
    if (bestRate > 0) {
      g.tune = bestT;
      free_group(g);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  free_samples();
  if (rcAll) return rcAll;
  drop_graph(b);
  int rc = ensure_built(b);
  if (rc) return rc;
  if (best) {
    const Group* m = main_group(b);
    best[0] = m ? m->K : 0;
    best[1] = m ? m->ct : 0;
    best[2] = m ? m->Bt : 0;
    best[3] = m ? m->R : 0;
    best[4] = m ? m->threads : 0;
    best[5] = tried;
  }
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_check(ObitDFTBatch* b) {
  set_last_error("");
  if (!b) return fail(OBIT_DFT_EBADARG, "NULL batch");
  CUDA_TRY(cudaSetDevice(b->device));
  CUDA_TRY(cudaDeviceSynchronize());
  int h = 0;
  CUDA_TRY(cudaMemcpy(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CUDA_TRY(cudaMemset(b->d_err, 0, sizeof(int)));
    std::string msg;
    const int rc = kernel_flag_status(h, &msg);
    return fail(rc, msg);
  }
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_info(ObitDFTBatch* b, long long* info, int n) {
  set_last_error("");
  if (!b || (!info && n > 0)) return fail(OBIT_DFT_EBADARG, "NULL argument");
  long long items = 0, evals = 0, launches = 0;
  for (const Group& g : b->groups) {
    items += g.items;
    evals += g.evals;
    launches += g.items > 0;
  }
  const Group* m = main_group(b);
  const long long v[10] = {(long long)b->facets.size(), launches, items, evals,
                           m ? m->K : 0, m ? m->ct : 0, m ? m->Bt : 0, m ? m->R : 0,
                           m ? m->threads : 0, m ? m->grid : 0};
  for (int i = 0; i < std::min(n, 10); i++) info[i] = v[i];
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_batch_destroy(ObitDFTBatch* b) {
  set_last_error("");
  if (!b) return OBIT_DFT_OK;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  drop_graph(b);
  for (Group& g : b->groups) free_group(g);
  for (Facet& f : b->facets)
    for (int k = 0; k < 2; k++)
      if (f.haveSingle[k]) free_plan(&f.single[k]);
  if (b->d_comps) cudaFree(b->d_comps);
  if (b->d_err) cudaFree(b->d_err);
  if (b->capStream) cudaStreamDestroy(b->capStream);
  delete b;
  return OBIT_DFT_OK;
}
