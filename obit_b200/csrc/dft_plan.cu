// Planner and launcher for the DFT kernels (see dft_kernels.cuh).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "dft_kernels.cuh"
#include "dft_plan.h"

namespace obit {

namespace {

using KernelFn = void (*)(const KParams);

template <int K, bool kLo>
KernelFn pick_recur(int mode) {
  switch (mode) {
    case kPoint: return dft_recur_kernel<K, kPoint, false, kLo>;
    case kPointSpec: return dft_recur_kernel<K, kPointSpec, false, kLo>;
    case kPointTSpec: return dft_recur_kernel<K, kPointTSpec, false, kLo>;
    case kGauss: return dft_recur_kernel<K, kGauss, false, kLo>;
    case kGaussSpec: return dft_recur_kernel<K, kGaussSpec, false, kLo>;
    case kGaussTSpec: return dft_recur_kernel<K, kGaussTSpec, false, kLo>;
  }
  return nullptr;
}

template <int K, bool kLo>
KernelFn pick_plain(int mode) {
  switch (mode) {
    case kPoint: return dft_plain_kernel<K, kPoint, kLo>;
    case kPointSpec: return dft_plain_kernel<K, kPointSpec, kLo>;
    case kPointTSpec: return dft_plain_kernel<K, kPointTSpec, kLo>;
    case kGauss: return dft_plain_kernel<K, kGauss, kLo>;
    case kGaussSpec: return dft_plain_kernel<K, kGaussSpec, kLo>;
    case kGaussTSpec: return dft_plain_kernel<K, kGaussTSpec, kLo>;
  }
  return nullptr;
}

// Spectral-factored instances: point families with one spectral index, K a
// multiple of 8.
template <int K, bool kLo>
KernelFn pick_spec_factored(int mode) {
  if constexpr (K >= 8 && K % 8 == 0) {
    if (mode == kPointSpec) return dft_recur_kernel<K, kPointSpec, false, kLo, true>;
    if (mode == kPointTSpec) return dft_recur_kernel<K, kPointTSpec, false, kLo, true>;
  }
  return nullptr;
}

// Mixed instances: a Gaussian family with one spectral index whose untapered
// components run as the point family in the spectral-factored form.
template <int K>
KernelFn pick_mixed(int mode) {
  if constexpr (K >= 8 && K % 8 == 0) {
    if (mode == kGaussSpec) return dft_recur_kernel<K, kGaussSpec, false, false, false, true>;
    if (mode == kGaussTSpec) return dft_recur_kernel<K, kGaussTSpec, false, false, false, true>;
  }
  return nullptr;
}

template <bool kLo>
KernelFn pick_flavor(int flavor, int K, int mode, bool fs) {
  if (fs) {
    if (flavor != kFlavorRecur) return nullptr;
    switch (K) {
      case 8: return pick_spec_factored<8, kLo>(mode);
      case 16: return pick_spec_factored<16, kLo>(mode);
      case 32: return pick_spec_factored<32, kLo>(mode);
    }
    return nullptr;
  }
  if (flavor == kFlavorRecur) {
    switch (K) {
      case 2: return pick_recur<2, kLo>(mode);
      case 4: return pick_recur<4, kLo>(mode);
      case 8: return pick_recur<8, kLo>(mode);
      case 16: return pick_recur<16, kLo>(mode);
      case 32: return pick_recur<32, kLo>(mode);
    }
  } else if (flavor == kFlavorPlain) {
    switch (K) {
      case 1: return pick_plain<1, kLo>(mode);
      case 2: return pick_plain<2, kLo>(mode);
      case 4: return pick_plain<4, kLo>(mode);
      case 8: return pick_plain<8, kLo>(mode);
      case 16: return pick_plain<16, kLo>(mode);
    }
  }
  return nullptr;
}

// The wait-limit diagnostic runs its own instance (32 channels, point +
// spectrum) so that no production instance reads the limit at run time; FP64
// positions (lo) select the instances that stage and add the low parts; fs the
// spectral-factored instances.
KernelFn pick_kernel(int flavor, int K, int mode, bool probe, bool lo, bool fs) {
  if (probe)
    return (flavor == kFlavorRecur && K == 32 && mode == kPointSpec && !lo && !fs)
               ? dft_recur_kernel<32, kPointSpec, true>
               : nullptr;
  return lo ? pick_flavor<true>(flavor, K, mode, fs) : pick_flavor<false>(flavor, K, mode, fs);
}

KernelFn plan_kernel(const Plan& plan) {
  if (plan.mixed) {  // no FP64-position or diagnostic instances
    if (plan.tune.flavor != kFlavorRecur || plan.kp.compsLo || plan.kp.waitPolls != kDefaultWaitPolls)
      return nullptr;
    switch (plan.tune.K) {
      case 8: return pick_mixed<8>(plan.model.kind);
      case 16: return pick_mixed<16>(plan.model.kind);
      case 32: return pick_mixed<32>(plan.model.kind);
    }
    return nullptr;
  }
  return pick_kernel(plan.tune.flavor, plan.tune.K, plan.model.kind,
                     plan.kp.waitPolls != kDefaultWaitPolls, plan.kp.compsLo != nullptr,
                     plan.specFactored);
}

}  // namespace

// The dynamic shared-memory limit is an attribute of the kernel function, not
// of a launch: plans of one kernel with different tile sizes share it.  Only
// ever raise it (per device), so that a plan finalized earlier with a larger
// tile still launches after a smaller one was finalized.
int raise_smem_limit(const void* fn, size_t bytes, std::string* err) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limit;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[{dev, fn}];
  if (bytes <= cur) return 0;
  cudaError_t ce = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (ce != cudaSuccess) {
    *err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ce);
    return 2;
  }
  cur = bytes;
  return 0;
}

int build_plan(const LayoutDesc& L, const ModelDesc& M, const ApplyDesc& A, const TuneDesc& T,
               Plan* plan, std::string* err) {
  int rc = plan_layout(L, M, A, T, plan, err);
  if (rc) return rc;
  return finalize_plan(plan, nullptr, 0, err);
}

int finalize_plan(Plan* plan, BlockDesc* dst, cudaStream_t stream, std::string* err) {
  KParams& kp = plan->kp;
  const int threads = plan->threads;
  const int nblocks = kp.nblocks;
  const bool probe = kp.waitPolls != kDefaultWaitPolls;
  KernelFn fn = plan_kernel(*plan);
  if (!fn) {
    *err = probe ? "the wait-limit diagnostic runs 32-channel point+spectrum plans without FP64 positions only"
                 : "no kernel for this flavor and channel count";
    return 3;
  }
  if (int rc = raise_smem_limit((const void*)fn, plan->smemBytes, err)) return rc;
  cudaError_t ce;
  int perSM = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, threads, plan->smemBytes);
  if (ce != cudaSuccess || perSM < 1) {
    *err = std::string("kernel cannot be resident: ") + cudaGetErrorString(ce);
    return 2;
  }
  plan->gridCap = perSM * nsm;

  BlockDesc* table = dst;
  if (!table) {
    ce = cudaMalloc(&plan->d_blocks, sizeof(BlockDesc) * (size_t)std::max(1, nblocks));
    if (ce != cudaSuccess) {
      *err = std::string("cudaMalloc blocks: ") + cudaGetErrorString(ce);
      return 2;
    }
    table = plan->d_blocks;
  }
  // an owned table is filled synchronously (later launches may use any
  // stream); a caller's buffer is filled in order on the caller's stream
  if (nblocks)
    ce = dst ? cudaMemcpyAsync(table, plan->blocks.data(), sizeof(BlockDesc) * nblocks,
                               cudaMemcpyHostToDevice, stream)
             : cudaMemcpy(table, plan->blocks.data(), sizeof(BlockDesc) * nblocks,
                          cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    *err = std::string("block table copy: ") + cudaGetErrorString(ce);
    return 2;
  }
  kp.blocks = table;
  return 0;
}

void free_plan(Plan* plan) {
  if (plan->d_blocks) cudaFree(plan->d_blocks);
  plan->d_blocks = nullptr;
  plan->blocks.clear();
}

int launch_plan(const Plan& plan, float* d_vis, int rowBase, int nvis, const float* d_comps,
                int* d_err, cudaStream_t stream, std::string* err) {
  // An empty model leaves the data untouched for every operation, as the
  // reference CPU DFT does (ObitSkyModel.c:2405, "if (ncomp<=0) goto finish").
  if (nvis <= 0 || plan.kp.nblocks <= 0 || plan.model.ncomp <= 0) return 0;
  KParams kp = plan.kp;
  kp.vis = d_vis;
  kp.rowBase = rowBase;
  kp.nvis = nvis;
  kp.comps = d_comps;
  kp.ncomp = plan.model.ncomp;
  kp.compsPt = nullptr;
  kp.ncompPt = 0;
  if (plan.mixed) {  // point sub-table first, the Gaussian rows after it
    kp.compsPt = d_comps;
    kp.ncompPt = plan.model.ncompPt;
    kp.comps = d_comps + (size_t)plan.model.ncompPt * kp.cstride;
  }
  kp.errFlag = d_err;
  const long long nItems = (long long)((nvis + kp.R - 1) / kp.R) * kp.nBlockTiles;
  const int grid = (int)std::min<long long>(nItems, (long long)plan.gridCap);
  KernelFn fn = plan_kernel(plan);
  if (!fn) {
    *err = "no kernel for this plan";
    return 3;
  }
  // an error left by an earlier, unrelated runtime call would otherwise be
  // reported as this launch's
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("error pending before the kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  fn<<<grid, plan.threads, plan.smemBytes, stream>>>(kp);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, fn);
    cudaGetLastError();
    *err = std::string("kernel launch (grid ") + std::to_string(grid) + ", " +
           std::to_string(plan.threads) + " threads, " + std::to_string(plan.smemBytes) +
           " B shared; kernel allows " + std::to_string(fa.maxDynamicSharedSizeBytes) +
           " B dynamic, " + std::to_string(fa.sharedSizeBytes) + " B static, " +
           std::to_string(fa.maxThreadsPerBlock) + " threads): " + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
