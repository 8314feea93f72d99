// Instantiations, attributes and launch of the batched recurrence kernel
// (dft_recur_batch_kernel in dft_kernels.cuh), compiled apart from the
// single-facet kernels so the two sets build in parallel.
#include <algorithm>
#include <string>

#include "dft_kernels.cuh"
#include "dft_plan.h"

namespace obit {

namespace {

using BatchFn = void (*)(const BatchParams);

template <int K>
BatchFn pick_batch_k(int mode) {
  switch (mode) {
    case kPoint: return dft_recur_batch_kernel<K, kPoint>;
    case kPointSpec: return dft_recur_batch_kernel<K, kPointSpec>;
    case kPointTSpec: return dft_recur_batch_kernel<K, kPointTSpec>;
    case kGauss: return dft_recur_batch_kernel<K, kGauss>;
    case kGaussSpec: return dft_recur_batch_kernel<K, kGaussSpec>;
    case kGaussTSpec: return dft_recur_batch_kernel<K, kGaussTSpec>;
  }
  return nullptr;
}

BatchFn pick_batch(int K, int mode) {
  switch (K) {
    case 2: return pick_batch_k<2>(mode);
    case 4: return pick_batch_k<4>(mode);
    case 8: return pick_batch_k<8>(mode);
    case 16: return pick_batch_k<16>(mode);
    case 32: return pick_batch_k<32>(mode);
  }
  return nullptr;
}

}  // namespace

bool batch_kernel_exists(int K) { return pick_batch(K, kPoint) != nullptr; }

int batch_prepare(int K, int mode, int threads, size_t smemBytes, int* gridCap, std::string* err) {
  BatchFn fn = pick_batch(K, mode);
  if (!fn) {
    *err = "no batched kernel for K=" + std::to_string(K);
    return 3;
  }
  if (int rc = raise_smem_limit((const void*)fn, smemBytes, err)) return rc;
  cudaError_t ce;
  int perSM = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, threads, smemBytes);
  if (ce != cudaSuccess || perSM < 1) {
    *err = std::string("batched kernel cannot be resident: ") + cudaGetErrorString(ce);
    return 2;
  }
  *gridCap = perSM * nsm;
  return 0;
}

int launch_batch(int K, int mode, const BatchParams& bp, int grid, int threads, size_t smemBytes,
                 cudaStream_t stream, std::string* err) {
  BatchFn fn = pick_batch(K, mode);
  if (!fn || grid < 1) {
    *err = "invalid batched launch";
    return 3;
  }
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("error pending before the batched launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  fn<<<grid, threads, smemBytes, stream>>>(bp);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("batched kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
