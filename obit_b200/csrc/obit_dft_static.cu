// obit_dft_calc_noalloc: the DFT subtract / divide / replace for callers that
// cannot allocate device memory.
//
// Some hosts cannot let a library call cudaMalloc: a process whose device
// memory is all owned by its own pool (a caching allocator that must see every
// byte, or a job sized to fill HBM, where an extra allocation can fail in the
// middle of a pass), and latency-bound callers for which cudaFree's implicit
// device-wide synchronization is not acceptable.  The regular entry points keep
// per-GPUInfo state and allocate a padded component table, a channel-block
// table and an error flag.  This entry point instead keeps that scratch in one
// file-scope device array of fixed size (kScratchBytes) and asks the caller
// only for its inputs and outputs.
//
// The array exists once per GPU that loads the library and lives until the
// process exits.  Every call looks up the array's device address
// (cudaGetSymbolAddress) with the caller's device current -- cheap next to the
// copies and the synchronization, and never stale after a context is re-created.
// The call is synchronous: it reads device descriptors on the caller's stream,
// waits for the stream and copies the error flag back, so it must not be made
// while a stream is capturing.  Every call reuses the array and leaves the last
// call's contents behind, so calls that overlap on the GPU (other streams, other
// host threads) race: serialize them.
#include <cuda_runtime.h>

#include <string>

#include "abi_internal.h"
#include "dft_plan.h"

namespace {

using namespace obit;

// Scratch limit: error flag, channel-block table and the padded component table.
constexpr size_t kScratchBytes = 8u << 20;  // 8 MiB
constexpr size_t kFlagBytes = 256;

__device__ __align__(256) unsigned char g_dft_scratch[kScratchBytes];

size_t round256(size_t n) { return (n + 255) & ~(size_t)255; }

// Device address of the scratch array in the current device's context.  Host
// code must not use g_dft_scratch itself: there it names a host-side stand-in.
int scratch_address(unsigned char** out, std::string* err) {
  void* p = nullptr;
  cudaError_t ce = cudaGetSymbolAddress(&p, g_dft_scratch);
  if (ce != cudaSuccess || !p) {
    *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce);
    return OBIT_DFT_ECUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return OBIT_DFT_OK;
}

int failed(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int obit_dft_calc_noalloc(const GPUVisInfo* visInfo, const GPUModelInfo* modelInfo,
                                     const double* freqArr, double uvRefFreq, double modelRefFreq,
                                     const double* specFreq, int nSpec, float* d_vis, int nvis,
                                     void* stream) {
  set_last_error("");
  if (!visInfo || !modelInfo) return failed(OBIT_DFT_EBADARG, "NULL descriptor");
  if (nvis < 0) return failed(OBIT_DFT_EBADARG, "negative record count");
  if (nvis > 0 && !d_vis) return failed(OBIT_DFT_EBADARG, "NULL visibility buffer");
  std::string err;
  cudaStream_t st = (cudaStream_t)stream;
  ModelCfg mc;
  // device descriptors (specIndex, freqScale) are read in order on the caller's stream
  int rc = model_from_info(modelInfo, modelInfo->nmodel[0], modelInfo->size, visInfo, &mc, &err, &st);
  if (rc) return failed(rc, err);
  FreqSide fs;
  if (freqArr) {
    if (!(uvRefFreq > 0.0)) return failed(OBIT_DFT_EBADARG, "bad FP64 reference frequency");
    const int nfreq = visInfo->nchan * (visInfo->nIF > 0 ? visInfo->nIF : 1);
    fs.have = true;
    fs.freqArr.assign(freqArr, freqArr + nfreq);
    fs.uvRef = uvRefFreq;
    fs.modelRef = modelRefFreq;
    if (specFreq && nSpec > 0) fs.specFreq.assign(specFreq, specFreq + nSpec);
  }
  LayoutDesc L;
  ApplyDesc A;
  rc = layout_from_info(visInfo, mc, fs, &L, &err, &st);
  if (!rc) rc = apply_from_info(mc, PolnRules(), L, &A, &err);
  if (rc) return failed(rc, err);
  if (nvis == 0 || mc.model.ncomp == 0) return OBIT_DFT_OK;
  Plan plan;
  TuneDesc T;
  T.ct = 128;  // the tile this entry point plans with (not the planner's 160 choice)
  rc = plan_layout(L, mc.model, A, T, &plan, &err);
  if (rc) return failed(rc, err);

  // scratch layout: [error flag][channel-block table][padded component table]
  const size_t blkBytes = round256(sizeof(BlockDesc) * (size_t)plan.kp.nblocks);
  const size_t compBytes = (size_t)mc.model.ncomp * comp_stride(mc.model) * sizeof(float);
  const size_t need = kFlagBytes + blkBytes + compBytes;
  if (need > kScratchBytes)
    return failed(OBIT_DFT_EUNSUPPORTED,
                  "model needs " + std::to_string(need) + " bytes of scratch; the static limit is " +
                      std::to_string(kScratchBytes) + " (use obit_dft_calc_device)");
  unsigned char* base = nullptr;
  rc = scratch_address(&base, &err);
  if (rc) return failed(rc, err);
  int* d_flag = reinterpret_cast<int*>(base);
  BlockDesc* d_blocks = reinterpret_cast<BlockDesc*>(base + kFlagBytes);
  float* d_comps = reinterpret_cast<float*>(base + kFlagBytes + blkBytes);

  // the previous call's flag and tables are still in the array: clear the flag
  cudaError_t ce = cudaMemsetAsync(d_flag, 0, sizeof(int), st);
  if (ce != cudaSuccess) return failed(OBIT_DFT_ECUDA, std::string("flag clear: ") + cudaGetErrorString(ce));
  rc = finalize_plan(&plan, d_blocks, st, &err);
  if (!rc) rc = copy_comps(d_comps, modelInfo->model[0], mc.model, st, &err);
  if (!rc) rc = launch_plan(plan, d_vis, 0, nvis, d_comps, d_flag, st, &err);
  if (rc) return failed(rc, err);
  // synchronous: the records are final and the flag can be read on return
  int flag = 0;
  ce = cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return failed(OBIT_DFT_ECUDA, std::string("completion: ") + cudaGetErrorString(ce));
  if (flag) {
    std::string msg;
    const int frc = kernel_flag_status(flag, &msg);
    return failed(frc, msg);
  }
  return OBIT_DFT_OK;
}
