// Records resident in device memory across CLEAN major cycles
// (include/obit_dft.h, obit_dft_resident_*).  The reference re-reads the data
// and copies every buffer to the GPU and back each major cycle (the residual
// of ObitDConCleanVisMF's cycle, ObitDConCleanVisMF.c:907, through
// ObitSkyModelSubUV and ObitGPUSkyModel.c:510-517); here the original records
// are uploaded once, and each cycle resets a work copy on the device (a
// device-to-device copy), applies any number of models to it with the
// device-resident calls, and downloads the residual.
#include <cuda_runtime.h>

#include <string>

#include "abi_internal.h"
#include "obit_dft.h"

struct ObitDFTResident {
  int device = 0;
  int nvis = 0, lenvis = 0;
  size_t bytes = 0;
  float* d_orig = nullptr;  // the records as uploaded
  float* d_work = nullptr;  // the copy models are applied to
};

namespace {

int fail(int code, const std::string& msg) {
  obit::set_last_error(msg);
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess)                                                          \
      return fail(OBIT_DFT_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)

void release(ObitDFTResident* r) {
  if (!r) return;
  cudaFree(r->d_orig);
  cudaFree(r->d_work);
  delete r;
}

}  // namespace

extern "C" int obit_dft_resident_create(const float* h_vis, int nvis, int lenvis, void* stream,
                                        ObitDFTResident** out) {
  if (!out) return fail(OBIT_DFT_EBADARG, "resident: null output");
  *out = nullptr;
  if (nvis <= 0 || lenvis <= 0 || !h_vis) return fail(OBIT_DFT_EBADARG, "resident: bad records");
  ObitDFTResident* r = new ObitDFTResident();
  r->nvis = nvis;
  r->lenvis = lenvis;
  r->bytes = sizeof(float) * (size_t)nvis * (size_t)lenvis;
  cudaError_t e = cudaGetDevice(&r->device);
  if (e == cudaSuccess) e = cudaMalloc(&r->d_orig, r->bytes);
  if (e == cudaSuccess) e = cudaMalloc(&r->d_work, r->bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r->d_orig, h_vis, r->bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(r->d_work, r->d_orig, r->bytes, cudaMemcpyDeviceToDevice,
                                            (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) {
    release(r);
    return fail(OBIT_DFT_ECUDA, std::string("resident create: ") + cudaGetErrorString(e));
  }
  *out = r;
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_resident_reset(ObitDFTResident* r, void* stream) {
  if (!r) return fail(OBIT_DFT_EBADARG, "resident: null handle");
  CUDA_TRY(cudaSetDevice(r->device));
  CUDA_TRY(cudaMemcpyAsync(r->d_work, r->d_orig, r->bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return OBIT_DFT_OK;
}

extern "C" float* obit_dft_resident_records(ObitDFTResident* r) { return r ? r->d_work : nullptr; }

extern "C" int obit_dft_resident_download(ObitDFTResident* r, float* h_out, void* stream) {
  if (!r || !h_out) return fail(OBIT_DFT_EBADARG, "resident: null argument");
  CUDA_TRY(cudaSetDevice(r->device));
  CUDA_TRY(cudaMemcpyAsync(h_out, r->d_work, r->bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_resident_destroy(ObitDFTResident* r) {
  if (!r) return OBIT_DFT_OK;
  cudaSetDevice(r->device);
  release(r);
  return OBIT_DFT_OK;
}
