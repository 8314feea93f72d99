/* Test infrastructure only: stand-in for the CUDA samples' helper_cuda.h that
 * ObitCUDASkyModel.cu includes.  checkCudaErrors reports a failed runtime call
 * on stderr and continues (the samples' version exits the process). */
#pragma once
#include <cuda_runtime.h>
#include <stdio.h>
#define checkCudaErrors(call)                                                    \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      fprintf(stderr, "reference CUDA call failed: %s\n", cudaGetErrorString(e_)); \
  } while (0)
