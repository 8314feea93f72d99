// Test infrastructure (never linked into the product): the reference's
// per-component Jones corrections for linear feeds, cudaJonesCor1_Lin_{I,Q,U,V}
// (ObitSystem/Obit/include/CUDALinCorSum.h:104-455), compiled for the host from
// the reference's own header where it lies (oracle/Makefile, target refjones)
// so that the beam oracle's coefficients (oracle_beam.c) can be checked
// against the reference's code rather than a restatement of it.
#include <math.h>
#include <string.h>

#include <cuda_runtime_api.h>  // stream and event types named by the reference's headers

#define __device__
#define __forceinline__ inline
#define __sincosf sincosf
#define HAVE_GPU 1
#define IS_CUDA 1
#include "CUDALinCorSum.h"

// One component: sumVis (XX, XY, YX, YY as re, im) of flux (cos, sin) with the
// Jones pair J1, J2 (8 floats each, XX, XY, YX, YY) for Stokes 1..4.
extern "C" int ref_jones_cor1(int stokType, float flux, float sinPh, float cosPh, const float* J1,
                              const float* J2, float c2p, float s2p, float* out) {
  cudaMatx a, b, sum;
  memcpy(&a, J1, sizeof(a));
  memcpy(&b, J2, sizeof(b));
  cudaMatxZero2C(&sum);
  switch (stokType) {
    case 1: cudaJonesCor1_Lin_I(flux, sinPh, cosPh, &a, &b, c2p, s2p, &sum); break;
    case 2: cudaJonesCor1_Lin_Q(flux, sinPh, cosPh, &a, &b, c2p, s2p, &sum); break;
    case 3: cudaJonesCor1_Lin_U(flux, sinPh, cosPh, &a, &b, c2p, s2p, &sum); break;
    case 4: cudaJonesCor1_Lin_V(flux, sinPh, cosPh, &a, &b, c2p, s2p, &sum); break;
    default: return -1;
  }
  memcpy(out, &sum, sizeof(sum));
  return 0;
}
