// Packed FP32 pair arithmetic (PTX add/sub/mul/fma .f32x2, sm_100a).
//
// One instruction performs the same IEEE single-precision operation (round
// to nearest even, no flush) on both halves of a 64-bit register pair, so a
// warp instruction carries 64 FP32 operations: the FP32 pipe stays full at
// half the issue rate of scalar code.
#pragma once
#include <cuda_runtime.h>

namespace obit {

using f2x = unsigned long long;  // {lo, hi} float pair in one 64-bit register

__device__ __forceinline__ f2x pk2(float lo, float hi) {
  f2x r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}

__device__ __forceinline__ void up2(f2x v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ f2x add2(f2x a, f2x b) {
  f2x d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

__device__ __forceinline__ f2x sub2(f2x a, f2x b) {
  f2x d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
  f2x d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// a * b + c, one rounding per half
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
  f2x d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

}  // namespace obit
