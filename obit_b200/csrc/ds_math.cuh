// Split-FP32 ("double-single") arithmetic used to form the DFT phase argument
// without FP64.  A value is carried as an unevaluated sum hi + lo of two floats
// with |lo| <= ulp(hi)/2, giving ~48 significant bits.
//
// The building blocks are the classical error-free transformations:
//   two_sum   (Knuth, TAOCP vol. 2, 4.2.2, Theorem B)
//   fast_two_sum (Dekker 1971, requires |a| >= |b|)
//   two_prod  via fused multiply-add (exact product error)
// and the Dekker/Bailey double-single product.
#pragma once
#include <cuda_runtime.h>

namespace obit {

// 1/(2 pi) as a split-FP32 pair: hi = float(1/(2 pi)), lo = float(1/(2 pi) - hi).
constexpr float kInv2PiHi = 0.15915493667125702f;
constexpr float kInv2PiLo = 6.4206382432985265e-09f;

struct ds {
  float hi, lo;
};

__device__ __forceinline__ ds two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}

__device__ __forceinline__ ds fast_two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float e = __fsub_rn(b, __fsub_rn(s, a));
  return {s, e};
}

__device__ __forceinline__ ds two_prod(float a, float b) {
  float p = __fmul_rn(a, b);
  float e = __fmaf_rn(a, b, -p);
  return {p, e};
}

// (a.hi + a.lo) * (b.hi + b.lo), relative error ~2^-46.
__device__ __forceinline__ ds ds_mul(ds a, ds b) {
  float p = __fmul_rn(a.hi, b.hi);
  float e = __fmaf_rn(a.hi, b.hi, -p);
  e = __fmaf_rn(a.hi, b.lo, __fmaf_rn(a.lo, b.hi, e));
  return fast_two_sum(p, e);
}

// x*u + y*v + z*w for float inputs, returned as a double-single.  The three
// products are exact as pairs; the sums are error-free except for the final
// accumulation of the low parts.
__device__ __forceinline__ ds ds_dot3(float x, float u, float y, float v, float z, float w) {
  ds p1 = two_prod(x, u);
  ds p2 = two_prod(y, v);
  ds p3 = two_prod(z, w);
  ds s = two_sum(p1.hi, p2.hi);
  ds t = two_sum(s.hi, p3.hi);
  float lo = __fadd_rn(__fadd_rn(__fadd_rn(p1.lo, p2.lo), __fadd_rn(p3.lo, s.lo)), t.lo);
  return fast_two_sum(t.hi, lo);
}

// (x + xl) u + (y + yl) v + (z + zl) w for coefficients given as float pairs
// (x = nearest float of an FP64 value, xl = the float of the remainder): the
// products of the low parts, at most 2^-24 of the leading terms, enter the
// low word of the result.
__device__ __forceinline__ ds ds_dot3_lo(float x, float xl, float u, float y, float yl, float v,
                                         float z, float zl, float w) {
  ds p1 = two_prod(x, u);
  ds p2 = two_prod(y, v);
  ds p3 = two_prod(z, w);
  ds s = two_sum(p1.hi, p2.hi);
  ds t = two_sum(s.hi, p3.hi);
  float lo = __fadd_rn(__fadd_rn(__fadd_rn(p1.lo, p2.lo), __fadd_rn(p3.lo, s.lo)), t.lo);
  lo = __fmaf_rn(xl, u, __fmaf_rn(yl, v, __fmaf_rn(zl, w, lo)));
  return fast_two_sum(t.hi, lo);
}

// Fractional turns of the product (a.hi + a.lo) * (b.hi + b.lo) as one float in
// [-0.5, 0.5] (up to rounding): the exact high product and its error term, the
// cross terms, then the nearest integer removed from the high part.  Absolute
// error ~2^-24 turns plus 2^-46 of the product; used where only the reduced
// angle is needed.
__device__ __forceinline__ float ds_mul_frac(ds a, ds b) {
  const float hi = __fmul_rn(a.hi, b.hi);
  const float lo = __fmaf_rn(a.hi, b.lo, __fmaf_rn(a.lo, b.hi, __fmaf_rn(a.hi, b.hi, -hi)));
  return __fadd_rn(__fsub_rn(hi, rintf(hi)), lo);
}

// Fractional part of a double-single number of turns, in [-0.5, 0.5] (up to
// rounding), returned as float plus the float rounding residual.
__device__ __forceinline__ ds ds_frac_turns(ds t) {
  float n = rintf(t.hi);
  float d = __fsub_rn(t.hi, n);  // exact: n is the nearest integer to t.hi
  ds r = fast_two_sum(d, t.lo);  // |d| <= 0.5 >= |t.lo| except when both tiny
  return r;
}

}  // namespace obit
