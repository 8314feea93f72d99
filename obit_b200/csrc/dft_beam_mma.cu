// Beam-corrected DFT, tensor-core form (every model family on uniformly
// spaced channels).
//
// The model of record r at channel k for correlation q is
//   M_q(r, k) = sum_c C_q(pair(r), c, plane) A_c(k) exp(2 pi i P(r, c) f_k):
// per record, a (channel x component) matrix of phasors times a (component x
// correlation) matrix of the Jones coefficients of the record's antenna-type
// pair.  The reference forms every term on the FP32 pipe with the Jones
// products recomputed per evaluation (ObitCUDABeamModel.cu:139-1226); here the
// products go to the tensor cores.  A CTA item is kBeamMmaWarps records (one
// per warp) x one run of at most 256 uniformly spaced channels in one Jones
// plane (BeamSeg).  The warp forms its record's phasors in registers and
// multiplies them by the coefficients with mma.sync m16n8k8 (TF32 inputs, FP32
// accumulate): the A operand is produced per warp in registers and changes for
// every 16 x 8 tile, which the register-fed product takes directly (tcgen05.mma
// reads A from shared or tensor memory, which would add a store, a fence and a
// CTA-wide hand-off per tile), with the coefficient matrix (8 columns) as B:
//   rows     16 channels of the run (lane group g = lane / 4 holds g, g + 8)
//   k        4 components: real parts at k = 0..3, imaginary parts at 4..7
//   columns  re, im of the model correlations XX, XY, YX, YY (RR, RL, LR, LL)
// Real form of the complex product: column 2q takes Vr Cr - Vi Ci and column
// 2q + 1 takes Vr Ci + Vi Cr.  FP32 accuracy from TF32 inputs by the
// three-product split of error-corrected TF32 products (each operand x = hi +
// lo with hi carrying TF32's 10 mantissa bits; hi hi + hi lo + lo hi, as in
// CUTLASS's 3xTF32 and Ootomo and Yokota, "Recovering single precision
// accuracy from Tensor Cores while surpassing the FP32 theoretical peak
// performance", 2022): the dropped lo lo term and the truncation of lo are
// below 2^-20 of each term.
//
// Per call (before the first chunk of a host call), prologue kernels form the
// coefficient fragments of every (Jones plane, antenna-type pair, component),
// split, and the spectral amplitudes of every (run, component, channel), both
// in the order the lanes read them.  Per component tile (ct components, the fragments of the run's
// plane for every type pair and the run's amplitudes, staged by bulk copies on
// one mbarrier):
//   (record, component)        phase turns P (split-FP32) and the step of one
//                              matrix tile s16 = exp(2 pi i P 16 df) (accurate
//                              sin/cos);
//   (record, component, lane)  anchors at channels g and g + 8 (MUFU sin/cos of
//                              the range-reduced split-FP32 phase), then per
//                              matrix tile of the run the amplitude, the split,
//                              three products and one packed complex step.
// Gaussian families carry their taper exp(Q f^2) (Q per record and component)
// on the lane's chain as well: over one matrix tile the taper changes by
// R = exp(Q (32 f df + 256 df^2)), and R itself by exp(512 Q df^2), so two
// packed multiplies per tile advance it.
// Tile partial sums are folded into compensated (Kahan) totals.
#include <stdint.h>

#include <algorithm>

#include "beam_common.cuh"
#include "dft_beam.h"
#include "dft_kernels.cuh"
#include "dft_plan.h"

namespace obit {

namespace {

constexpr int kMmaThreads = kBeamMmaWarps * 32;
// Matrix tiles per branch-free group of the run (their three dependent
// products per tile interleave); runs are padded to a multiple of it.
constexpr int kMmaChunk = 4;
// float2 entries of one component group of the amplitude table: one
// (g, g + 8) channel pair per matrix tile, lane group and component
constexpr int kAmpGroup = kBeamMmaTiles * 32;
// float2 entries per component of the (record, component) tables: padded so
// that a warp's four components fall in different banks
constexpr int kPStride = kBeamMmaWarps + 1;
constexpr int kCmpSlots = kBeamMmaTiles * 2;  // packed compensation terms per thread

// Shared-memory layout of one CTA (offsets in floats, each a multiple of 4).
struct MmaLayout {
  int comp, coef, pp, ss, qq, amp, cmp, uvw, pair, total;
};

__host__ __device__ inline int pad4(int n) { return (n + 3) & ~3; }

__host__ __device__ inline MmaLayout mma_layout(int ct, int cstride, int npair, bool table, bool gauss) {
  MmaLayout L;
  int o = 0;
  L.comp = o;
  o += ct * cstride;
  L.coef = o;
  o += npair * ct * 32;  // float4 per (type pair, component, column)
  L.pp = o;
  o += pad4(ct * kPStride * 2);
  L.ss = o;
  o += pad4(ct * kPStride * 2);
  L.qq = o;
  o += gauss ? pad4(ct * kPStride) : 0;
  L.amp = o;
  o += table ? (ct / 4) * kAmpGroup * 2 : 0;
  L.cmp = o;
  o += kMmaThreads * kCmpSlots * 2;
  L.uvw = o;
  o += 4 * kBeamMmaWarps;
  L.pair = o;
  o += kBeamMmaWarps;
  L.total = o;
  return L;
}

// Model families: spectral amplitudes from the prologue's table; Gaussian taper.
__host__ __device__ constexpr bool mma_amp(int mode) {
  return mode == kPointSpec || mode == kPointTSpec || mode == kGaussSpec || mode == kGaussTSpec;
}
__host__ __device__ constexpr bool mma_gauss(int mode) {
  return mode == kGauss || mode == kGaussSpec || mode == kGaussTSpec;
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// High part of the split: the leading 10 mantissa bits (exact truncation).
__device__ __forceinline__ float tf32_hi(float x) {
  return __uint_as_float(__float_as_uint(x) & 0xffffe000u);
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], float a0, float a1, float a2, float a3,
                                         uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(__float_as_uint(a0)), "r"(__float_as_uint(a1)), "r"(__float_as_uint(a2)),
        "r"(__float_as_uint(a3)), "r"(b0), "r"(b1));
}

__device__ __forceinline__ ds ds_add(ds a, ds b) {
  const ds s = two_sum(a.hi, b.hi);
  return fast_two_sum(s.hi, __fadd_rn(s.lo, __fadd_rn(a.lo, b.lo)));
}

// Prologue: the coefficient fragments of every (Jones plane, antenna-type
// pair, component), split into TF32 hi and lo parts, in the order the main
// kernel's lanes read them.  Lane (g, t) of a warp holds column n = g = 2q + ri
// for component 4j + t: b0 = B[re of c][n], b1 = B[im of c][n], i.e. (Cr, -Ci)
// for ri = 0 and (Ci, Cr) for ri = 1.
__global__ void __launch_bounds__(256) beam_coef_kernel(const __grid_constant__ BeamKParams bp) {
  const int npair = bp.numAntType * bp.numAntType;
  const long long n = (long long)bp.numJChan * npair * bp.ncompPad;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % bp.ncompPad);
    const long long r = i / bp.ncompPad;
    const int pr = (int)(r % npair);
    const int jp = (int)(r / npair);
    float4* d = bp.coefTab + ((size_t)(jp * npair + pr) * bp.ncompPad + (c & ~3)) * 8 + (c & 3);
    if (c >= bp.k.ncomp) {
#pragma unroll
      for (int gg = 0; gg < 8; gg++) d[gg * 4] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    const int ta = pr / bp.numAntType, tc = pr - ta * bp.numAntType;
    const float* J1 = bp.jones + (((size_t)ta * bp.jonesComps + c) * bp.numJChan + jp) * 8;
    const float* J2 = bp.jones + (((size_t)tc * bp.jonesComps + c) * bp.numJChan + jp) * 8;
    const float4 a0 = __ldg(reinterpret_cast<const float4*>(J1));
    const float4 a1 = __ldg(reinterpret_cast<const float4*>(J1 + 4));
    const float4 b0 = __ldg(reinterpret_cast<const float4*>(J2));
    const float4 b1 = __ldg(reinterpret_cast<const float4*>(J2 + 4));
    const float J1r[4] = {a0.x, a0.z, a1.x, a1.z}, J1i[4] = {a0.y, a0.w, a1.y, a1.w};
    const float J2r[4] = {b0.x, b0.z, b1.x, b1.z}, J2i[4] = {b0.y, b0.w, b1.y, b1.w};
    float cr[4], ci[4];
    beam_coeffs(bp, J1r, J1i, J2r, J2i, cr, ci);
#pragma unroll
    for (int gg = 0; gg < 8; gg++) {
      const int q = gg >> 1;
      const float v0 = (gg & 1) ? ci[q] : cr[q];
      const float v1 = (gg & 1) ? cr[q] : -ci[q];
      const uint32_t h0 = tf32_rna(v0), h1 = tf32_rna(v1);
      const uint32_t l0 = tf32_rna(v0 - __uint_as_float(h0)), l1 = tf32_rna(v1 - __uint_as_float(h1));
      d[gg * 4] = make_float4(__uint_as_float(h0), __uint_as_float(h1), __uint_as_float(l0), __uint_as_float(l1));
    }
  }
}

// Prologue of the families with a spectrum: the amplitude A exp(sum_t a_t
// L^(t+1)) (PointSpec, GaussSpec; L the log-frequency term of the channel) or
// A_plane exp(alpha L) (PointTSpec, GaussTSpec) of every (run, component, channel), as the
// per-channel form computes it, in the lanes' order (BeamKParams.ampTab).
template <int MODE>
__global__ void __launch_bounds__(256) beam_amp_kernel(const __grid_constant__ BeamKParams bp) {
  using F = Fields<MODE>;
  const KParams& p = bp.k;
  const long long n = (long long)bp.nseg * (bp.ncompPad / 4) * kAmpGroup;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i & 3);
    const int g = (int)((i >> 2) & 7);
    const int m = (int)((i >> 5) & (kBeamMmaTiles - 1));
    const long long r = i / kAmpGroup;
    const int cg = (int)(r % (bp.ncompPad / 4));
    const int sg = (int)(r / (bp.ncompPad / 4));
    const int c = 4 * cg + t;
    const BeamSeg seg = bp.segs[sg];
    float a[2] = {0.f, 0.f};
    if (c < p.ncomp) {
      const float* cp = p.comps + (size_t)c * p.cstride;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int k = m * kBeamMmaRows + g + 8 * h;
        if (k < seg.nch) {
          const int ifq = seg.ifq0 + k * bp.kincf;
          const double L = bp.lnspec ? bp.lnspec[ifq] : 0.0;
          double e = 0.0;
          float A;
          if constexpr (F::kTSpec) {
            A = cp[F::kTabOff + (bp.plane ? bp.plane[ifq] : 0)];
            e = (double)cp[F::kAlphaOff] * L;
          } else {
            A = cp[0];
            double pw = L;
            for (int tt = 0; tt < p.nterm && tt < kMaxNTerm; tt++) {
              e += (double)cp[F::kSpecOff + tt] * pw;
              pw *= L;
            }
          }
          a[h] = A * expf((float)e);
        }
      }
    }
    bp.ampTab[i] = make_float2(a[0], a[1]);
  }
}

// Stage component tile c0 and its coefficient fragments at plane jp (one
// slice per type pair) by bulk copies on one mbarrier, with the bounded waits
// of stage_comps.  Bulk copies need 16-byte aligned addresses and sizes:
// cstride is a multiple of 4 floats, a slice ct * 128 bytes, the tables
// cudaMalloc'd.
template <bool kAmp>
__device__ __forceinline__ bool stage_tile(const BeamKParams& bp, float* sComp, float4* sCoef, float2* sAmp,
                                           int c0, int sg, int jp, int npair, uint64_t* bar, uint32_t& phase) {
  const KParams& p = bp.k;
  const int ct = p.ct;
  const int nc = min(ct, p.ncomp - c0);
  const uint32_t cbytes = (uint32_t)nc * p.cstride * 4u;
  const uint32_t fbytes = (uint32_t)ct * 128u;
  const uint32_t abytes = kAmp ? (uint32_t)(ct / 4) * kAmpGroup * 8u : 0u;
  const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_s),
                 "r"(cbytes + (uint32_t)npair * fbytes + abytes)
                 : "memory");
    if (kAmp) {
      const float2* src = bp.ampTab + ((size_t)sg * (bp.ncompPad / 4) + c0 / 4) * kAmpGroup;
      asm volatile(
          "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              (uint32_t)__cvta_generic_to_shared(sAmp)),
          "l"(src), "r"(abytes), "r"(bar_s)
          : "memory");
    }
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            (uint32_t)__cvta_generic_to_shared(sComp)),
        "l"(p.comps + (size_t)c0 * p.cstride), "r"(cbytes), "r"(bar_s)
        : "memory");
    for (int pr = 0; pr < npair; pr++) {
      const float4* src = bp.coefTab + ((size_t)(jp * npair + pr) * bp.ncompPad + c0) * 8;
      asm volatile(
          "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              (uint32_t)__cvta_generic_to_shared(sCoef + (size_t)pr * ct * 8)),
          "l"(src), "r"(fbytes), "r"(bar_s)
          : "memory");
    }
  }
  for (int i = nc * p.cstride + threadIdx.x; i < ct * p.cstride; i += blockDim.x) sComp[i] = 0.0f;
  uint32_t done = 0;
  for (int it = 0; it < kDefaultWaitPolls && !done; it++) {
    asm volatile(
        "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
        : "=r"(done)
        : "r"(bar_s), "r"(phase)
        : "memory");
  }
  phase ^= 1u;
  const bool failed = __syncthreads_or(done == 0) != 0;
  if (failed) {
    if (threadIdx.x == 0 && p.errFlag) atomicMax(p.errFlag, 2);
    // a second bounded window for copies in flight, as stage_comps
    for (int it = 0; it < (1 << 22) && !done; it++) {
      asm volatile(
          "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
          : "=r"(done)
          : "r"(bar_s), "r"(phase ^ 1u)
          : "memory");
    }
    if (__syncthreads_or(done == 0) && threadIdx.x == 0 && p.errFlag) atomicMax(p.errFlag, 5);
  }
  return !failed;
}

template <int MODE>
__global__ void __launch_bounds__(kMmaThreads, 1) dft_beam_mma_kernel(const __grid_constant__ BeamKParams bp) {
  using F = Fields<MODE>;
  constexpr bool kAmp = mma_amp(MODE), kGau = mma_gauss(MODE);
  static_assert(kBeamMmaWarps == 8, "the (record, component) tables index records by 3 bits");
  const KParams& p = bp.k;
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  const int ct = p.ct;
  const int npair = bp.numAntType * bp.numAntType;
  const MmaLayout lay = mma_layout(ct, p.cstride, npair, kAmp, kGau);
  float* sComp = smem + lay.comp;
  float4* sCoef = reinterpret_cast<float4*>(smem + lay.coef);
  float2* sP = reinterpret_cast<float2*>(smem + lay.pp);
  float2* sS = reinterpret_cast<float2*>(smem + lay.ss);
  float* sQ = smem + lay.qq;
  float2* sAmp = reinterpret_cast<float2*>(smem + lay.amp);
  f2x* sCmp = reinterpret_cast<f2x*>(smem + lay.cmp);
  float* sUVW = smem + lay.uvw;
  int* sPair = reinterpret_cast<int*>(smem + lay.pair);
  init_bar(&bar);
  uint32_t phase = 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // the lane's model correlation t (XX, XY, YX, YY) in the record's order XX, YY, XY, YX
  const int slot = (t == 0) ? 0 : (t == 1) ? 2 : (t == 2) ? 3 : 1;
  const int nItems = ((p.nvis + kBeamMmaWarps - 1) / kBeamMmaWarps) * bp.nseg;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int rt = item / bp.nseg;
    const int sg = item - rt * bp.nseg;
    const BeamSeg seg = bp.segs[sg];
    const int row0 = rt * kBeamMmaWarps;
    const int nb = (seg.nch + kBeamMmaRows - 1) / kBeamMmaRows;
    __syncthreads();  // the previous item is done with shared memory
#pragma unroll
    for (int j = 0; j < kCmpSlots; j++) sCmp[j * kMmaThreads + threadIdx.x] = 0ull;
    load_uvw(p, sUVW, row0);
    if (threadIdx.x < kBeamMmaWarps) {  // antenna-type pair of each record (-1: none)
      const int row = row0 + threadIdx.x;
      int pr = -1;
      if (row < p.nvis) {
        const float* rec = p.vis + (size_t)(p.rowBase + row) * p.lrec;
        int a1, a2;
        beam_ants(bp, rec, a1, a2);
        if (a1 < 0 || a1 >= bp.numAnt || a2 < 0 || a2 >= bp.numAnt) {
          if (p.errFlag) atomicExch(p.errFlag, 3);
        } else {
          pr = bp.antType[a1] * bp.numAntType + bp.antType[a2];
        }
      }
      sPair[threadIdx.x] = pr;
    }
    __syncthreads();
    const int row = row0 + warp;
    const int pr = sPair[warp];
    const bool mine = (row < p.nvis) && (pr >= 0);
    // frequency ratios of the lane's channels g and g + 8 of the first matrix tile
    const ds dfd = {p.df_hi[seg.dfc], p.df_lo[seg.dfc]};
    const ds f0 = {seg.f0_hi, seg.f0_lo};
    const ds fa = ds_add(f0, ds_mul(ds{(float)g, 0.f}, dfd));
    const ds fb = ds_add(f0, ds_mul(ds{(float)(g + 8), 0.f}, dfd));
    const ds d16 = {16.f * dfd.hi, 16.f * dfd.lo};
    f2x tot[kBeamMmaTiles][2];
#pragma unroll
    for (int m = 0; m < kBeamMmaTiles; m++) tot[m][0] = tot[m][1] = 0ull;

    for (int c0 = 0; c0 < p.ncomp; c0 += ct) {
      __syncthreads();  // the previous tile's readers are done with shared memory
      if (!stage_tile<kAmp>(bp, sComp, sCoef, sAmp, c0, sg, seg.jplane, npair, &bar, phase)) return;
      const int nc = min(ct, p.ncomp - c0);
      // (record, component): phase turns and the step of one matrix tile
      for (int idx = threadIdx.x; idx < kBeamMmaWarps * ct; idx += kMmaThreads) {
        const int c = idx >> 3;  // kBeamMmaWarps == 8 records
        const int r = idx & 7;
        const float* cp = sComp + c * p.cstride;
        const float u = sUVW[3 * r], v = sUVW[3 * r + 1], w = sUVW[3 * r + 2];
        const ds P = beam_phase_turns(p, cp, c0 + c, u, v, w);
        sP[c * kPStride + r] = make_float2(P.hi, P.lo);
        const ds ts = ds_mul(P, d16);
        sS[c * kPStride + r] = phasor_accurate(ds{__fsub_rn(ts.hi, rintf(ts.hi)), ts.lo});
        if constexpr (kGau) sQ[c * kPStride + r] = cp[4] * u * u + cp[5] * v * v + cp[6] * u * v;
      }
      __syncthreads();

      if (mine) {
        float acc[kBeamMmaTiles][4];
#pragma unroll
        for (int m = 0; m < kBeamMmaTiles; m++) acc[m][0] = acc[m][1] = acc[m][2] = acc[m][3] = 0.f;
        const int ngrp = (nc + 3) >> 2;
        const float4* cf = sCoef + (size_t)pr * ct * 8 + lane;
        for (int j = 0; j < ngrp; j++) {
          const int c = 4 * j + t;
          const float2 Pp = sP[c * kPStride + warp];
          const float2 st = sS[c * kPStride + warp];
          const float4 bf = cf[j * 32];
          const uint32_t bh0 = __float_as_uint(bf.x), bh1 = __float_as_uint(bf.y);
          const uint32_t bl0 = __float_as_uint(bf.z), bl1 = __float_as_uint(bf.w);
          float2 za = phasor_fast(ds_mul_frac(ds{Pp.x, Pp.y}, fa));
          float2 zb = phasor_fast(ds_mul_frac(ds{Pp.x, Pp.y}, fb));
          if constexpr (!kAmp && !kGau) {  // constant amplitude: carried by the chain
            const float A = sComp[c * p.cstride];
            za.x *= A;
            za.y *= A;
            zb.x *= A;
            zb.y *= A;
          }
          // Gaussian taper at the lane's channels (times a constant amplitude),
          // its ratio over one matrix tile and that ratio's own constant ratio
          f2x TP = 0ull, RP = 0ull, CP = 0ull;
          if constexpr (kGau) {
            const float Q = sQ[c * kPStride + warp];
            const float D = d16.hi;
            float ta = exp_fast(Q * fa.hi * fa.hi), tb = exp_fast(Q * fb.hi * fb.hi);
            if constexpr (!kAmp) {
              const float A = sComp[c * p.cstride];
              ta *= A;
              tb *= A;
            }
            TP = pk2(ta, tb);
            RP = pk2(exp_fast(Q * D * (2.f * fa.hi + D)), exp_fast(Q * D * (2.f * fb.hi + D)));
            const float c2 = exp_fast(2.f * Q * D * D);
            CP = pk2(c2, c2);
          }
          f2x ZR = pk2(za.x, zb.x), ZI = pk2(za.y, zb.y);
          const f2x SR = pk2(st.x, st.x), SI = pk2(st.y, st.y), NSI = pk2(-st.y, -st.y);
          const float2* ap = sAmp + (size_t)j * kAmpGroup + lane;
#pragma unroll
          for (int mc = 0; mc < kBeamMmaTiles; mc += kMmaChunk) {
            if (mc < nb) {
#pragma unroll
              for (int i = 0; i < kMmaChunk; i++) {
                const int m = mc + i;
                f2x VR = ZR, VI = ZI;
                if constexpr (kAmp || kGau) {
                  f2x AP = TP;
                  if constexpr (kAmp) {
                    const float2 a = ap[m * 32];
                    AP = pk2(a.x, a.y);
                    if constexpr (kGau) AP = mul2(AP, TP);
                  }
                  VR = mul2(ZR, AP);
                  VI = mul2(ZI, AP);
                }
                float vr0, vr1, vi0, vi1;
                up2(VR, vr0, vr1);
                up2(VI, vi0, vi1);
                const float h0 = tf32_hi(vr0), h1 = tf32_hi(vr1), h2 = tf32_hi(vi0), h3 = tf32_hi(vi1);
                float l0, l1, l2, l3;
                up2(sub2(VR, pk2(h0, h1)), l0, l1);
                up2(sub2(VI, pk2(h2, h3)), l2, l3);
                // A fragment: a0 (row g, k = t) real part at channel g, a1 row
                // g + 8, a2 / a3 the imaginary parts (k = t + 4)
                mma_tf32(acc[m], l0, l1, l2, l3, bh0, bh1);
                mma_tf32(acc[m], h0, h1, h2, h3, bl0, bl1);
                mma_tf32(acc[m], h0, h1, h2, h3, bh0, bh1);
                // to the same lanes' channels of the next matrix tile
                const f2x nr = fma2(ZR, SR, mul2(ZI, NSI));
                ZI = fma2(ZR, SI, mul2(ZI, SR));
                ZR = nr;
                if constexpr (kGau) {
                  TP = mul2(TP, RP);
                  RP = mul2(RP, CP);
                }
              }
            }
          }
        }
        // compensated fold of the tile's sums: C fragment (c0, c1) is model
        // correlation t (re, im) at channel g, (c2, c3) at channel g + 8
        f2x* cmp = sCmp + threadIdx.x;
#pragma unroll
        for (int m = 0; m < kBeamMmaTiles; m++) {
          if (m < nb) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int e = (2 * m + h) * kMmaThreads;
              const f2x a = pk2(acc[m][2 * h], acc[m][2 * h + 1]);
              const f2x cc = cmp[e];
              const f2x y = sub2(a, cc);
              const f2x s = add2(tot[m][h], y);
              cmp[e] = sub2(sub2(s, tot[m][h]), y);
              tot[m][h] = s;
            }
          }
        }
      }
    }

    // apply the model to the record: lane (g, t) writes correlation slot
    // `slot` at channels 16 m + g and 16 m + g + 8
    if (mine && slot < bp.ncorr) {
      float* base = p.vis + (size_t)(p.rowBase + row) * p.lrec + seg.off0 + slot * p.incs;
      const float pf = bp.polFact[slot];
#pragma unroll
      for (int m = 0; m < kBeamMmaTiles; m++) {
        if (m < nb) {
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int k = m * kBeamMmaRows + g + 8 * h;
            if (k < seg.nch) {
              float Mr, Mi;
              up2(tot[m][h], Mr, Mi);
              Mr *= pf;
              Mi *= pf;
              float* o = base + (size_t)k * p.incf;
              if (o[2] <= 0.0f && p.op != kOpRepl) continue;
              if (p.op == kOpRepl) {
                o[0] = Mr;
                o[1] = Mi;
              } else if (p.op == kOpDiv) {
                const float a2 = Mr * Mr + Mi * Mi;
                const float Vr = o[0], Vi = o[1];
                o[0] = (Vr * Mr + Vi * Mi) / a2;
                o[1] = (Vi * Mr - Vr * Mi) / a2;
              } else {
                o[0] -= Mr;
                o[1] -= Mi;
              }
            }
          }
        }
      }
    }
  }
  inval_bar(&bar);
}

}  // namespace

bool beam_mma_supported(int mode) { return mode >= kPoint && mode <= kGaussTSpec; }

size_t beam_mma_coef_bytes(const BeamKParams& p) {
  return (size_t)p.numJChan * p.numAntType * p.numAntType * (size_t)p.ncompPad * 8 * sizeof(float4);
}

size_t beam_mma_amp_bytes(const BeamKParams& p) {
  if (!mma_amp(p.mode)) return 0;
  return (size_t)p.nseg * (size_t)(p.ncompPad / 4) * kAmpGroup * sizeof(float2);
}

size_t beam_mma_smem_bytes(const BeamKParams& p) {
  const int npair = p.numAntType * p.numAntType;
  return sizeof(float) * (size_t)mma_layout(p.k.ct, p.k.cstride, npair, mma_amp(p.mode), mma_gauss(p.mode)).total;
}

int beam_mma_fit_tile(BeamKParams* p) {
  for (int ct = 128; ct >= 8; ct -= 4) {
    p->k.ct = ct;
    if (beam_mma_smem_bytes(*p) <= 220 * 1024) return ct;
  }
  p->k.ct = 0;
  return 0;
}

int launch_beam_prologue(const BeamKParams& kp, cudaStream_t stream, std::string* err) {
  const KParams& k = kp.k;
  if (k.ncomp <= 0 || kp.nseg <= 0) return 0;
  const bool table = mma_amp(kp.mode);
  if (!kp.coefTab || kp.ncompPad < k.ncomp || (table && !kp.ampTab)) {
    *err = "tensor-core beam prologue without its tables";
    return 3;
  }
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t ce;
  if (table) {  // prologue: spectral amplitudes of every (run, component, channel)
    const long long n = (long long)kp.nseg * (kp.ncompPad / 4) * kAmpGroup;
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)nsm * 8);
    switch (kp.mode) {
      case kPointSpec:
        beam_amp_kernel<kPointSpec><<<(unsigned)blocks, 256, 0, stream>>>(kp);
        break;
      case kPointTSpec:
        beam_amp_kernel<kPointTSpec><<<(unsigned)blocks, 256, 0, stream>>>(kp);
        break;
      case kGaussSpec:
        beam_amp_kernel<kGaussSpec><<<(unsigned)blocks, 256, 0, stream>>>(kp);
        break;
      default:
        beam_amp_kernel<kGaussTSpec><<<(unsigned)blocks, 256, 0, stream>>>(kp);
        break;
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
      *err = std::string("beam amplitude kernel launch: ") + cudaGetErrorString(ce);
      return 2;
    }
  }
  {  // prologue: coefficient fragments of every (plane, type pair, component)
    const long long n = (long long)kp.numJChan * kp.numAntType * kp.numAntType * kp.ncompPad;
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)nsm * 8);
    beam_coef_kernel<<<(unsigned)blocks, 256, 0, stream>>>(kp);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
      *err = std::string("beam coefficient kernel launch: ") + cudaGetErrorString(ce);
      return 2;
    }
  }
  return 0;
}

int launch_beam_mma(const BeamKParams& kp, cudaStream_t stream, std::string* err, bool prologue) {
  const KParams& k = kp.k;
  if (k.nvis <= 0 || k.ncomp <= 0 || kp.nseg <= 0) return 0;
  if (k.ct < 4 || (k.ct & 3) || k.R != kBeamMmaWarps) {
    *err = "tensor-core beam launch with an invalid tile";
    return 3;
  }
  using Fn = void (*)(const BeamKParams);
  Fn fn = nullptr;
  switch (kp.mode) {
    case kPoint:
      fn = dft_beam_mma_kernel<kPoint>;
      break;
    case kPointSpec:
      fn = dft_beam_mma_kernel<kPointSpec>;
      break;
    case kPointTSpec:
      fn = dft_beam_mma_kernel<kPointTSpec>;
      break;
    case kGauss:
      fn = dft_beam_mma_kernel<kGauss>;
      break;
    case kGaussSpec:
      fn = dft_beam_mma_kernel<kGaussSpec>;
      break;
    case kGaussTSpec:
      fn = dft_beam_mma_kernel<kGaussTSpec>;
      break;
    default:
      break;
  }
  if (!fn) {
    *err = "no tensor-core beam kernel for this model type";
    return 3;
  }
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("error pending before the beam kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  const size_t smem = beam_mma_smem_bytes(kp);
  if (int rc = raise_smem_limit((const void*)fn, smem, err)) return rc;
  int perSM = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, kMmaThreads, smem);
  if (ce != cudaSuccess || perSM < 1) {
    *err = std::string("tensor-core beam kernel cannot be resident: ") + cudaGetErrorString(ce);
    return 2;
  }
  const bool table = mma_amp(kp.mode);
  if (!kp.coefTab || kp.ncompPad < k.ncomp || kp.ncompPad % k.ct || (table && !kp.ampTab)) {
    *err = "tensor-core beam launch without its tables";
    return 3;
  }
  if (prologue)
    if (int rc = launch_beam_prologue(kp, stream, err)) return rc;
  const long long nItems = (long long)((k.nvis + kBeamMmaWarps - 1) / kBeamMmaWarps) * kp.nseg;
  const long long grid = std::min<long long>(nItems, (long long)perSM * nsm);
  fn<<<(unsigned)grid, kMmaThreads, smem, stream>>>(kp);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("tensor-core beam kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
