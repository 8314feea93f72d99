// DFT sky-model predict / subtract kernels for sm_100a.
//
// Work decomposition.  A visibility record (ObitUVDesc layout: nrparm random
// parameters then {re, im, weight} per correlation) is one "row".  The selected
// (channel, IF) pairs of a row are cut on the host into channel blocks of at
// most K channels that share one IF, one channel increment and (for tabulated
// spectra) one coarse plane.  A CTA tile is R rows x Bt blocks; each thread owns
// one (row, block) pair and keeps its K complex model sums in registers.
//
// Per component and tile the work splits in three levels:
//   (row, component)          prepass: phase argument P = (X u + Y v + Z w)/2pi in
//                             split-FP32, one accurate step phasor exp(2 pi i P df)
//                             per channel-increment class, and the Gaussian form
//                             g1 u^2 + g2 v^2 + g3 u v; stored in shared memory and
//                             shared by every block of the row.
//   (row, component, block)   anchor phasor exp(2 pi i P f0) from the range-reduced
//                             split-FP32 product, amplitude exponent fitted as
//                             e0 + e1 k + e2 k^2 over the block.
//   (row, component, channel) complex recurrence z <- z * w (w <- w * q for
//                             channel-dependent amplitudes) and z accumulated.
// Component partial sums are plain FP32 within a tile and folded into a
// compensated (Kahan) total at each tile boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ds_math.cuh"

namespace obit {

constexpr int kThreads = 256;
constexpr int kMaxNTerm = 4;   // spectral terms supported (ObitSkyModel nSpecTerm)
constexpr int kMaxDf = 8;      // distinct channel increments per launch
constexpr int kMaxPol = 4;

// Model families; numbering matches GPUModType (ObitCUDASkyModelInfoDef.h:44-52).
enum ModelKind : int {
  kPoint = 0,
  kPointSpec = 1,
  kPointTSpec = 2,
  kGauss = 3,
  kGaussSpec = 4,
  kGaussTSpec = 5
};
enum OpKind : int { kOpSub = 0, kOpDiv = 1, kOpRepl = 2 };
enum KernelFlavor : int { kFlavorRecur = 0, kFlavorPlain = 1 };

// One channel block: up to K consecutive channels of one IF.
struct BlockDesc {
  float f0_hi, f0_lo;  // frequency ratio nu/nu_uvref of the first channel (split-FP32)
  float df;            // channel increment of the ratio (float copy, Gaussian exponent)
  int off0;            // float offset of the first channel's pol-0 triplet in the record
  int len;             // valid channels, 1..K
  int dfc;             // channel-increment class (index into KParams.df_*)
  int plane;           // coarse spectral plane (tabulated spectra)
  int ifq0;            // frequency-table index of the first channel
  // Quadratic fits over the block, L^(t+1)(k) ~ l[t][0] + l[t][1] k + l[t][2] k^2,
  // of the log frequency ratio used by the spectral term (k = 0..len-1).
  float l[kMaxNTerm][3];
};

struct KParams {
  float* vis;  // device records, nvis x lrec floats
  int nvis, lrec, ilocu, ilocv, ilocw;
  int incs, incf;  // float increments between polarizations and channels
  int pol0, npol;  // selected polarizations
  int op;          // OpKind
  int flipMask;    // bit j: multiply the j-th selected polarization's model by i
  int cumulative;  // 1: CPU rule, stokFactor advances only on written polarizations
  float stokFactor;
  float polFact[kMaxPol];
  const BlockDesc* blocks;
  int nblocks;      // blocks per row
  int Bt, R;        // tile shape: blocks per tile, rows per tile (Bt * R <= kThreads)
  int nBlockTiles;  // ceil(nblocks / Bt)
  int ndf;
  float df_hi[kMaxDf], df_lo[kMaxDf];
  const float* comps;  // ncomp records of cstride floats (reference field order)
  int ncomp, cstride, ct, nterm;
  int nspec;           // planes (tabulated spectra)
  int rowBase;         // first row index of this launch within vis
  int* errFlag;        // set non-zero on an internal error (never traps)
};

// Reference field offsets inside a component record (ObitSkyModel.c:1965-2063,
// ObitSkyModelMF.c:1497-1514).
template <int MODE>
struct Fields {
  static constexpr bool kGaussian = (MODE == kGauss || MODE == kGaussSpec || MODE == kGaussTSpec);
  static constexpr bool kSpec = (MODE == kPointSpec || MODE == kGaussSpec);
  static constexpr bool kTSpec = (MODE == kPointTSpec || MODE == kGaussTSpec);
  static constexpr bool kQuad = (MODE != kPoint);
  static constexpr int kSpecOff = (MODE == kPointSpec) ? 4 : 7;   // first spectral coefficient
  static constexpr int kAlphaOff = (MODE == kPointTSpec) ? 4 : 7; // TSpec spectral index
  static constexpr int kTabOff = (MODE == kPointTSpec) ? 5 : 8;   // TSpec first plane flux
};

__device__ __forceinline__ float exp_fast(float x) {
  // exp(x) = 2^(x log2 e); one MUFU.EX2 after the scaling multiply
  return exp2f(x * 1.4426950408889634f);
}

// Complex multiply-accumulate helpers.
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -a.y * b.y), __fmaf_rn(a.x, b.y, a.y * b.x));
}

// Accurate unit phasor exp(2 pi i r) for |r| <= ~0.5 turns with residual rlo
// (first-order correction of the float rounding of r).
__device__ __forceinline__ float2 phasor_accurate(ds r) {
  float s, c;
  sincospif(2.0f * r.hi, &s, &c);
  const float d = 6.283185307179586f * r.lo;
  return make_float2(__fmaf_rn(-d, s, c), __fmaf_rn(d, c, s));
}

// Anchor phasor: MUFU sin/cos of the reduced angle (error does not compound).
__device__ __forceinline__ float2 phasor_fast(float r) {
  float s, c;
  __sincosf(6.283185307179586f * r, &s, &c);
  return make_float2(c, s);
}

//--------------------------------------------------------------------------
// Shared memory layout per CTA (dynamic), sized by the host:
//   comps  : ct * cstride floats (component tile, zero-filled past ncomp)
//   uvw    : R * 3 floats
//   P      : ct * R float2       (phase turns, split-FP32)
//   S      : ndf * ct * R float2 (step phasors)
//   Q      : ct * R floats       (Gaussian form, Gaussian models only)
// The model stage of the epilogue (R * Bt * K float2) reuses the same space.
//--------------------------------------------------------------------------
__host__ __device__ inline size_t smem_floats_main(int R, int ct, int cstride, int ndf, bool gauss) {
  size_t n = (size_t)ct * cstride + (size_t)R * 3 + 2 * (size_t)ct * R + 2 * (size_t)ndf * ct * R;
  if (gauss) n += (size_t)ct * R;
  return n;
}
__host__ __device__ inline size_t smem_floats_stage(int R, int Bt, int K) {
  return (size_t)R * Bt * K * 2;
}

// Apply the staged model of one tile to its records (subtract / divide /
// replace), with the CPU reference's polarization rules.
template <int K>
__device__ __forceinline__ void apply_tile(const KParams& p, const float2* stage, int row0,
                                           int blk0, int nblkTile) {
  const int per_row = p.Bt * K;
  for (int idx = threadIdx.x; idx < p.R * per_row; idx += blockDim.x) {
    const int tr = idx / per_row;
    const int j = idx - tr * per_row;
    const int tb = j / K;
    const int k = j - tb * K;
    const int row = row0 + tr;
    if (row >= p.nvis || tb >= nblkTile) continue;
    const BlockDesc& bd = p.blocks[blk0 + tb];
    if (k >= bd.len) continue;
    const float2 S = stage[idx];
    float* rec = p.vis + (size_t)(p.rowBase + row) * p.lrec + bd.off0 + k * p.incf;
    // any selected polarization with positive weight?
    bool any = (p.op == kOpRepl);
    for (int jp = 0; jp < p.npol; jp++) any = any || (rec[(p.pol0 + jp) * p.incs + 2] > 0.0f);
    if (!any) continue;
    float cum = 1.0f;
    for (int jp = 0; jp < p.npol; jp++) {
      float* v = rec + (p.pol0 + jp) * p.incs;
      const float wt = v[2];
      if (wt <= 0.0f && p.op != kOpRepl) continue;
      const float fac = p.polFact[jp] * cum;
      float mr = S.x * fac, mi = S.y * fac;
      if (p.flipMask & (1 << jp)) { const float t = mr; mr = -mi; mi = t; }
      if (p.op == kOpDiv) {
        const float a2 = mr * mr + mi * mi;
        const float dr = mr / a2, di = mi / a2;
        const float vr = v[0], vi = v[1];
        v[0] = dr * vr + di * vi;
        v[1] = dr * vi - di * vr;
        v[2] = wt * sqrtf(a2);
      } else if (p.op == kOpRepl) {
        v[0] = mr;
        v[1] = mi;
      } else {
        v[0] -= mr;
        v[1] -= mi;
      }
      if (p.cumulative) cum *= p.stokFactor;
    }
  }
}

// Stage one component tile into shared memory with a 1-D bulk copy (TMA engine,
// no multicast) completed on an mbarrier; the tail past ncomp is zero-filled.
// Every thread waits on the barrier with a bounded number of polls; the return
// value is uniform across the CTA (false: the copy did not land, the error
// flag is set and the caller must leave the kernel).
__device__ __forceinline__ bool stage_comps(const KParams& p, float* sComp, int c0, uint64_t* bar,
                                            uint32_t& phase) {
  const int nc = min(p.ct, p.ncomp - c0);
  const uint32_t bytes = (uint32_t)nc * p.cstride * 4u;
  const float* src = p.comps + (size_t)c0 * p.cstride;
  const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
  // Bulk copies need 16-byte aligned addresses and sizes; cstride is a multiple
  // of 4 floats and the table base is 256-byte aligned, so this always holds.
  if (threadIdx.x == 0) {
    const uint32_t dst_s = (uint32_t)__cvta_generic_to_shared(sComp);
    // order earlier generic-proxy accesses of this shared memory before the
    // async-proxy write of the copy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_s), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_s),
        "l"(src), "r"(bytes), "r"(bar_s)
        : "memory");
  }
  // zero-fill the tail of the tile
  for (int i = nc * p.cstride + threadIdx.x; i < p.ct * p.cstride; i += blockDim.x) sComp[i] = 0.0f;
  uint32_t done = 0;
  for (int it = 0; it < (1 << 22) && !done; it++) {
    asm volatile(
        "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
        : "=r"(done)
        : "r"(bar_s), "r"(phase)
        : "memory");
  }
  phase ^= 1u;
  const bool failed = __syncthreads_or(done == 0) != 0;
  if (failed) {
    if (threadIdx.x == 0 && p.errFlag) atomicExch(p.errFlag, 2);
    // give an in-flight copy a second bounded window to land before exiting
    for (int it = 0; it < (1 << 22) && !done; it++) {
      asm volatile(
          "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
          : "=r"(done)
          : "r"(bar_s), "r"(phase ^ 1u)
          : "memory");
    }
  }
  return !failed;
}

//--------------------------------------------------------------------------
// Recurrence kernel.  K channels per thread, MODE model family.
//--------------------------------------------------------------------------
template <int K, int MODE>
__global__ void __launch_bounds__(kThreads, (K >= 32 ? 1 : 2)) dft_recur_kernel(const KParams p) {
  using F = Fields<MODE>;
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;

  const int R = p.R, Bt = p.Bt, ct = p.ct;
  float* sComp = smem;
  float* sUVW = sComp + ct * p.cstride;
  float2* sP = reinterpret_cast<float2*>(sUVW + ((R * 3 + 1) & ~1));
  float2* sS = sP + ct * R;
  float* sQ = reinterpret_cast<float*>(sS + p.ndf * ct * R);
  float2* stage = reinterpret_cast<float2*>(smem);

  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;

  const int tr = threadIdx.x / Bt;
  const int tb = threadIdx.x - tr * Bt;
  const bool active = (tr < R);

  const int nRowTiles = (p.nvis + R - 1) / R;
  const int nItems = nRowTiles * p.nBlockTiles;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int rt = item / p.nBlockTiles;
    const int bt = item - rt * p.nBlockTiles;
    const int row0 = rt * R;
    const int blk0 = bt * Bt;
    const int nblkTile = min(Bt, p.nblocks - blk0);
    __syncthreads();  // the previous item's epilogue is done with the stage

    // rows' (u, v, w) at the reference frequency
    for (int i = threadIdx.x; i < R; i += blockDim.x) {
      const int row = row0 + i;
      float u = 0.f, v = 0.f, w = 0.f;
      if (row < p.nvis) {
        const float* rec = p.vis + (size_t)(p.rowBase + row) * p.lrec;
        u = rec[p.ilocu];
        v = rec[p.ilocv];
        w = rec[p.ilocw];
      }
      sUVW[3 * i] = u;
      sUVW[3 * i + 1] = v;
      sUVW[3 * i + 2] = w;
    }

    // this thread's channel block
    BlockDesc bd;
    const bool mine = active && (tb < nblkTile);
    if (mine) {
      bd = p.blocks[blk0 + tb];
    } else {
      bd = p.blocks[0];
    }
    const ds f0 = {bd.f0_hi, bd.f0_lo};
    const float df = bd.df;

    float2 tot[K], cmp[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      tot[k] = make_float2(0.f, 0.f);
      cmp[k] = make_float2(0.f, 0.f);
    }

    for (int c0 = 0; c0 < p.ncomp; c0 += ct) {
      __syncthreads();  // previous tile's readers are done with shared memory
      if (!stage_comps(p, sComp, c0, &bar, phase)) return;
      __syncthreads();

      // prepass over (component, row) pairs of this tile
      for (int idx = threadIdx.x; idx < ct * R; idx += blockDim.x) {
        const int c = idx / R;
        const int r = idx - c * R;
        const float* cp = sComp + c * p.cstride;
        const float u = sUVW[3 * r], v = sUVW[3 * r + 1], w = sUVW[3 * r + 2];
        // turns = (X u + Y v + Z w) / (2 pi)
        const ds P = ds_mul(ds_dot3(cp[1], u, cp[2], v, cp[3], w), ds{kInv2PiHi, kInv2PiLo});
        sP[idx] = make_float2(P.hi, P.lo);
        for (int d = 0; d < p.ndf; d++) {
          ds t = ds_mul(P, ds{p.df_hi[d], p.df_lo[d]});
          ds fr = ds_frac_turns(t);
          fr.hi -= rintf(fr.hi);
          sS[d * ct * R + idx] = phasor_accurate(fr);
        }
        if (F::kGaussian) sQ[idx] = cp[4] * u * u + cp[5] * v * v + cp[6] * u * v;
      }
      __syncthreads();

      float2 acc[K];
#pragma unroll
      for (int k = 0; k < K; k++) acc[k] = make_float2(0.f, 0.f);

      if (mine) {
        const int nc = min(ct, p.ncomp - c0);
        for (int c = 0; c < nc; c++) {
          const int idx = c * R + tr;
          const float2 Pp = sP[idx];
          const float2 st = sS[bd.dfc * ct * R + idx];
          const float* cp = sComp + c * p.cstride;
          // anchor phasor at the block's first channel
          const ds t = ds_mul(ds{Pp.x, Pp.y}, f0);
          const ds fr = ds_frac_turns(t);
          float2 z = phasor_fast(fr.hi);
          if constexpr (!F::kQuad) {
            const float A = cp[0];
            z.x *= A;
            z.y *= A;
            float2 wv = st;
#pragma unroll
            for (int k = 0; k < K; k++) {
              acc[k].x += z.x;
              acc[k].y += z.y;
              z = cmul(z, wv);
            }
          } else {
            // amplitude exponent e0 + e1 k + e2 k^2 over the block
            float e0 = 0.f, e1 = 0.f, e2 = 0.f;
            float A;
            if constexpr (F::kTSpec) {
              A = cp[F::kTabOff + bd.plane];
              const float al = cp[F::kAlphaOff];
              e0 = al * bd.l[0][0];
              e1 = al * bd.l[0][1];
              e2 = al * bd.l[0][2];
            } else {
              A = cp[0];
            }
            if constexpr (F::kSpec) {
#pragma unroll
              for (int tt = 0; tt < kMaxNTerm; tt++) {
                if (tt < p.nterm) {
                  const float a = cp[F::kSpecOff + tt];
                  e0 = __fmaf_rn(a, bd.l[tt][0], e0);
                  e1 = __fmaf_rn(a, bd.l[tt][1], e1);
                  e2 = __fmaf_rn(a, bd.l[tt][2], e2);
                }
              }
            }
            if constexpr (F::kGaussian) {
              // Q (f0 + k df)^2 with f0 ~ 1: expand exactly in k
              const float Q = sQ[idx];
              const float f = bd.f0_hi;
              e0 = __fmaf_rn(Q * f, f, e0);
              e1 = __fmaf_rn(2.0f * Q * f, df, e1);
              e2 = __fmaf_rn(Q * df, df, e2);
            }
            const float a0 = A * exp_fast(e0);
            float r0 = exp_fast(e1 + e2);
            const float q = exp_fast(2.0f * e2);
            z.x *= a0;
            z.y *= a0;
            float2 wv = make_float2(st.x * r0, st.y * r0);
#pragma unroll
            for (int k = 0; k < K; k++) {
              acc[k].x += z.x;
              acc[k].y += z.y;
              z = cmul(z, wv);
              wv.x *= q;
              wv.y *= q;
            }
          }
        }
      }
      // compensated fold of this tile's partial sums
#pragma unroll
      for (int k = 0; k < K; k++) {
        float y = acc[k].x - cmp[k].x;
        float s = tot[k].x + y;
        cmp[k].x = (s - tot[k].x) - y;
        tot[k].x = s;
        y = acc[k].y - cmp[k].y;
        s = tot[k].y + y;
        cmp[k].y = (s - tot[k].y) - y;
        tot[k].y = s;
      }
    }

    // stage the tile's model and apply it to the records
    __syncthreads();
    if (active) {
#pragma unroll
      for (int k = 0; k < K; k++) stage[(tr * Bt + tb) * K + k] = tot[k];
    }
    __syncthreads();
    apply_tile<K>(p, stage, row0, blk0, nblkTile);
  }
  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(&bar);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar_s) : "memory");
  }
}

//--------------------------------------------------------------------------
// Plain comparator: direct FP64 phase and one sin/cos per (row, channel,
// component), FP32 accumulation.  Same tiling and epilogue; every channel of
// the block evaluated independently.
//--------------------------------------------------------------------------
template <int K, int MODE>
__global__ void __launch_bounds__(kThreads, 2) dft_plain_kernel(const KParams p) {
  using F = Fields<MODE>;
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  const int R = p.R, Bt = p.Bt, ct = p.ct;
  float* sComp = smem;
  float* sUVW = sComp + ct * p.cstride;
  float2* stage = reinterpret_cast<float2*>(smem);
  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;
  const int tr = threadIdx.x / Bt;
  const int tb = threadIdx.x - tr * Bt;
  const bool active = (tr < R);
  const int nRowTiles = (p.nvis + R - 1) / R;
  const int nItems = nRowTiles * p.nBlockTiles;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int rt = item / p.nBlockTiles;
    const int bt = item - rt * p.nBlockTiles;
    const int row0 = rt * R;
    const int blk0 = bt * Bt;
    const int nblkTile = min(Bt, p.nblocks - blk0);
    __syncthreads();  // the previous item's epilogue is done with the stage
    for (int i = threadIdx.x; i < R; i += blockDim.x) {
      const int row = row0 + i;
      float u = 0.f, v = 0.f, w = 0.f;
      if (row < p.nvis) {
        const float* rec = p.vis + (size_t)(p.rowBase + row) * p.lrec;
        u = rec[p.ilocu];
        v = rec[p.ilocv];
        w = rec[p.ilocw];
      }
      sUVW[3 * i] = u;
      sUVW[3 * i + 1] = v;
      sUVW[3 * i + 2] = w;
    }
    const bool mine = active && (tb < nblkTile);
    BlockDesc bd = p.blocks[mine ? blk0 + tb : 0];
    float2 tot[K], cmp[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      tot[k] = make_float2(0.f, 0.f);
      cmp[k] = make_float2(0.f, 0.f);
    }
    for (int c0 = 0; c0 < p.ncomp; c0 += ct) {
      __syncthreads();
      if (!stage_comps(p, sComp, c0, &bar, phase)) return;
      __syncthreads();
      float2 acc[K];
#pragma unroll
      for (int k = 0; k < K; k++) acc[k] = make_float2(0.f, 0.f);
      if (mine) {
        const double u = sUVW[3 * tr], v = sUVW[3 * tr + 1], w = sUVW[3 * tr + 2];
        const int nc = min(ct, p.ncomp - c0);
        const double dfk = (double)p.df_hi[bd.dfc] + (double)p.df_lo[bd.dfc];
        const double f0 = (double)bd.f0_hi + (double)bd.f0_lo;
        for (int c = 0; c < nc; c++) {
          const float* cp = sComp + c * p.cstride;
          const double Pt = ((double)cp[1] * u + (double)cp[2] * v + (double)cp[3] * w) *
                            0.15915494309189535;
          float A = cp[0];
          float Qg = 0.f, al = 0.f;
          if constexpr (F::kTSpec) {
            A = cp[F::kTabOff + bd.plane];
            al = cp[F::kAlphaOff];
          }
          if constexpr (F::kGaussian) Qg = cp[4] * (float)(u * u) + cp[5] * (float)(v * v) +
                                          cp[6] * (float)(u * v);
#pragma unroll
          for (int k = 0; k < K; k++) {
            const double f = f0 + (double)k * dfk;
            const double t = Pt * f;
            const float r = (float)(t - rint(t));
            float s, cph;
            __sincosf(6.283185307179586f * r, &s, &cph);
            float amp = A;
            if constexpr (F::kQuad) {
              const float kk = (float)k;
              float e = 0.f;
              if constexpr (F::kTSpec) e = al * (bd.l[0][0] + kk * (bd.l[0][1] + kk * bd.l[0][2]));
              if constexpr (F::kSpec) {
                for (int tt = 0; tt < p.nterm && tt < kMaxNTerm; tt++)
                  e += cp[F::kSpecOff + tt] * (bd.l[tt][0] + kk * (bd.l[tt][1] + kk * bd.l[tt][2]));
              }
              if constexpr (F::kGaussian) {
                const float ff = (float)f;
                e += Qg * ff * ff;
              }
              amp *= exp_fast(e);
            }
            acc[k].x = __fmaf_rn(amp, cph, acc[k].x);
            acc[k].y = __fmaf_rn(amp, s, acc[k].y);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        float y = acc[k].x - cmp[k].x;
        float s = tot[k].x + y;
        cmp[k].x = (s - tot[k].x) - y;
        tot[k].x = s;
        y = acc[k].y - cmp[k].y;
        s = tot[k].y + y;
        cmp[k].y = (s - tot[k].y) - y;
        tot[k].y = s;
      }
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int k = 0; k < K; k++) stage[(tr * Bt + tb) * K + k] = tot[k];
    }
    __syncthreads();
    apply_tile<K>(p, stage, row0, blk0, nblkTile);
  }
  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(&bar);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar_s) : "memory");
  }
}

}  // namespace obit
