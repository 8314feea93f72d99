// DFT sky-model predict / subtract kernels for sm_100a.
//
// Work decomposition.  A visibility record (ObitUVDesc layout: nrparm random
// parameters then {re, im, weight} per correlation) is one "row".  The selected
// (channel, IF) pairs of a row are cut on the host into channel blocks of at
// most K channels that share one IF, one channel increment and (for tabulated
// spectra) one coarse plane.  A CTA tile is R rows x Bt blocks (R * Bt = 256);
// thread t owns row t % R of block t / R and keeps its K complex model sums in
// registers, so a warp covers 32 rows of one block (R >= 32) or 32/R blocks.
//
// Per component tile (ct components staged by a bulk copy) the work splits in
// levels that are each computed once and shared:
//   (row, component)            phase argument P = (X u + Y v + Z w) / 2pi in
//                               split-FP32; per channel-increment class the unit
//                               step s = exp(2 pi i P df) (accurate sin/cos) and
//                               s^(K/2); the Gaussian form g1 u^2 + g2 v^2 + g3 u v.
//   (component, block, channel) spectral amplitude A exp(E(k)) with E fitted as a
//                               quadratic in k over the block (row-independent;
//                               point families -- Gaussian families carry taper
//                               and spectrum in one per-row amplitude recurrence).
//   (row, component, block)     anchor exp(2 pi i P f0) from the range-reduced
//                               split-FP32 product (MUFU sin/cos).
//   (row, component, channel)   two packed recurrences z <- z * s over the block's
//                               halves k and k + K/2 (one f32x2 complex multiply
//                               advances both) and the packed accumulate.
//                               Point models (constant amplitude) factor channel
//                               k = 8a + b instead: G_b = A z0 s^b by a short
//                               packed chain, H_a = s^(8a) from the (row,
//                               component) level, and one packed complex
//                               multiply-accumulate G_b H_a per pair of channels.
// Component partial sums are plain FP32 within a tile and folded into a
// compensated (Kahan) total at each tile boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dft_types.h"
#include "ds_math.cuh"
#include "f32x2.cuh"

namespace obit {

// Reference field offsets inside a component record (ObitSkyModel.c:1965-2063,
// ObitSkyModelMF.c:1497-1514).
template <int MODE>
struct Fields {
  static constexpr bool kGaussian = (MODE == kGauss || MODE == kGaussSpec || MODE == kGaussTSpec);
  static constexpr bool kSpec = (MODE == kPointSpec || MODE == kGaussSpec);
  static constexpr bool kTSpec = (MODE == kPointTSpec || MODE == kGaussTSpec);
  // Point families with a spectrum read a row-independent amplitude table;
  // Gaussian families fold the spectral exponent into the per-row taper
  // recurrence (both are exp of a quadratic in the channel index).
  static constexpr bool kTable = (kSpec || kTSpec) && !kGaussian;
  static constexpr bool kQuad = (MODE != kPoint);
  static constexpr int kSpecOff = (MODE == kPointSpec) ? 4 : 7;   // first spectral coefficient
  static constexpr int kAlphaOff = (MODE == kPointTSpec) ? 4 : 7; // TSpec spectral index
  static constexpr int kTabOff = (MODE == kPointTSpec) ? 5 : 8;   // TSpec first plane flux
  // Packed chains per component: point models (unit amplitude, no per-channel
  // factor) run one chain of K/2 steps over the pairs (j, j + K/2), which
  // halves the chain starts of each (row, component, block); the others run
  // two chains of K/4 steps, keeping their amplitude recurrences short.
  static constexpr int kChains = (MODE == kPoint) ? 1 : 2;
};

// exp(x) as one MUFU.EX2 of x log2(e); flushes results below ~1e-38 to zero.
__device__ __forceinline__ float exp_fast(float x) {
  float y, t = x * 1.4426950408889634f;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(t));
  return y;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -a.y * b.y), __fmaf_rn(a.x, b.y, a.y * b.x));
}

// Accurate unit phasor exp(2 pi i r) for |r| <= ~0.5 turns; r.lo corrects the
// float rounding of r to first order.
__device__ __forceinline__ float2 phasor_accurate(ds r) {
  float s, c;
  sincospif(2.0f * r.hi, &s, &c);
  const float d = 6.283185307179586f * r.lo;
  return make_float2(__fmaf_rn(-d, s, c), __fmaf_rn(d, c, s));
}

// Anchor phasor: MUFU sin/cos of the reduced angle (its error does not compound).
__device__ __forceinline__ float2 phasor_fast(float r) {
  float s, c;
  __sincosf(6.283185307179586f * r, &s, &c);
  return make_float2(c, s);
}

// Apply the staged model of one tile to its records (subtract / divide /
// replace), with the CPU reference's polarization rules.  stage is indexed
// ((row * Bt) + block) * K + channel.
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
// kProbe (the wait-limit diagnostic instance only) takes the first wait's poll
// count from p.waitPolls; every other instance keeps it a constant, which the
// hot loops' register allocation is sensitive to.
// kLo (FP64 positions) instances also bring the tile's low parts of X, Y, Z
// (4 floats per component) into sLo on the same mbarrier; the other instances
// never touch them.
template <bool kProbe = false, bool kLo = false>
__device__ __forceinline__ bool stage_comps(const KParams& p, const float* tab, int ncomp, float* sComp,
                                            int c0, uint64_t* bar, uint32_t& phase,
                                            float* sLo = nullptr) {
  const int nc = min(p.ct, ncomp - c0);
  const uint32_t bytes = (uint32_t)nc * p.cstride * 4u;
  const float* src = tab + (size_t)c0 * p.cstride;
  const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
  const uint32_t bytesLo = kLo ? (uint32_t)nc * 16u : 0u;
  // Bulk copies need 16-byte aligned addresses and sizes; cstride is a multiple
  // of 4 floats and the table base is 256-byte aligned, so this always holds.
  if (threadIdx.x == 0) {
    const uint32_t dst_s = (uint32_t)__cvta_generic_to_shared(sComp);
    // order earlier generic-proxy accesses of this shared memory before the
    // async-proxy write of the copy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_s),
                 "r"(bytes + bytesLo)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_s),
        "l"(src), "r"(bytes), "r"(bar_s)
        : "memory");
    if (kLo && bytesLo) {
      const uint32_t lo_s = (uint32_t)__cvta_generic_to_shared(sLo);
      asm volatile(
          "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(lo_s),
          "l"(p.compsLo + (size_t)c0 * 4), "r"(bytesLo), "r"(bar_s)
          : "memory");
    }
  }
  // zero-fill the tail of the tile (and of its low parts)
  for (int i = nc * p.cstride + threadIdx.x; i < p.ct * p.cstride; i += blockDim.x) sComp[i] = 0.0f;
  if constexpr (kLo)
    for (int i = nc * 4 + threadIdx.x; i < p.ct * 4; i += blockDim.x) sLo[i] = 0.0f;
  uint32_t done = 0;
  const int polls = kProbe ? p.waitPolls : kDefaultWaitPolls;
  for (int it = 0; it < polls && !done; it++) {
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
    // give an in-flight copy a second bounded window to land before exiting
    for (int it = 0; it < (1 << 22) && !done; it++) {
      asm volatile(
          "{ .reg .pred P; mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2; selp.u32 %0, 1, 0, P; }"
          : "=r"(done)
          : "r"(bar_s), "r"(phase ^ 1u)
          : "memory");
    }
    // still in flight after both windows: the CTA leaves with the copy
    // writing its shared memory, which the host must treat as fatal for the
    // context (code 5 outranks code 2)
    if (__syncthreads_or(done == 0) && threadIdx.x == 0 && p.errFlag) atomicMax(p.errFlag, 5);
  }
  return !failed;
}

__device__ __forceinline__ void init_bar(uint64_t* bar) {
  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

__device__ __forceinline__ void inval_bar(uint64_t* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar_s) : "memory");
  }
}

// (u, v, w) of the tile's rows at the reference frequency (zero past nvis).
__device__ __forceinline__ void load_uvw(const KParams& p, float* sUVW, int row0) {
  for (int i = threadIdx.x; i < p.R; i += blockDim.x) {
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
}

// One channel step of a packed chain (two channels k and k + H): accumulate the
// model term, then advance the phasor by the unit step s (and a Gaussian
// amplitude -- taper times spectrum -- by its ratio).  g is the pair's spectral
// amplitudes (point families with a spectrum).
template <int MODE>
__device__ __forceinline__ void chain_step(f2x& ar, f2x& ai, f2x& zr, f2x& zi, const f2x g, f2x& gg,
                                           f2x& hh, const f2x qq, const f2x sr, const f2x si,
                                           const f2x nsi) {
  using F = Fields<MODE>;
  if constexpr (MODE == kPoint) {
    ar = add2(ar, zr);
    ai = add2(ai, zi);
  } else if constexpr (F::kGaussian) {
    ar = fma2(gg, zr, ar);
    ai = fma2(gg, zi, ai);
    gg = mul2(gg, hh);
    hh = mul2(hh, qq);
  } else {  // spectral table
    const f2x gv = g;
    ar = fma2(gv, zr, ar);
    ai = fma2(gv, zi, ai);
  }
  const f2x t1 = mul2(zi, nsi);
  const f2x t2 = mul2(zi, sr);
  const f2x nr = fma2(zr, sr, t1);
  zi = fma2(zr, si, t2);
  zr = nr;
}

// Recurrence state of one component over one block: two packed chains, a over
// channels (j, j + H) and b over (j + Q, j + Q + H), Q = H/2, with the shared
// unit step, and the Gaussian taper ratios when present.
template <int H>
struct CompChains {
  f2x ZRa, ZIa, ZRb, ZIb;
  f2x SR, SI, NSI;
  f2x GGa, HHa, GGb, HHb, QQ;
};

// Per (row, component, block) prologue: anchor phasor at the block's first
// channel from the split-FP32 phase, the chain starts z0, z_Q, z_H, z_(Q+H)
// (complex products with s^Q), and for Gaussian families the amplitude
// A exp(Q (f0 + k df)^2 + E_spec(k)) -- taper and spectrum, one exponential
// quadratic in the channel index k -- at the chain starts with its ratios.
template <int MODE, int H>
__device__ __forceinline__ void comp_setup(CompChains<H>& x, int c, float2 Pp, float4 st,
                                           const float* sQ, int qidx, const float* sComp,
                                           int cstride, ds f0, const BlockDesc& bd, float df,
                                           int nterm) {
  const float f0hi = bd.f0_hi;
  using F = Fields<MODE>;
  constexpr int Q = H / 2;
  float2 z0 = phasor_fast(ds_mul_frac(ds{Pp.x, Pp.y}, f0));
  if constexpr (MODE == kPoint) {
    const float A = sComp[c * cstride];
    z0.x *= A;
    z0.y *= A;
  }
  if constexpr (F::kChains == 1 || Q == 0) {
    // one chain over (j, j + H): st.zw holds s^H
    const float2 zh = cmul(z0, make_float2(st.z, st.w));
    x.ZRa = pk2(z0.x, zh.x);
    x.ZIa = pk2(z0.y, zh.y);
    x.ZRb = x.ZIb = 0ull;
  } else {
    const float2 sq = make_float2(st.z, st.w);
    const float2 zq = cmul(z0, sq);
    const float2 zh = cmul(zq, sq);
    const float2 z3 = cmul(zh, sq);
    x.ZRa = pk2(z0.x, zh.x);
    x.ZIa = pk2(z0.y, zh.y);
    x.ZRb = pk2(zq.x, z3.x);
    x.ZIb = pk2(zq.y, z3.y);
  }
  x.SR = pk2(st.x, st.x);
  x.SI = pk2(st.y, st.y);
  x.NSI = pk2(-st.y, -st.y);
  x.GGa = x.HHa = x.GGb = x.HHb = x.QQ = 0ull;
  if constexpr (F::kGaussian) {
    const float Qf = sQ[qidx];
    float e0 = Qf * f0hi * f0hi;
    float e1 = 2.0f * Qf * f0hi * df;
    float e2 = Qf * df * df;
    const float* cp = sComp + c * cstride;
    float A = cp[0];
    if constexpr (F::kSpec) {  // exp(sum_t a_t L^(t+1)), L^(t+1) fitted over the block
#pragma unroll
      for (int t = 0; t < kMaxNTerm; t++) {
        if (t < nterm) {
          const float a = cp[F::kSpecOff + t];
          e0 = __fmaf_rn(a, bd.l[t][0], e0);
          e1 = __fmaf_rn(a, bd.l[t][1], e1);
          e2 = __fmaf_rn(a, bd.l[t][2], e2);
        }
      }
    } else if constexpr (F::kTSpec) {  // plane flux x exp(alpha ln(nu / nu_plane))
      A = cp[F::kTabOff + bd.plane];
      const float al = cp[F::kAlphaOff];
      e0 = __fmaf_rn(al, bd.l[0][0], e0);
      e1 = __fmaf_rn(al, bd.l[0][1], e1);
      e2 = __fmaf_rn(al, bd.l[0][2], e2);
    }
    auto E = [&](float k) { return A * exp_fast(__fmaf_rn(k, __fmaf_rn(k, e2, e1), e0)); };
    auto D = [&](float k) { return exp_fast(__fmaf_rn(e2, 2.0f * k + 1.0f, e1)); };
    const float fh = (float)H, fq = (float)Q;
    x.GGa = pk2(E(0.f), E(fh));
    x.HHa = pk2(D(0.f), D(fh));
    if constexpr (Q > 0) {
      x.GGb = pk2(E(fq), E(fq + fh));
      x.HHb = pk2(D(fq), D(fq + fh));
    }
    const float q = exp_fast(2.0f * e2);
    x.QQ = pk2(q, q);
  }
}

//--------------------------------------------------------------------------
// Recurrence kernel.  K channels per thread (even), MODE model family.
//--------------------------------------------------------------------------

// One work item: rows [rt R, rt R + R) x channel-block tile bt of plan p, where
// item = rt * nBlockTiles + bt.  smem is the CTA's dynamic shared memory, bar
// its bulk-copy mbarrier with the running parity in phase.  Returns false (the
// error flag set, uniformly across the CTA) when a component copy did not land;
// the caller must then leave the kernel.  kFS (point families with one spectral
// index, K a multiple of 8) selects the spectral-factored form; its component
// table must be ordered by spectral index for the planner to have chosen it.
template <int K, int MODE, bool kProbe = false, bool kLo = false, bool kFS = false,
          bool kMix = false>
__device__ __forceinline__ bool recur_item(const KParams& p, int item, float* smem, uint64_t* bar,
                                           uint32_t& phase) {
  static_assert(K >= 2 && (K & 1) == 0, "K must be even");
  constexpr int H = K / 2;
  using F = Fields<MODE>;
  constexpr bool kSF = kFS && spec_factorable(MODE, K);
  constexpr bool kFact = point_factored(MODE, K) || kSF;
  // spectral amplitude table of the chain form (point families with a spectrum)
  constexpr bool kChainTable = F::kTable && !kSF;
  // Mixed instances (a Gaussian family with one spectral index): the model's
  // untapered components, taken out by the host into a point sub-table
  // (p.compsPt, ordered by spectral index), run first as the matching point
  // family in the spectral-factored form; the Gaussian components then run the
  // chain form into the same compensated totals.
  constexpr int kPtMode = (MODE == kGaussTSpec) ? kPointTSpec : kPointSpec;
  constexpr bool kMixOn =
      kMix && (MODE == kGaussSpec || MODE == kGaussTSpec) && spec_factorable(kPtMode, K);
  // shared-memory regions: the union of both passes' in mixed instances
  constexpr bool lFact = kFact || kMixOn;
  constexpr bool lSF = kSF || kMixOn;

  const int R = p.R, Bt = p.Bt, ct = p.ct;
  float* sComp = smem;
  float* sUVW = sComp + ct * p.cstride;
  BlockDesc* sBlk = reinterpret_cast<BlockDesc*>(sUVW + ((R * 3 + 3) & ~3));
  float2* sP = reinterpret_cast<float2*>(sBlk + Bt);
  float4* sS = reinterpret_cast<float4*>(sP + ct * R);
  float2* sT = reinterpret_cast<float2*>(sS + p.ndf * ct * R);
  float* sQ = reinterpret_cast<float*>(sT + (lFact ? p.ndf * ct * R : 0));
  float* sG = sQ + (F::kGaussian ? ct * R : 0);
  // spectral-factored instances: per (component, block) {A exp(e0), exp(e1),
  // exp(4 e1), exp(8 e1)}, then per (block, pair) the tile's quadratic factor
  float4* sF = reinterpret_cast<float4*>(sG);
  f2x* sPhi = reinterpret_cast<f2x*>(sG + ct * Bt * 4);
  f2x* sCmp = reinterpret_cast<f2x*>(
      sG + (lSF ? ct * Bt * 4 + Bt * K : kChainTable ? ct * Bt * 4 * ((K >= 4 ? K / 4 : 1) + 1) : 0));
  // low parts of X, Y, Z (kLo instances), after everything else
  float* sLo = reinterpret_cast<float*>(sCmp) + (lFact ? 2 * K * R * Bt : 0);
  float2* stage = reinterpret_cast<float2*>(smem);

  // R and Bt are powers of two (R * Bt == CTA size)
  const int lgR = __ffs(R) - 1;
  const int lgBt = __ffs(Bt) - 1;
  constexpr int lgH = (H >= 16) ? 4 : (H >= 8) ? 3 : (H >= 4) ? 2 : (H >= 2) ? 1 : 0;
  static_assert((1 << lgH) == H, "K/2 must be a power of two");
  constexpr int Q = H / 2;  // offset of the second packed chain
  // spectral table entries per (component, block) row: 16-byte entries
  // {pair e, pair e + QE} (QE = max(Q, 1)), plus one of padding
  constexpr int QE = (Q > 0 ? Q : 1);
  constexpr int TE = QE + 1;
  const int tr = threadIdx.x & (R - 1);  // row within the tile
  const int tb = threadIdx.x >> lgR;     // block within the tile

  {
    const int rt = item / p.nBlockTiles;
    const int bt = item - rt * p.nBlockTiles;
    const int row0 = rt * R;
    const int blk0 = bt * Bt;
    const int nblkTile = min(Bt, p.nblocks - blk0);
    __syncthreads();  // the previous item's epilogue is done with the stage

    if constexpr (lFact) {  // this thread's compensation terms start at zero
#pragma unroll
      for (int j = 0; j < 2 * H; j++) sCmp[j * blockDim.x + threadIdx.x] = 0ull;
    }
    load_uvw(p, sUVW, row0);
    for (int i = threadIdx.x; i < Bt; i += blockDim.x) sBlk[i] = p.blocks[blk0 + min(i, nblkTile - 1)];
    __syncthreads();
    const BlockDesc& bd = sBlk[tb];
    const bool mine = (tb < nblkTile);
    const ds f0 = {bd.f0_hi, bd.f0_lo};

    f2x TR[H], TI[H], CR[H], CI[H];  // compensated totals: halves k and k + H
#pragma unroll
    for (int j = 0; j < H; j++) TR[j] = TI[j] = CR[j] = CI[j] = 0ull;

    // The component tiles of a work item.  dft_recur_tile.inc is the body of
    // one tile; it reads the pass's names defined before each loop: PM (the
    // table's model family), PF = Fields<PM>, pSF (spectral-factored form),
    // pFact (factored form), pChainTable, pRemap (factored partial sums folded
    // in the chain form's pairing), tab and ncomp (the table and its size).
    if constexpr (kMixOn) {
      {  // the untapered components: point sub-table, spectral-factored form
        constexpr int PM = kPtMode;
        using PF = Fields<PM>;
        constexpr bool pSF = true, pFact = true, pChainTable = false, pRemap = true;
        const float* const tab = p.compsPt;
        const int ncomp = p.ncompPt;
        for (int c0 = 0; c0 < ncomp; c0 += ct) {
#include "dft_recur_tile.inc"
        }
      }
      {  // the Gaussian pass continues the compensated totals in registers
        const f2x* cmp = sCmp + threadIdx.x;
        const int nt = blockDim.x;
#pragma unroll
        for (int j = 0; j < H; j++) {
          CR[j] = cmp[(2 * j) * nt];
          CI[j] = cmp[(2 * j + 1) * nt];
        }
      }
      {  // the Gaussian components, chain form
        constexpr int PM = MODE;
        using PF = Fields<PM>;
        constexpr bool pSF = false, pFact = false, pChainTable = false, pRemap = false;
        const float* const tab = p.comps;
        const int ncomp = p.ncomp;
        for (int c0 = 0; c0 < ncomp; c0 += ct) {
#include "dft_recur_tile.inc"
        }
      }
    } else {
      constexpr int PM = MODE;
      using PF = Fields<PM>;
      constexpr bool pSF = kSF, pFact = kFact, pChainTable = kChainTable, pRemap = false;
      const float* const tab = p.comps;
      const int ncomp = p.ncomp;
      for (int c0 = 0; c0 < ncomp; c0 += ct) {
#include "dft_recur_tile.inc"
      }
    }

    // stage the tile's model and apply it to the records
    __syncthreads();
    {
      float2* out = stage + (tr * Bt + tb) * K;
#pragma unroll
      for (int j = 0; j < H; j++) {
        float ra, rb, ia, ib;
        up2(TR[j], ra, rb);
        up2(TI[j], ia, ib);
        // pair j: channels (j, j + H), or (8a + b, 8a + b + 4) for j = 4a + b
        const int k1 = kFact ? 8 * (j >> 2) + (j & 3) : j;
        const int k2 = kFact ? k1 + 4 : j + H;
        out[k1] = make_float2(ra, ia);
        out[k2] = make_float2(rb, ib);
      }
    }
    __syncthreads();
    apply_tile<K>(p, stage, row0, blk0, nblkTile);
  }
  return true;
}

template <int K, int MODE, bool kProbe = false, bool kLo = false, bool kFS = false,
          bool kMix = false>
__global__ void __launch_bounds__(kThreads, (K >= 32 ? 1 : 2))
    dft_recur_kernel(const __grid_constant__ KParams p) {
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  init_bar(&bar);
  uint32_t phase = 0;
  const int nItems = ((p.nvis + p.R - 1) / p.R) * p.nBlockTiles;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x)
    if (!recur_item<K, MODE, kProbe, kLo, kFS, kMix>(p, item, smem, &bar, phase)) return;
  inval_bar(&bar);
}

// Batched recurrence kernel: many facets (each its own records, layout,
// channel blocks and component table; one tile shape and model family) in one
// persistent launch.  The work items of all facets form one list, facets in
// decreasing cost per item; CTAs take items from a device counter (zero at
// launch) so uneven facets balance across the SMs, and load a facet's
// parameter block into shared memory when they move to a new facet.
template <int K, int MODE>
__global__ void __launch_bounds__(kThreads, (K >= 32 ? 1 : 2))
    dft_recur_batch_kernel(const __grid_constant__ BatchParams bp) {
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(16) KParams sp;
  __shared__ int sItem, sFacet;
  init_bar(&bar);
  uint32_t phase = 0;
  const int total = bp.itemStart[bp.nfacet];
  int cur = -1;
  for (;;) {
    __syncthreads();  // every thread is done with the previous item and with sp
    if (threadIdx.x == 0) {
      const int it = atomicAdd(bp.counter, 1);
      int f = 0;
      if (it < total) {  // facet f with itemStart[f] <= it < itemStart[f + 1]
        int lo = 0, hi = bp.nfacet - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (bp.itemStart[mid] <= it) lo = mid; else hi = mid - 1;
        }
        f = lo;
      }
      sItem = it;
      sFacet = f;
    }
    __syncthreads();
    const int it = sItem;
    if (it >= total) break;
    const int f = sFacet;
    if (f != cur) {
      const int* src = reinterpret_cast<const int*>(bp.facets + f);
      int* dst = reinterpret_cast<int*>(&sp);
      for (int i = threadIdx.x; i < (int)(sizeof(KParams) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
      cur = f;
      __syncthreads();
    }
    if (!recur_item<K, MODE>(sp, it - bp.itemStart[f], smem, &bar, phase)) return;
  }
  inval_bar(&bar);
}

//--------------------------------------------------------------------------
// Plain comparator: direct FP64 phase and one sin/cos per (row, channel,
// component), FP32 accumulation.  Same tiling, component staging and epilogue;
// every channel of the block evaluated independently.
//--------------------------------------------------------------------------
template <int K, int MODE, bool kLo = false>
__global__ void __launch_bounds__(kThreads, 2) dft_plain_kernel(const KParams p) {
  using F = Fields<MODE>;
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  const int R = p.R, Bt = p.Bt, ct = p.ct;
  float* sComp = smem;
  float* sUVW = sComp + ct * p.cstride;
  float* sLo = sUVW + ((R * 3 + 3) & ~3);  // low parts of X, Y, Z (kLo instances)
  float2* stage = reinterpret_cast<float2*>(smem);
  init_bar(&bar);
  uint32_t phase = 0;
  const int tr = threadIdx.x % R;
  const int tb = threadIdx.x / R;
  const int nRowTiles = (p.nvis + R - 1) / R;
  const int nItems = nRowTiles * p.nBlockTiles;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int rt = item / p.nBlockTiles;
    const int bt = item - rt * p.nBlockTiles;
    const int row0 = rt * R;
    const int blk0 = bt * Bt;
    const int nblkTile = min(Bt, p.nblocks - blk0);
    __syncthreads();  // the previous item's epilogue is done with the stage
    load_uvw(p, sUVW, row0);
    const bool mine = (tb < nblkTile);
    const BlockDesc bd = p.blocks[blk0 + min(tb, nblkTile - 1)];
    float2 tot[K], cmp[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      tot[k] = make_float2(0.f, 0.f);
      cmp[k] = make_float2(0.f, 0.f);
    }
    for (int c0 = 0; c0 < p.ncomp; c0 += ct) {
      __syncthreads();
      if (!stage_comps<false, kLo>(p, p.comps, p.ncomp, sComp, c0, &bar, phase, sLo)) return;
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
          double Pt = (double)cp[1] * u + (double)cp[2] * v + (double)cp[3] * w;
          if constexpr (kLo) {  // FP64 positions: the low parts' share of the phase
            const float* lo = sLo + 4 * c;
            Pt += (double)lo[0] * u + (double)lo[1] * v + (double)lo[2] * w;
          }
          Pt *= 0.15915494309189535;
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
#pragma unroll
    for (int k = 0; k < K; k++) stage[(tr * Bt + tb) * K + k] = tot[k];
    __syncthreads();
    apply_tile<K>(p, stage, row0, blk0, nblkTile);
  }
  inval_bar(&bar);
}

}  // namespace obit
