// Beam-corrected DFT kernels (linear feeds; Stokes I, Q, U or V sky).
//
// Recurrence form (default).  A CTA tile is R records x Bt channel blocks of
// at most kBeamK = 8 channels, each block within one Jones plane; thread (row,
// block) keeps, per correlation slot (XX and YY, or XX, XY, YX, YY), the model
// of its block as 4 packed channel pairs (k, k + 4).  Per component tile:
//   (type pair, component, plane)  the coefficients of the model correlations
//                                  from the two antennas' Jones matrices
//                                  (beam_coeffs), once for the CTA, where the
//                                  reference recomputes the Jones products
//                                  for every evaluation;
//   (row, component)               split-FP32 phase turns P, the unit step s
//                                  and s^4 (accurate sin/cos), shared by the
//                                  row's blocks; the Gaussian form;
//   (component, block)             the block's spectral amplitudes (point
//                                  families with a spectrum), exact;
//   (row, component, block)        the anchor exp(2 pi i P f0) (MUFU), a packed
//                                  chain over the 4 pairs, the amplitude, and
//                                  per correlation slot one packed complex
//                                  multiply-accumulate of the baseline's
//                                  coefficient with each pair.
// Sums are FP32 per tile, folded into compensated totals (compensation terms
// in shared memory).  Records hold XX, YY, XY, YX; each modelled correlation
// with positive weight (any, when replacing) is subtracted from, divided into
// or replaced by its model, independently of the others; weights are not
// changed by a divide, as in the reference beam kernels.
//
// Plain form (the comparator, kFlavorPlain): one thread per (record, selected
// channel-IF), the phase in FP64 and MUFU sin/cos per evaluation.
#include <stdint.h>

#include <algorithm>

#include "beam_common.cuh"
#include "dft_beam.h"
#include "dft_kernels.cuh"
#include "dft_plan.h"

namespace obit {

namespace {

template <int MODE>
__global__ void __launch_bounds__(256) dft_beam_plain_kernel(const __grid_constant__ BeamKParams p) {
  using F = Fields<MODE>;
  extern __shared__ __align__(16) float sComp[];
  const int nsel = p.nchanSel * p.nifSel;
  const long long nitems = (long long)p.k.nvis * nsel;
  const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = item < nitems;
  float* rec = nullptr;
  int offCh = 0, jc = 0, plane = 0, t1 = 0, t2 = 0;
  double u = 0.0, v = 0.0, w = 0.0, L = 0.0;
  if (active) {
    const int r = (int)(item / nsel);
    const int s = (int)(item - (long long)r * nsel);
    const int ich = p.chanb + s % p.nchanSel, iIF = p.ifb + s / p.nchanSel;
    const int ifq = ich * p.kincf + iIF * p.kincif;
    rec = p.k.vis + (size_t)(p.k.rowBase + r) * p.k.lrec;
    offCh = p.nrparm + iIF * p.incif + ich * p.k.incf;
    int a1, a2;
    beam_ants(p, rec, a1, a2);
    if (a1 < 0 || a1 >= p.numAnt || a2 < 0 || a2 >= p.numAnt) {
      if (p.k.errFlag) atomicExch(p.k.errFlag, 3);
      active = false;
    } else {
      t1 = p.antType[a1];
      t2 = p.antType[a2];
    }
    const double f = p.fscale[ifq];
    u = (double)rec[p.k.ilocu] * f;
    v = (double)rec[p.k.ilocv] * f;
    w = (double)rec[p.k.ilocw] * f;
    jc = p.jchan[ifq];
    if (p.lnspec) L = p.lnspec[ifq];
    if (p.plane) plane = p.plane[ifq];
    if (p.k.op != kOpRepl) {  // nothing to do when every modelled correlation is flagged
      bool any = false;
      for (int q = 0; q < p.ncorr; q++) any = any || (rec[offCh + q * p.k.incs + 2] > 0.0f);
      if (!any) active = false;
    }
  }
  // coefficients of the tile: [type pair][component][plane] x 8 floats
  float* sC = sComp + p.k.ct * p.k.cstride;
  const int crow = p.numJChan * 8;
  const float* Cb = sC + (size_t)(t1 * p.numAntType + t2) * p.k.ct * crow + jc * 8;
  const int npair = p.numAntType * p.numAntType;
  float totR[4], totI[4], cmpR[4], cmpI[4];
#pragma unroll
  for (int q = 0; q < 4; q++) totR[q] = totI[q] = cmpR[q] = cmpI[q] = 0.0f;

  for (int c0 = 0; c0 < p.k.ncomp; c0 += p.k.ct) {
    const int nc = min(p.k.ct, p.k.ncomp - c0);
    __syncthreads();  // the previous tile's readers are done
    const float* src = p.k.comps + (size_t)c0 * p.k.cstride;
    for (int i = threadIdx.x; i < nc * p.k.cstride; i += blockDim.x) sComp[i] = src[i];
    for (int i = threadIdx.x; i < npair * nc * p.numJChan; i += blockDim.x) {
      const int pr = i / (nc * p.numJChan);
      const int rem = i - pr * nc * p.numJChan;
      const int c = rem / p.numJChan, j = rem - c * p.numJChan;
      const int ta = pr / p.numAntType, tb = pr - ta * p.numAntType;
      const float* J1 = p.jones + (((size_t)ta * p.jonesComps + c0 + c) * p.numJChan + j) * 8;
      const float* J2 = p.jones + (((size_t)tb * p.jonesComps + c0 + c) * p.numJChan + j) * 8;
      const float4 a0 = __ldg(reinterpret_cast<const float4*>(J1));
      const float4 a1 = __ldg(reinterpret_cast<const float4*>(J1 + 4));
      const float4 b0 = __ldg(reinterpret_cast<const float4*>(J2));
      const float4 b1 = __ldg(reinterpret_cast<const float4*>(J2 + 4));
      const float J1r[4] = {a0.x, a0.z, a1.x, a1.z}, J1i[4] = {a0.y, a0.w, a1.y, a1.w};
      const float J2r[4] = {b0.x, b0.z, b1.x, b1.z}, J2i[4] = {b0.y, b0.w, b1.y, b1.w};
      float cr[4], ci[4];
      beam_coeffs(p, J1r, J1i, J2r, J2i, cr, ci);
      float4* d = reinterpret_cast<float4*>(sC + ((size_t)pr * p.k.ct + c) * crow + j * 8);
      d[0] = make_float4(cr[0], ci[0], cr[1], ci[1]);
      d[1] = make_float4(cr[2], ci[2], cr[3], ci[3]);
    }
    __syncthreads();
    if (!active) continue;
    float accR[4] = {0.f, 0.f, 0.f, 0.f}, accI[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < nc; c++) {
      const float* cp = sComp + c * p.k.cstride;
      float A = cp[0];
      double e = 0.0;
      if constexpr (F::kTSpec) {
        A = cp[F::kTabOff + plane];
        e = (double)cp[F::kAlphaOff] * L;
      }
      if constexpr (F::kSpec) {
        double pw = L;
        for (int t = 0; t < p.k.nterm && t < kMaxNTerm; t++) {
          e += (double)cp[F::kSpecOff + t] * pw;
          pw *= L;
        }
      }
      if constexpr (F::kGaussian) e += (double)cp[4] * u * u + (double)cp[5] * v * v + (double)cp[6] * u * v;
      if (e != 0.0) A *= expf((float)e);
      double X = cp[1], Y = cp[2], Z = cp[3];
      if (p.k.compsLo && c0 + c < p.k.ncomp) {  // FP64 positions: the low parts of X, Y, Z
        const float* lo = p.k.compsLo + (size_t)(c0 + c) * 4;
        X += lo[0];
        Y += lo[1];
        Z += lo[2];
      }
      const double t = (X * u + Y * v + Z * w) * 0.15915494309189535;
      const float rr = (float)(t - rint(t));
      float sn, cs;
      __sincosf(6.283185307179586f * rr, &sn, &cs);
      const float vr = A * cs, vi = A * sn;
      // the baseline's coefficients for this component at the channel's plane
      const float4 k0 = *reinterpret_cast<const float4*>(Cb + (size_t)c * crow);
      const float4 k1 = *reinterpret_cast<const float4*>(Cb + (size_t)c * crow + 4);
      const float cr[4] = {k0.x, k0.z, k1.x, k1.z}, ci[4] = {k0.y, k0.w, k1.y, k1.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        accR[q] = __fmaf_rn(cr[q], vr, __fmaf_rn(-ci[q], vi, accR[q]));
        accI[q] = __fmaf_rn(cr[q], vi, __fmaf_rn(ci[q], vr, accI[q]));
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {  // compensated fold of the tile
      float y = accR[q] - cmpR[q];
      float s = totR[q] + y;
      cmpR[q] = (s - totR[q]) - y;
      totR[q] = s;
      y = accI[q] - cmpI[q];
      s = totI[q] + y;
      cmpI[q] = (s - totI[q]) - y;
      totI[q] = s;
    }
  }
  if (!active) return;
  // record correlation XX, YY, XY, YX <- model XX, YY, XY, YX
  constexpr int kModelOf[4] = {0, 3, 1, 2};
  for (int q = 0; q < p.ncorr; q++) {
    float* o = rec + offCh + q * p.k.incs;
    if (o[2] <= 0.0f && p.k.op != kOpRepl) continue;
    const int m = kModelOf[q];
    const float Mr = totR[m] * p.polFact[q], Mi = totI[m] * p.polFact[q];
    if (p.k.op == kOpRepl) {
      o[0] = Mr;
      o[1] = Mi;
    } else if (p.k.op == kOpDiv) {
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

// Model slot of each record correlation XX, YY, XY, YX: all four slots hold
// model XX, XY, YX, YY; two slots hold XX, YY.
__device__ __forceinline__ int beam_slot(int NQ, int q) {
  return NQ == 4 ? (q == 0 ? 0 : q == 1 ? 3 : q == 2 ? 1 : 2) : q;
}

template <int MODE, int NQ>
__global__ void __launch_bounds__(kThreads, 1) dft_beam_recur_kernel(const __grid_constant__ BeamKParams bp) {
  using F = Fields<MODE>;
  constexpr int K = kBeamK, H = K / 2;
  const KParams& p = bp.k;
  extern __shared__ __align__(16) float smem[];
  __shared__ __align__(8) uint64_t bar;
  const int R = p.R, Bt = p.Bt, ct = p.ct;
  const int npair = bp.numAntType * bp.numAntType;
  const int crow = bp.numJChan * 8;  // floats of one (pair, component) row of coefficients
  // floats per type pair: padded by 32 bytes so that rows of different pairs
  // (read together by a warp's records) fall in different banks
  const int pstride = ct * crow + 8;
  float* sComp = smem;
  float* sUVW = sComp + ct * p.cstride;
  int* sPair = reinterpret_cast<int*>(sUVW + ((R * 3 + 3) & ~3));
  BlockDesc* sBlk = reinterpret_cast<BlockDesc*>(sPair + ((R + 3) & ~3));
  int* sJp = reinterpret_cast<int*>(sBlk + Bt);
  float2* sP = reinterpret_cast<float2*>(sJp + ((Bt + 3) & ~3));
  float4* sS = reinterpret_cast<float4*>(sP + ct * R);
  float* sQ = reinterpret_cast<float*>(sS + p.ndf * ct * R);
  f2x* sAmp = reinterpret_cast<f2x*>(sQ + (F::kGaussian ? ct * R : 0));
  float* sC = reinterpret_cast<float*>(sAmp + (F::kTable ? ct * Bt * H : 0));
  f2x* sCmp = reinterpret_cast<f2x*>(sC + (size_t)npair * pstride);
  init_bar(&bar);
  uint32_t phase = 0;
  const int lgR = __ffs(R) - 1;
  const int lgBt = __ffs(Bt) - 1;
  const int tr = threadIdx.x & (R - 1);
  const int tb = threadIdx.x >> lgR;
  const int nt = blockDim.x;
  const int nItems = ((p.nvis + R - 1) / R) * p.nBlockTiles;
  for (int item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int rt = item / p.nBlockTiles;
    const int bt = item - rt * p.nBlockTiles;
    const int row0 = rt * R;
    const int blk0 = bt * Bt;
    const int nblkTile = min(Bt, p.nblocks - blk0);
    __syncthreads();  // the previous item is done with shared memory
#pragma unroll
    for (int j = 0; j < NQ * 2 * H; j++) sCmp[j * nt + threadIdx.x] = 0ull;
    load_uvw(p, sUVW, row0);
    for (int i = threadIdx.x; i < R; i += nt) {  // antenna-type pair of each row (-1: none)
      const int row = row0 + i;
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
      sPair[i] = pr;
    }
    for (int i = threadIdx.x; i < Bt; i += nt) {
      const BlockDesc b = p.blocks[blk0 + min(i, nblkTile - 1)];
      sBlk[i] = b;
      sJp[i] = bp.jchan[b.ifq0];
    }
    __syncthreads();
    const BlockDesc& bd = sBlk[tb];
    const int pr = sPair[tr];
    const bool mine = (tb < nblkTile) && (pr >= 0);
    const ds f0 = {bd.f0_hi, bd.f0_lo};
    const float df = bd.df;
    const float* Cb = sC + (size_t)(mine ? pr : 0) * pstride + sJp[tb] * 8;
    f2x TR[NQ][H], TI[NQ][H];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
      for (int j = 0; j < H; j++) TR[q][j] = TI[q][j] = 0ull;

    for (int c0 = 0; c0 < p.ncomp; c0 += ct) {
      __syncthreads();  // the previous tile's readers are done with shared memory
      if (!stage_comps(p, p.comps, p.ncomp, sComp, c0, &bar, phase)) return;
      const int nc = min(ct, p.ncomp - c0);
      // coefficients of the tile: [type pair][component][plane] x 8 floats
      for (int i = threadIdx.x; i < npair * ct * bp.numJChan; i += nt) {
        const int prr = i / (ct * bp.numJChan);
        const int rem = i - prr * ct * bp.numJChan;
        const int c = rem / bp.numJChan, j = rem - c * bp.numJChan;
        float4* d = reinterpret_cast<float4*>(sC + (size_t)prr * pstride + (size_t)c * crow + j * 8);
        if (c >= nc) {
          d[0] = d[1] = make_float4(0.f, 0.f, 0.f, 0.f);
          continue;
        }
        const int ta = prr / bp.numAntType, tc = prr - ta * bp.numAntType;
        const float* J1 = bp.jones + (((size_t)ta * bp.jonesComps + c0 + c) * bp.numJChan + j) * 8;
        const float* J2 = bp.jones + (((size_t)tc * bp.jonesComps + c0 + c) * bp.numJChan + j) * 8;
        const float4 a0 = __ldg(reinterpret_cast<const float4*>(J1));
        const float4 a1 = __ldg(reinterpret_cast<const float4*>(J1 + 4));
        const float4 b0 = __ldg(reinterpret_cast<const float4*>(J2));
        const float4 b1 = __ldg(reinterpret_cast<const float4*>(J2 + 4));
        const float J1r[4] = {a0.x, a0.z, a1.x, a1.z}, J1i[4] = {a0.y, a0.w, a1.y, a1.w};
        const float J2r[4] = {b0.x, b0.z, b1.x, b1.z}, J2i[4] = {b0.y, b0.w, b1.y, b1.w};
        float cr[4], ci[4];
        beam_coeffs(bp, J1r, J1i, J2r, J2i, cr, ci);
        d[0] = make_float4(cr[0], ci[0], cr[1], ci[1]);
        d[1] = make_float4(cr[2], ci[2], cr[3], ci[3]);
      }
      // (row, component): phase turns, step s and s^4, Gaussian form
      for (int idx = threadIdx.x; idx < ct * R; idx += nt) {
        const int c = idx >> lgR;
        const int r = idx & (R - 1);
        const float* cp = sComp + c * p.cstride;
        const float u = sUVW[3 * r], v = sUVW[3 * r + 1], w = sUVW[3 * r + 2];
        const ds P = beam_phase_turns(p, cp, c0 + c, u, v, w);
        sP[idx] = make_float2(P.hi, P.lo);
        if constexpr (F::kGaussian) sQ[idx] = cp[4] * u * u + cp[5] * v * v + cp[6] * u * v;
        for (int d = 0; d < p.ndf; d++) {
          const ds t = ds_mul(P, ds{p.df_hi[d], p.df_lo[d]});
          const float2 s = phasor_accurate(ds{__fsub_rn(t.hi, rintf(t.hi)), t.lo});
          const float2 s2 = cmul(s, s);
          const float2 s4 = cmul(s2, s2);
          sS[d * ct * R + idx] = make_float4(s.x, s.y, s4.x, s4.y);
        }
      }
      // (component, block): spectral amplitudes of the block's channels as
      // pairs (k, k + 4), exponentials (MUFU ex2) of the block's log-frequency
      // fits
      if constexpr (F::kTable) {
        for (int idx = threadIdx.x; idx < ct * Bt; idx += nt) {
          const int c = idx >> lgBt;
          const int b = idx & (Bt - 1);
          const float* cp = sComp + c * p.cstride;
          const BlockDesc& bb = sBlk[b];
          float A, e0 = 0.f, e1 = 0.f, e2 = 0.f;
          if constexpr (F::kTSpec) {
            A = cp[F::kTabOff + bb.plane];
            const float al = cp[F::kAlphaOff];
            e0 = al * bb.l[0][0];
            e1 = al * bb.l[0][1];
            e2 = al * bb.l[0][2];
          } else {
            A = cp[0];
#pragma unroll
            for (int t = 0; t < kMaxNTerm; t++) {
              if (t < p.nterm) {
                const float a = cp[F::kSpecOff + t];
                e0 = __fmaf_rn(a, bb.l[t][0], e0);
                e1 = __fmaf_rn(a, bb.l[t][1], e1);
                e2 = __fmaf_rn(a, bb.l[t][2], e2);
              }
            }
          }
#pragma unroll
          for (int j = 0; j < H; j++) {
            const float k1 = (float)j, k2 = (float)(j + H);
            sAmp[idx * H + j] = pk2(A * exp_fast(__fmaf_rn(k1, __fmaf_rn(k1, e2, e1), e0)),
                                    A * exp_fast(__fmaf_rn(k2, __fmaf_rn(k2, e2, e1), e0)));
          }
        }
      }
      __syncthreads();

      f2x AR[NQ][H], AI[NQ][H];
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int j = 0; j < H; j++) AR[q][j] = AI[q][j] = 0ull;
      if (mine) {
        const float4* sSd = sS + bd.dfc * ct * R;
        for (int c = 0; c < nc; c++) {
          const int i = c * R + tr;
          const float2 Pp = sP[i];
          const float4 st = sSd[i];
          float2 z0 = phasor_fast(ds_mul_frac(ds{Pp.x, Pp.y}, f0));
          const float* cp = sComp + c * p.cstride;
          if constexpr (MODE == kPoint) {
            z0.x *= cp[0];
            z0.y *= cp[0];
          }
          // pairs (b, b + 4) of the block's channels, b = 0..3
          const float2 z4 = cmul(z0, make_float2(st.z, st.w));
          f2x ZR[H], ZI[H];
          ZR[0] = pk2(z0.x, z4.x);
          ZI[0] = pk2(z0.y, z4.y);
          const f2x SR = pk2(st.x, st.x), SI = pk2(st.y, st.y), NSI = pk2(-st.y, -st.y);
#pragma unroll
          for (int j = 1; j < H; j++) {
            const f2x t1 = mul2(ZI[j - 1], NSI);
            const f2x t2 = mul2(ZI[j - 1], SR);
            ZR[j] = fma2(ZR[j - 1], SR, t1);
            ZI[j] = fma2(ZR[j - 1], SI, t2);
          }
          if constexpr (F::kTable) {
            const f2x* g = sAmp + (c * Bt + tb) * H;
#pragma unroll
            for (int j = 0; j < H; j++) {
              const f2x gj = g[j];
              ZR[j] = mul2(ZR[j], gj);
              ZI[j] = mul2(ZI[j], gj);
            }
          } else if constexpr (F::kGaussian) {
            // taper and spectrum: A exp(Q f(k)^2 + spectral exponent), one
            // exponential quadratic in the channel index k
            const float Qf = sQ[i];
            float A = cp[0];
            float e0 = Qf * bd.f0_hi * bd.f0_hi, e1 = 2.0f * Qf * bd.f0_hi * df, e2 = Qf * df * df;
            if constexpr (F::kSpec) {
#pragma unroll
              for (int t = 0; t < kMaxNTerm; t++) {
                if (t < p.nterm) {
                  const float a = cp[F::kSpecOff + t];
                  e0 = __fmaf_rn(a, bd.l[t][0], e0);
                  e1 = __fmaf_rn(a, bd.l[t][1], e1);
                  e2 = __fmaf_rn(a, bd.l[t][2], e2);
                }
              }
            } else if constexpr (F::kTSpec) {
              A = cp[F::kTabOff + bd.plane];
              const float al = cp[F::kAlphaOff];
              e0 = __fmaf_rn(al, bd.l[0][0], e0);
              e1 = __fmaf_rn(al, bd.l[0][1], e1);
              e2 = __fmaf_rn(al, bd.l[0][2], e2);
            }
#pragma unroll
            for (int j = 0; j < H; j++) {
              const float k1 = (float)j, k2 = (float)(j + H);
              const f2x gj = pk2(A * exp_fast(__fmaf_rn(k1, __fmaf_rn(k1, e2, e1), e0)),
                                 A * exp_fast(__fmaf_rn(k2, __fmaf_rn(k2, e2, e1), e0)));
              ZR[j] = mul2(ZR[j], gj);
              ZI[j] = mul2(ZI[j], gj);
            }
          }
          // the baseline's coefficients of this component at the block's plane
          const float4 k0 = *reinterpret_cast<const float4*>(Cb + (size_t)c * crow);
          const float4 k1 = *reinterpret_cast<const float4*>(Cb + (size_t)c * crow + 4);
          const float cr[4] = {k0.x, k0.z, k1.x, k1.z}, ci[4] = {k0.y, k0.w, k1.y, k1.w};
          f2x NZI[H];  // -Im, once per component (the coefficients are broadcast per slot)
#pragma unroll
          for (int j = 0; j < H; j++) NZI[j] = mul2(ZI[j], pk2(-1.0f, -1.0f));
#pragma unroll
          for (int q = 0; q < NQ; q++) {
            const int m = (NQ == 4) ? q : (q == 0 ? 0 : 3);  // model XX, XY, YX, YY
            const f2x CR = pk2(cr[m], cr[m]), CI = pk2(ci[m], ci[m]);
#pragma unroll
            for (int j = 0; j < H; j++) {
              AR[q][j] = fma2(ZR[j], CR, AR[q][j]);
              AR[q][j] = fma2(NZI[j], CI, AR[q][j]);
              AI[q][j] = fma2(ZI[j], CR, AI[q][j]);
              AI[q][j] = fma2(ZR[j], CI, AI[q][j]);
            }
          }
        }
      }
      // compensated fold of the tile's partial sums
      {
        f2x* cmp = sCmp + threadIdx.x;
#pragma unroll
        for (int q = 0; q < NQ; q++) {
#pragma unroll
          for (int j = 0; j < H; j++) {
            const int e = 2 * (q * H + j);
            f2x cc = cmp[e * nt];
            f2x y = sub2(AR[q][j], cc);
            f2x sm = add2(TR[q][j], y);
            cmp[e * nt] = sub2(sub2(sm, TR[q][j]), y);
            TR[q][j] = sm;
            cc = cmp[(e + 1) * nt];
            y = sub2(AI[q][j], cc);
            sm = add2(TI[q][j], y);
            cmp[(e + 1) * nt] = sub2(sub2(sm, TI[q][j]), y);
            TI[q][j] = sm;
          }
        }
      }
    }

    // apply the block's model to its record, correlation by correlation
    const int row = row0 + tr;
    if (mine && row < p.nvis) {
      float* rec = p.vis + (size_t)(p.rowBase + row) * p.lrec + bd.off0;
      float mr[NQ][K], mi[NQ][K];
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int j = 0; j < H; j++) {
          up2(TR[q][j], mr[q][j], mr[q][j + H]);
          up2(TI[q][j], mi[q][j], mi[q][j + H]);
        }
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (k >= bd.len) break;
        float* ch = rec + k * p.incf;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (q >= bp.ncorr) break;
          float* o = ch + q * p.incs;
          if (o[2] <= 0.0f && p.op != kOpRepl) continue;
          const int sl = beam_slot(NQ, q);
          const float Mr = mr[sl][k] * bp.polFact[q], Mi = mi[sl][k] * bp.polFact[q];
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
  inval_bar(&bar);
}

}  // namespace

size_t beam_smem_bytes(const BeamKParams& p) {
  const KParams& k = p.k;
  const size_t npair = (size_t)p.numAntType * p.numAntType;
  const size_t coeffs = npair * k.ct * p.numJChan * 8;
  if (p.flavor == kFlavorPlain) return sizeof(float) * ((size_t)k.ct * k.cstride + coeffs);
  const size_t coeffsPadded = coeffs + npair * 8;  // 32 bytes of padding per type pair
  const bool gauss = p.mode == kGauss || p.mode == kGaussSpec || p.mode == kGaussTSpec;
  const bool table = p.mode == kPointSpec || p.mode == kPointTSpec;
  const int H = kBeamK / 2;
  size_t n = (size_t)k.ct * k.cstride + ((k.R * 3 + 3) & ~3) + ((k.R + 3) & ~3) +
             (size_t)k.Bt * (sizeof(BlockDesc) / 4) + ((k.Bt + 3) & ~3) + 2 * (size_t)k.ct * k.R +
             4 * (size_t)k.ndf * k.ct * k.R + coeffsPadded;
  if (gauss) n += (size_t)k.ct * k.R;
  if (table) n += 2 * (size_t)k.ct * k.Bt * H;
  n += 2 * (size_t)beam_nq(p) * 2 * H * kThreads;  // compensation terms
  return sizeof(float) * n;
}

int beam_fit_tile(BeamKParams* p, std::string* err) {
  // one CTA per SM: 227 KB of shared memory less the static part; the plain
  // form keeps its tile within 96 KB
  const size_t budget = (p->flavor == kFlavorPlain) ? 96 * 1024 : 200 * 1024;
  int ct = 128;
  for (; ct > 8; ct -= 8) {
    p->k.ct = ct;
    if (beam_smem_bytes(*p) <= budget) break;
  }
  p->k.ct = ct;
  if (beam_smem_bytes(*p) > 220 * 1024) {
    *err = "beam tables do not fit in shared memory (too many antenna types or Jones planes)";
    return 3;
  }
  return 0;
}

int launch_beam(const BeamKParams& kp, cudaStream_t stream, std::string* err, bool prologue) {
  if (kp.mma) return launch_beam_mma(kp, stream, err, prologue);
  const KParams& k = kp.k;
  if (k.nvis <= 0 || k.ncomp <= 0 || k.nblocks <= 0) return 0;
  using Fn = void (*)(const BeamKParams);
  Fn fn = nullptr;
  const bool plain = kp.flavor == kFlavorPlain;
  const bool four = beam_nq(kp) == 4;
  switch (kp.mode) {
#define OBIT_BEAM_CASE(M)                                                                        \
  case M:                                                                                        \
    fn = plain ? dft_beam_plain_kernel<M> : four ? dft_beam_recur_kernel<M, 4> : dft_beam_recur_kernel<M, 2>; \
    break;
    OBIT_BEAM_CASE(kPoint)
    OBIT_BEAM_CASE(kPointSpec)
    OBIT_BEAM_CASE(kPointTSpec)
    OBIT_BEAM_CASE(kGauss)
    OBIT_BEAM_CASE(kGaussSpec)
    OBIT_BEAM_CASE(kGaussTSpec)
#undef OBIT_BEAM_CASE
  }
  if (!fn) {
    *err = "no beam kernel for this model type";
    return 3;
  }
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("error pending before the beam kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  const size_t smem = beam_smem_bytes(kp);
  if (int rc = raise_smem_limit((const void*)fn, smem, err)) return rc;
  long long grid;
  int threads = 256;
  if (plain) {
    grid = ((long long)k.nvis * kp.nchanSel * kp.nifSel + 255) / 256;
  } else {
    int perSM = 0, dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, threads, smem);
    if (ce != cudaSuccess || perSM < 1) {
      *err = std::string("beam kernel cannot be resident: ") + cudaGetErrorString(ce);
      return 2;
    }
    const long long nItems = (long long)((k.nvis + k.R - 1) / k.R) * k.nBlockTiles;
    grid = std::min<long long>(nItems, (long long)perSM * nsm);
  }
  fn<<<(unsigned)grid, threads, smem, stream>>>(kp);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("beam kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
