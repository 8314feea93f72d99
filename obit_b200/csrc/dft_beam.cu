// Beam-corrected DFT kernel (linear feeds; Stokes I, Q, U or V sky).  One
// thread per (record, selected channel-IF).  Per component tile the CTA stages
// the components and computes, once for the whole tile, the coefficients of
// every antenna-type pair at every Jones plane (beam_coeffs) in shared memory: a thread then reads its baseline's coefficients with two
// 16-byte loads, where the reference recomputes the Jones products for every
// evaluation.  Per component the phase is formed in FP64 and range-reduced
// (MUFU sin/cos of the fractional turn), the amplitude carries the model
// family's spectrum and taper, and the four products go into FP32 sums folded
// per tile into compensated totals.
// Records hold XX, YY, XY, YX; each modelled correlation with positive weight
// (any, when replacing) is subtracted from, divided into or replaced by its
// model, independently of the others.
#include <stdint.h>

#include "dft_beam.h"
#include "dft_kernels.cuh"
#include "dft_plan.h"

namespace obit {

namespace {

// GetAnts (ObitCUDABeamModel.cu:82-99): BASELINE = 256 a1 + a2 (+ subarray
// fraction), else ANTENNA1 / ANTENNA2; 0-relative.
__device__ __forceinline__ void beam_ants(const BeamKParams& p, const float* rec, int& a1, int& a2) {
  if (p.ilocb >= 0) {
    const double cb = rec[p.ilocb];
    a1 = (int)(cb / 256.0 + 0.001);
    a2 = (int)(cb - (double)a1 * 256.0 + 0.001);
  } else {
    a1 = (int)(rec[p.iloca1] + 0.5f);
    a2 = (int)(rec[p.iloca2] + 0.5f);
  }
  a1 -= 1;
  a2 -= 1;
}

// J1[i] conj(J2[j]) added to (re, im)
__device__ __forceinline__ void pconj(float ar, float ai, float br, float bi, float& re, float& im) {
  re = __fmaf_rn(ar, br, __fmaf_rn(ai, bi, re));
  im = __fmaf_rn(ai, br, __fmaf_rn(-ar, bi, im));
}

// Coefficients of the model correlations XX, XY, YX, YY from P(i, j) =
// J1[i] conj(J2[j]) for the sky's Stokes, as cudaJonesCor1_Lin_{I,Q,U,V}
// (CUDALinCorSum.h:104-455) and ObitSkyModelVMBeamJonesCorSum
// (ObitSkyModelVMBeam.c:1117-1240) form them:
//   I: XX P00+P11  XY P13+P02  YX P20+P31  YY P22+P33
//   Q: c2p D - s2p S,  U: c2p S + s2p D, with per correlation
//      XX D = P00-P11 S = P10+P01   XY D = P02-P13 S = P12+P03
//      YX D = P20-P31 S = P30+P21   YY D = P22-P33 S = P32+P23
//   V: i (P01-P13), i (P03-P12), i (P21-P30), i (P23-P32)
__device__ __forceinline__ void beam_coeffs(const BeamKParams& p, const float* J1r, const float* J1i,
                                            const float* J2r, const float* J2i, float* cr, float* ci) {
  auto P = [&](int x, int y, float& re, float& im) {
    re = 0.f;
    im = 0.f;
    pconj(J1r[x], J1i[x], J2r[y], J2i[y], re, im);
  };
  float r0, i0, r1, i1;
  if (p.stokType == 1) {
    const int a[4][4] = {{0, 0, 1, 1}, {1, 3, 0, 2}, {2, 0, 3, 1}, {2, 2, 3, 3}};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      P(a[q][0], a[q][1], r0, i0);
      P(a[q][2], a[q][3], r1, i1);
      cr[q] = r0 + r1;
      ci[q] = i0 + i1;
    }
  } else if (p.stokType == 4) {
    const int a[4][4] = {{0, 1, 1, 3}, {0, 3, 1, 2}, {2, 1, 3, 0}, {2, 3, 3, 2}};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      P(a[q][0], a[q][1], r0, i0);
      P(a[q][2], a[q][3], r1, i1);
      cr[q] = -(i0 - i1);
      ci[q] = r0 - r1;
    }
  } else {  // Q or U: D = first pair difference, S = second pair sum
    const int d[4][4] = {{0, 0, 1, 1}, {0, 2, 1, 3}, {2, 0, 3, 1}, {2, 2, 3, 3}};
    const int sm[4][4] = {{1, 0, 0, 1}, {1, 2, 0, 3}, {3, 0, 2, 1}, {3, 2, 2, 3}};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      P(d[q][0], d[q][1], r0, i0);
      P(d[q][2], d[q][3], r1, i1);
      const float Dr = r0 - r1, Di = i0 - i1;
      P(sm[q][0], sm[q][1], r0, i0);
      P(sm[q][2], sm[q][3], r1, i1);
      const float Sr = r0 + r1, Si = i0 + i1;
      if (p.stokType == 2) {
        cr[q] = p.c2p * Dr - p.s2p * Sr;
        ci[q] = p.c2p * Di - p.s2p * Si;
      } else {
        cr[q] = p.c2p * Sr + p.s2p * Dr;
        ci[q] = p.c2p * Si + p.s2p * Di;
      }
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) dft_beam_kernel(const __grid_constant__ BeamKParams p) {
  using F = Fields<MODE>;
  extern __shared__ __align__(16) float sComp[];
  const int nsel = p.nchanSel * p.nifSel;
  const long long nitems = (long long)p.nvis * nsel;
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
    rec = p.vis + (size_t)r * p.lrec;
    offCh = p.nrparm + iIF * p.incif + ich * p.incf;
    int a1, a2;
    beam_ants(p, rec, a1, a2);
    if (a1 < 0 || a1 >= p.numAnt || a2 < 0 || a2 >= p.numAnt) {
      if (p.errFlag) atomicExch(p.errFlag, 3);
      active = false;
    } else {
      t1 = p.antType[a1];
      t2 = p.antType[a2];
    }
    const double f = p.fscale[ifq];
    u = (double)rec[p.ilocu] * f;
    v = (double)rec[p.ilocv] * f;
    w = (double)rec[p.ilocw] * f;
    jc = p.jchan[ifq];
    if (p.lnspec) L = p.lnspec[ifq];
    if (p.plane) plane = p.plane[ifq];
    if (p.op != kOpRepl) {  // nothing to do when every modelled correlation is flagged
      bool any = false;
      for (int q = 0; q < p.ncorr; q++) any = any || (rec[offCh + q * p.incs + 2] > 0.0f);
      if (!any) active = false;
    }
  }
  // coefficients of the tile: [type pair][component][plane] x 8 floats
  float* sC = sComp + p.ct * p.cstride;
  const int crow = p.numJChan * 8;
  const float* Cb = sC + (size_t)(t1 * p.numAntType + t2) * p.ct * crow + jc * 8;
  const int npair = p.numAntType * p.numAntType;
  float totR[4], totI[4], cmpR[4], cmpI[4];
#pragma unroll
  for (int q = 0; q < 4; q++) totR[q] = totI[q] = cmpR[q] = cmpI[q] = 0.0f;

  for (int c0 = 0; c0 < p.ncomp; c0 += p.ct) {
    const int nc = min(p.ct, p.ncomp - c0);
    __syncthreads();  // the previous tile's readers are done
    const float* src = p.comps + (size_t)c0 * p.cstride;
    for (int i = threadIdx.x; i < nc * p.cstride; i += blockDim.x) sComp[i] = src[i];
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
      float4* d = reinterpret_cast<float4*>(sC + ((size_t)pr * p.ct + c) * crow + j * 8);
      d[0] = make_float4(cr[0], ci[0], cr[1], ci[1]);
      d[1] = make_float4(cr[2], ci[2], cr[3], ci[3]);
    }
    __syncthreads();
    if (!active) continue;
    float accR[4] = {0.f, 0.f, 0.f, 0.f}, accI[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < nc; c++) {
      const float* cp = sComp + c * p.cstride;
      float A = cp[0];
      double e = 0.0;
      if constexpr (F::kTSpec) {
        A = cp[F::kTabOff + plane];
        e = (double)cp[F::kAlphaOff] * L;
      }
      if constexpr (F::kSpec) {
        double pw = L;
        for (int t = 0; t < p.nterm && t < kMaxNTerm; t++) {
          e += (double)cp[F::kSpecOff + t] * pw;
          pw *= L;
        }
      }
      if constexpr (F::kGaussian) e += (double)cp[4] * u * u + (double)cp[5] * v * v + (double)cp[6] * u * v;
      if (e != 0.0) A *= expf((float)e);
      const double t = ((double)cp[1] * u + (double)cp[2] * v + (double)cp[3] * w) * 0.15915494309189535;
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
    float* o = rec + offCh + q * p.incs;
    if (o[2] <= 0.0f && p.op != kOpRepl) continue;
    const int m = kModelOf[q];
    const float Mr = totR[m] * p.polFact[q], Mi = totI[m] * p.polFact[q];
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

}  // namespace

int launch_beam(const BeamKParams& kp, cudaStream_t stream, std::string* err) {
  const long long nitems = (long long)kp.nvis * kp.nchanSel * kp.nifSel;
  if (nitems <= 0 || kp.ncomp <= 0) return 0;
  void (*fn)(const BeamKParams) = nullptr;
  switch (kp.mode) {
    case kPoint: fn = dft_beam_kernel<kPoint>; break;
    case kPointSpec: fn = dft_beam_kernel<kPointSpec>; break;
    case kPointTSpec: fn = dft_beam_kernel<kPointTSpec>; break;
    case kGauss: fn = dft_beam_kernel<kGauss>; break;
    case kGaussSpec: fn = dft_beam_kernel<kGaussSpec>; break;
    case kGaussTSpec: fn = dft_beam_kernel<kGaussTSpec>; break;
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
  const long long grid = (nitems + 255) / 256;
  fn<<<(unsigned)grid, 256, smem, stream>>>(kp);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("beam kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
