// Device helpers shared by the beam-corrected DFT kernels: antenna numbers of a
// record and the coefficients of the model correlations from two antennas'
// Jones matrices.
#pragma once
#include <cuda_runtime.h>

#include "dft_beam.h"
#include "ds_math.cuh"

namespace obit {

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
  if (p.circular) {
    // Circular feeds (ObitSkyModelVMBeamJonesCorSum, ObitSkyModelVMBeam.c:1039-1073
    // and the product J1 W J2^H of its :1263-1268): correlation (a, b) of RR, RL,
    // LR, LL is sum_ij M(i, j) P(2a + i, 2b + j) with the sky's matrix M:
    //   I [[1, 0], [0, 1]]  Q [[0, 1], [1, 0]]  U [[0, i], [-i, 0]]  V [[1, 0], [0, -1]]
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int a = 2 * (q >> 1), b = 2 * (q & 1);
      if (p.stokType == 1 || p.stokType == 4) {
        P(a, b, r0, i0);
        P(a + 1, b + 1, r1, i1);
        const float sg = (p.stokType == 1) ? 1.0f : -1.0f;
        cr[q] = r0 + sg * r1;
        ci[q] = i0 + sg * i1;
      } else {
        P(a, b + 1, r0, i0);
        P(a + 1, b, r1, i1);
        if (p.stokType == 2) {
          cr[q] = r0 + r1;
          ci[q] = i0 + i1;
        } else {  // U: i (P(a, b+1) - P(a+1, b))
          cr[q] = -(i0 - i1);
          ci[q] = r0 - r1;
        }
      }
    }
    return;
  }
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

// Phase turns per unit frequency ratio, (X u + Y v + Z w) / 2 pi, in split FP32
// for component c of the table (tile entry cp); with FP64 positions
// (KParams.compsLo, 4 floats per component: the low parts of X, Y, Z) their
// low parts enter as in the DFT kernels.
__device__ __forceinline__ ds beam_phase_turns(const KParams& p, const float* cp, int c, float u, float v,
                                               float w) {
  ds d;
  if (p.compsLo && c < p.ncomp) {
    const float* lo = p.compsLo + (size_t)c * 4;
    d = ds_dot3_lo(cp[1], lo[0], u, cp[2], lo[1], v, cp[3], lo[2], w);
  } else {
    d = ds_dot3(cp[1], u, cp[2], v, cp[3], w);
  }
  return ds_mul(d, ds{kInv2PiHi, kInv2PiLo});
}

}  // namespace obit
