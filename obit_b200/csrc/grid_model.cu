// Device half of the gridded model FT (include/obit_dft_grid.h).
//
// Per field (obit_dft_grid_create): one thread per CC row finds its cell in the
// zeroed, quadrant-swapped grid of nx x ny floats (grid_rows_kernel), a stable
// radix sort by cell keeps each cell's rows in row order, and the first row of
// each cell sums them (grid_cells_kernel), as the reference adds them; cuFFT
// transforms it to ny rows of nx/2 + 1 complex values; one kernel then writes
// the interpolator's plane -- rows swapped (ObitCArray2DCenter), the Gaussian
// taper applied, HWIDTH conjugate columns in front (ObitCArrayAddConjg) -- in
// rows of `pitch` complex values, and the FFT buffers are released.
//
// Per call (obit_dft_grid_apply), grid_apply_kernel: one warp per 32
// consecutive (IF, channel) pairs of a record.  Phase A, a lane per pair: u, v,
// w at the channel, re-projection or rotation, the half-plane conjugation, the
// plane pixel and the interpolation window with its 25 + 25 weights (the
// reference's table rows, or exact Lagrange weights) into the warp's
// shared-memory slots.  Phase B, the whole warp, a group of up to kGroup
// pairs at a time whose windows fit one union of kUnion x kUnion cells
// (channels of a record move their windows by a fraction of a cell each, so
// neighbours share most of them): the 16 lanes of each half-warp read a row of
// the union as 16-byte column pairs, the half-warps take alternate rows, and
// each lane sums its column pair over the rows with every member's row
// weights; then each member's column weights and a warp reduction.  Each union
// row is read once per group instead of once per pair.  Phase C, a lane
// per pair again: normalization, field-offset phase, conjugation back, doFlip,
// and subtract / divide / replace over the selected polarizations.  Every
// single-precision step that decides a window or a table row rounds as the
// reference's code does (no contraction), so the windows and rows are the
// reference's.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cufft.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>

#include "abi_internal.h"
#include "grid_host.h"
#include "obit_dft_grid.h"

using obit::GridHostPlan;
using obit::kGridHalfWidth;
using obit::kGridTableRows;
using obit::kGridTaps;

struct ObitDFTGrid {
  int device = 0;
  int kernel = OBIT_DFT_GRID_KERNEL_REFERENCE;
  GridHostPlan hp;
  float2* d_plane = nullptr;  // hp.rows rows (ny, then zero rows) of hp.pitch complex values
  float* d_table = nullptr;   // kGridTableRows x kGridTaps
  float* d_stage = nullptr;   // records of apply_host
  size_t stageBytes = 0;
  float* d_fscale = nullptr;  // device copy of a host freqScale
  size_t fscaleCount = 0;
  // apply_host: copy/compute streams of the chunked pipeline and their events
  static constexpr int kHostStreams = 3;
  cudaStream_t hs[kHostStreams] = {};
  cudaEvent_t hev[kHostStreams + 1] = {};
  bool haveStreams = false;
};

namespace {

int fail(int code, const std::string& msg) {
  obit::set_last_error(msg);
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess)                                                          \
      return fail(OBIT_DFT_ECUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
  } while (0)

// ---- field set-up kernels ----------------------------------------------------

struct RowGridParams {
  const float *flux, *dx, *dy;
  int n;
  obit::GridRows r;
  int* keys;       // cell of each row in the quadrant-swapped grid, INT_MAX when the row is not gridded
  float* vals;     // its flux times factor
  int* counters;   // [0] rows gridded, [1] rows off a cell centre by more than 0.1
};

// ObitTableCCUtilGrid's row body (ObitTableCCUtil.c:230-290) for one row, in
// its single-precision steps: Factor, the reference-pixel offset, the flux
// window, the off-cell warning, the clip, the nearest cell.
__global__ void grid_rows_kernel(RowGridParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const obit::GridRows& r = p.r;
  const float flux = __fmul_rn(p.flux[i], r.factor);
  float dx = __fadd_rn(p.dx[i], r.xpoff), dy = __fadd_rn(p.dy[i], r.ypoff);
  int key = INT_MAX;
  const double af = fabs((double)flux);
  if (!(af < (double)r.minFlux || flux == 0.0f) && !(af > (double)r.maxGrid)) {
    const float tx = __fmul_rn(dx, r.iCellX), ty = __fmul_rn(dy, r.iCellY);
    const int ix = tx > 0.0f ? (int)((double)tx + 0.5) : (int)((double)tx - 0.5);
    const int iy = ty > 0.0f ? (int)((double)ty + 0.5) : (int)((double)ty - 0.5);
    if (__fsub_rn(tx, (float)ix) > 0.1f || __fsub_rn(ty, (float)iy) > 0.1f) atomicAdd(&p.counters[1], 1);
    dx = dx < r.minX ? r.minX : dx;  // MIN (maxX, MAX (dx, minX))
    dx = r.maxX < dx ? r.maxX : dx;
    dy = dy < r.minY ? r.minY : dy;
    dy = r.maxY < dy ? r.maxY : dy;
    dx = __fmul_rn(dx, r.iCellX);
    dy = __fmul_rn(dy, r.iCellY);
    int xPix = (int)((double)__fadd_rn(dx, (float)(r.nx / 2)) + 0.5);
    int yPix = (int)((double)__fadd_rn(dy, (float)(r.ny / 2)) + 0.5);
    // the reference's clip admits one cell past the last column or row (cdelt < 0),
    // where it would write outside its grid; such a component stays on the edge
    xPix = min(max(xPix, 0), r.nx - 1);
    yPix = min(max(yPix, 0), r.ny - 1);
    // ObitFArray2DCenter's quadrant swap folded into the cell index
    key = ((yPix + r.ny / 2) % r.ny) * r.nx + (xPix + r.nx / 2) % r.nx;
    atomicAdd(&p.counters[0], 1);
  }
  p.keys[i] = key;
  p.vals[i] = flux;
}

// After a stable sort by cell: the first row of each cell sums the cell's
// fluxes in row order, as the reference adds them into its grid.
__global__ void grid_cells_kernel(const int* __restrict__ keys, const float* __restrict__ vals, int n,
                                  float* __restrict__ grid) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int k = keys[j];
  if (k == INT_MAX || (j > 0 && keys[j - 1] == k)) return;
  float s = 0.0f;
  for (int t = j; t < n && keys[t] == k; t++) s = __fadd_rn(s, vals[t]);
  grid[k] = s;
}

struct PlaneParams {
  const float2* fft;  // ny rows of nx/2 + 1
  float2* plane;
  int nx, ny, pitch, nxp;
  int doGaus;
  float b1, b2, b3, dV;
  const float* UU;
};

// Tapered FFT value at centred row r (ky = r - ny/2) and half-plane column j,
// the taper in the reference's single-precision steps (ObitSkyModel.c:4315-4331).
__device__ __forceinline__ float2 tapered(const PlaneParams& p, int r, int j) {
  const int nh = p.nx / 2 + 1;
  float2 v = p.fft[(size_t)((r + p.ny / 2) % p.ny) * nh + j];
  if (p.doGaus) {
    const float VV = __fmul_rn(p.dV, (float)(r - p.nx / 2));
    const float bb2 = __fmul_rn(__fmul_rn(p.b2, VV), VV);
    const float bb3 = __fmul_rn(p.b3, VV);
    const float UU = p.UU[j];
    const float texp = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(p.b1, UU), UU), bb2), __fmul_rn(bb3, UU));
    const float t = texp > -14.0f ? (float)exp((double)texp) : 0.0f;
    v.x = __fmul_rn(v.x, t);
    v.y = __fmul_rn(v.y, t);
  }
  return v;
}

__global__ void grid_plane_kernel(PlaneParams p) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= p.pitch) return;
  float2 out = make_float2(0.0f, 0.0f);
  constexpr int H = kGridHalfWidth;
  if (c < p.nxp && r < p.ny) {
    if (c >= H) {
      out = tapered(p, r, c - H);
    } else {
      // conjugate columns; row 0 reads columns H + 1 .. 2H of itself (ObitCArray.c:1712-1722)
      const float2 s = r >= 1 ? tapered(p, p.ny - r, H - c) : tapered(p, 0, 2 * H - c);
      out = make_float2(s.x, -s.y);
    }
  }
  p.plane[(size_t)r * p.pitch + c] = out;
}

// ---- the per-record kernel ------------------------------------------------------

struct GridApplyParams {
  const float2* plane;
  int pitch, nxp, nyp;
  float crpix0, crpix1, cdelt0, cdelt1;
  const float* table;
  int exact;
  float flip;
  int do3Dmul, doRot, doPC;
  float um[9];
  float ccrot, ssrot;
  float d0, d1, d2;
  float* vis;
  int nvis, lrec, nrparm, ilocu, ilocv, ilocw;
  const float* fscale;
  int kincf, kincif;
  int chanb, nchan, ifb, nif;
  int incf, incif, incs;  // floats
  int stokb, nstok;
  int op;
  float stokFactor;
  int doFlip;
  int nsel, nchunk;       // selected (IF, channel) pairs per record; 32-pair chunks
};

constexpr int kApplyWarps = 4;
constexpr int kSlack = 6;                      // window starts of a group's members span at most this
constexpr int kUnion = kGridTaps + kSlack;     // union rows and columns (31)
constexpr int kGroup = 8;                      // members summed together (registers: 4 each)
// A lane's weight slots, zero-padded so that a member's weight at union row r
// (column c) is slot r - dy + kSlack (c - dx + kSlack + 1), dy, dx its window's
// offset in the union: rows 0..kUnion-1, columns -1..kUnion.
constexpr int kWX = kGridTaps + 2 * kSlack + 3;  // 40: [0, kSlack+1) zero, 25 weights, zeros
constexpr int kWY = kGridTaps + 2 * kSlack + 1;  // 38: [0, kSlack) zero, 25 weights, zeros

// SetConvKernal (ObitCInterpolate.c:699-745): window start, first table tap,
// taps and table row for a pixel (1-relative) on an axis of naxis pixels.
__device__ __forceinline__ void conv_setup(float pix, int naxis, int* start, int* k0, int* nterm, int* itab) {
  constexpr int hw = kGridHalfWidth, iwid = kGridTaps, ntab = kGridTableRows - 1;
  const int ipos = (int)((double)pix + 0.5);
  int cen = ipos - hw;
  cen = max(1, min(cen, naxis - iwid));
  float off = __fsub_rn(__fsub_rn(pix, (float)cen), (float)hw);
  const double od = (double)off;
  const int ioff = od > 0.0 ? (int)(od + 0.5) : (int)(od - 0.5);
  off = __fsub_rn(off, (float)ioff);
  int it = (int)(((0.5 + (double)off) * (double)ntab) + 0.5);
  *itab = max(0, min(it, ntab));
  *start = cen - 1;
  *k0 = abs(ioff);
  *nterm = iwid - abs(ioff);
}

// Reference weights from table row itab, taps k0 .. 24, into w[off + i].
__device__ __forceinline__ float table_weights(const float* __restrict__ tab, int itab, int k0, int nterm,
                                               float* w) {
  float s = 0.0f;
  for (int i = 0; i < kGridTaps; i++) {
    const float v = i < nterm ? __ldg(tab + itab * kGridTaps + k0 + i) : 0.0f;
    w[i] = v;
    s += v;
  }
  return s;
}

// Barycentric weights (-1)^i C(24, i) of 25 equispaced nodes (integers below 2^24).
__constant__ float kBaryLam[kGridTaps] = {
    1.f,        -24.f,      276.f,      -2024.f,    10626.f,    -42504.f,  134596.f,
    -346104.f,  735471.f,   -1307504.f, 1961256.f,  -2496144.f, 2704156.f, -2496144.f,
    1961256.f,  -1307504.f, 735471.f,   -346104.f,  134596.f,   -42504.f,  10626.f,
    -2024.f,    276.f,      -24.f,      1.f};

// Exact 25-point Lagrange weights at position t (0 .. 24) of the window, by the
// barycentric formula; the quotients in fast single precision (2 ulp), whose
// errors the normalization by their sum leaves at the 1e-7 level.
__device__ __forceinline__ float exact_weights(float t, float* w) {
  float s = 0.0f;
  int hit = -1;
  for (int i = 0; i < kGridTaps; i++) {
    const float d = t - (float)i;
    if (d == 0.0f) hit = i;
    const float v = d != 0.0f ? __fdividef(kBaryLam[i], d) : 0.0f;
    w[i] = v;
    s += v;
  }
  if (hit >= 0) {
    for (int i = 0; i < kGridTaps; i++) w[i] = i == hit ? 1.0f : 0.0f;
    return 1.0f;
  }
  const float inv = 1.0f / s;
  for (int i = 0; i < kGridTaps; i++) w[i] *= inv;
  return 1.0f;
}

// Rows of a window union summed for G members: this lane's column pair of
// rows half, half + 2, ... (the other half-warp takes the rest), each row
// weighted by every member's row weight; members beyond G are zero.
template <int G>
__device__ __forceinline__ void union_rows(const float4* __restrict__ base4, size_t step, int half,
                                           const float* swb, const int* wo, float4* acc) {
#pragma unroll
  for (int k = 0; k < kGroup; k++) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int rr = 0; rr < (kUnion + 1) / 2; rr++) {
    if (2 * rr + half < kUnion) {
      const float4 q = __ldg(base4 + rr * step);
#pragma unroll
      for (int k = 0; k < G; k++) {
        const float w = swb[wo[k] + 2 * rr];
        acc[k].x = fmaf(w, q.x, acc[k].x);
        acc[k].y = fmaf(w, q.y, acc[k].y);
        acc[k].z = fmaf(w, q.z, acc[k].z);
        acc[k].w = fmaf(w, q.w, acc[k].w);
      }
    }
  }
}

__global__ void __launch_bounds__(kApplyWarps * 32, 3) grid_apply_kernel(GridApplyParams p) {
  __shared__ float sw[kApplyWarps][32][kWX + kWY];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float* mywx = sw[wib][lane];
  float* mywy = mywx + kWX;
  const long long nitems = (long long)p.nvis * p.nchunk;
  for (long long item = (long long)blockIdx.x * kApplyWarps + wib; item < nitems;
       item += (long long)gridDim.x * kApplyWarps) {
    const int rec = (int)(item / p.nchunk), chunk = (int)(item % p.nchunk);
    const int fidx = chunk * 32 + lane;
    const bool valid = fidx < p.nsel;
    const int iIF = p.ifb + (valid ? fidx / p.nchan : 0);
    const int iCh = p.chanb + (valid ? fidx % p.nchan : 0);
    float* rp = p.vis + (size_t)rec * p.lrec;

    // ---- phase A: this lane's (IF, channel) ----
    float u = 0.f, v = 0.f, w = 0.f, sumwt = 0.f;
    int sx = 0, sy = 0;
    bool bad = true, conj = false;
    if (valid) {
      const float ff = __ldg(p.fscale + iIF * p.kincif + iCh * p.kincf);
      u = __fmul_rn(ff, rp[p.ilocu]);
      v = __fmul_rn(ff, rp[p.ilocv]);
      w = __fmul_rn(ff, rp[p.ilocw]);
      if (p.do3Dmul) {
        const float* m = p.um;
        const float ut = __fadd_rn(__fadd_rn(__fmul_rn(u, m[0]), __fmul_rn(v, m[1])), __fmul_rn(w, m[2]));
        const float vt = __fadd_rn(__fadd_rn(__fmul_rn(u, m[3]), __fmul_rn(v, m[4])), __fmul_rn(w, m[5]));
        const float wt = __fadd_rn(__fadd_rn(__fmul_rn(u, m[6]), __fmul_rn(v, m[7])), __fmul_rn(w, m[8]));
        u = ut;
        v = vt;
        w = wt;
      } else if (p.doRot) {
        const float ut = __fsub_rn(__fmul_rn(p.ccrot, u), __fmul_rn(p.ssrot, v));
        const float vt = __fadd_rn(__fmul_rn(p.ccrot, v), __fmul_rn(p.ssrot, u));
        u = ut;
        v = vt;
      }
      conj = __fmul_rn(p.flip, u) < 0.0f;
      if (conj) {
        u = -u;
        v = -v;
        w = -w;
      }
      const float px = __fadd_rn(p.crpix0, __fdiv_rn(u, p.cdelt0));
      const float py = __fadd_rn(p.crpix1, __fdiv_rn(v, p.cdelt1));
      if (px >= 1.0f && px <= (float)p.nxp && py >= 1.0f && py <= (float)p.nyp) {
        for (int i = 0; i < kSlack + 1; i++) mywx[i] = 0.0f;
        for (int i = kSlack + 1 + kGridTaps; i < kWX; i++) mywx[i] = 0.0f;
        for (int i = 0; i < kSlack; i++) mywy[i] = 0.0f;
        for (int i = kSlack + kGridTaps; i < kWY; i++) mywy[i] = 0.0f;
        float* wxs = mywx + kSlack + 1;
        float* wys = mywy + kSlack;
        if (!p.exact) {
          int k0, nt, it;
          conv_setup(px, p.nxp, &sx, &k0, &nt, &it);
          const float swx = table_weights(p.table, it, k0, nt, wxs);
          conv_setup(py, p.nyp, &sy, &k0, &nt, &it);
          const float swy = table_weights(p.table, it, k0, nt, wys);
          sumwt = swx * swy;
        } else {
          // the requested point itself: 0-relative position px (py) on the plane, a
          // window centred on it; a point whose window would leave the plane is
          // blanked as off the plane (an edge window would extrapolate)
          sx = (int)floorf(px + 0.5f) - kGridHalfWidth;
          sy = (int)floorf(py + 0.5f) - kGridHalfWidth;
          if (sx >= 0 && sx + kGridTaps <= p.nxp && sy >= 0 && sy + kGridTaps <= p.nyp) {
            exact_weights(px - (float)sx, wxs);
            sumwt = exact_weights(py - (float)sy, wys);
          }
        }
        bad = !(sumwt > 0.5f);
      }
    }
    __syncwarp();

    // ---- phase B: the window sums, a group of members per union ----
    float mr = 0.f, mi = 0.f;
    unsigned todo = __ballot_sync(0xffffffffu, valid && !bad);
    const int cp = lane & 15, half = lane >> 4;
    while (todo) {
      // anchor: the first pending pair; the union extends from its window in the
      // direction the last pending pair's window lies
      const int c0 = __ffs(todo) - 1, cl = 31 - __clz(todo);
      const int ax = __shfl_sync(0xffffffffu, sx, c0), ay = __shfl_sync(0xffffffffu, sy, c0);
      const int lx = __shfl_sync(0xffffffffu, sx, cl), ly = __shfl_sync(0xffffffffu, sy, cl);
      const int ux = max(lx >= ax ? ax : ax - kSlack, 0);
      const int uy = max(ly >= ay ? ay : ay - kSlack, 0);
      const bool fits = ((todo >> lane) & 1u) && sx >= ux && sx <= ux + kSlack && sy >= uy && sy <= uy + kSlack;
      unsigned sel = __ballot_sync(0xffffffffu, fits);
      int mem[kGroup], dxm[kGroup], dym[kGroup];
      int cnt = 0;
#pragma unroll
      for (int k = 0; k < kGroup; k++) {
        mem[k] = sel ? __ffs(sel) - 1 : 0;
        if (sel) {
          sel &= sel - 1;
          cnt = k + 1;
        }
      }
#pragma unroll
      for (int k = 0; k < kGroup; k++) {
        dxm[k] = __shfl_sync(0xffffffffu, sx, mem[k]) - ux;
        dym[k] = __shfl_sync(0xffffffffu, sy, mem[k]) - uy;
        if (k < cnt) todo &= ~(1u << mem[k]);
      }
      const int x0e = ux & ~1;
      const float4* base4 = reinterpret_cast<const float4*>(p.plane + (size_t)(uy + half) * p.pitch + x0e) + cp;
      const size_t step = (size_t)p.pitch;  // two rows, in float4
      // each member's row weight of this lane's first row (slot offsets in the warp's slots)
      const float* swb = &sw[wib][0][0];
      int wo[kGroup];
#pragma unroll
      for (int k = 0; k < kGroup; k++)  // members beyond cnt read lane 0's slots (in range; unused)
        wo[k] = k < cnt ? mem[k] * (kWX + kWY) + kWX + kSlack - dym[k] + half : kWX;
      float4 acc[kGroup];
      if (cnt <= kGroup / 2)
        union_rows<kGroup / 2>(base4, step, half, swb, wo, acc);
      else
        union_rows<kGroup>(base4, step, half, swb, wo, acc);
      const int cc = x0e + 2 * cp - ux;  // union column of this lane's first value: -1 .. kUnion
      float V[2 * kGroup];                // each member's column-weighted (re, im) of this lane
#pragma unroll
      for (int k = 0; k < kGroup; k++) {
        V[2 * k] = V[2 * k + 1] = 0.f;
        if (k < cnt) {
          const float* wxk = sw[wib][mem[k]];
          const int i0 = cc - dxm[k] + kSlack + 1;
          const float wa = wxk[i0], wb = wxk[i0 + 1];
          V[2 * k] = fmaf(wa, acc[k].x, wb * acc[k].z);
          V[2 * k + 1] = fmaf(wa, acc[k].y, wb * acc[k].w);
        }
      }
      int myk = -1;
#pragma unroll
      for (int k = 0; k < kGroup; k++)
        if (k < cnt && mem[k] == lane) myk = k;
      if (cnt <= 2) {
        // few members: one warp sum each
#pragma unroll
        for (int k = 0; k < 2; k++) {
          if (k < cnt) {
            float sr = V[2 * k], si = V[2 * k + 1];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              sr += __shfl_xor_sync(0xffffffffu, sr, o);
              si += __shfl_xor_sync(0xffffffffu, si, o);
            }
            if (myk == k) {
              mr = sr;
              mi = si;
            }
          }
        }
      } else {
        // the 16 values summed over the warp by recursive halving: after the
        // steps of 16, 8, 4, 2 lanes each lane holds the partial sum of value
        // lane >> 1 over 16 lanes, and the step of 1 completes it
#pragma unroll
        for (int m = kGroup, o = 16; m >= 1; m >>= 1, o >>= 1) {
          const bool upper = (lane & o) != 0;
#pragma unroll
          for (int j = 0; j < m; j++) {
            const float send = upper ? V[j] : V[j + m];
            const float keep = upper ? V[j + m] : V[j];
            V[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
          }
        }
        V[0] += __shfl_xor_sync(0xffffffffu, V[0], 1);
        const int src = myk < 0 ? 0 : 4 * myk;
        const float sr = __shfl_sync(0xffffffffu, V[0], src);
        const float si = __shfl_sync(0xffffffffu, V[0], src + 2);
        if (myk >= 0) {
          mr = sr;
          mi = si;
        }
      }
    }
    __syncwarp();

    // ---- phase C: this lane's (IF, channel) applied to its polarizations ----
    if (valid) {
      float wtf = 1.0f;
      if (!bad) {
        mr = __fdiv_rn(mr, sumwt);
        mi = __fdiv_rn(mi, sumwt);
        if (p.doPC) {
          const float pc = __fadd_rn(__fadd_rn(__fmul_rn(u, p.d0), __fmul_rn(v, p.d1)), __fmul_rn(w, p.d2));
          double sd, cd;
          sincos((double)pc, &sd, &cd);
          const float cs = (float)cd, sn = (float)sd;
          const float rt = __fsub_rn(__fmul_rn(cs, mr), __fmul_rn(sn, mi));
          const float it = __fadd_rn(__fmul_rn(cs, mi), __fmul_rn(sn, mr));
          mr = rt;
          mi = it;
        }
        if (conj) mi = -mi;
        if (p.doFlip) {
          const float t = mr;
          mr = -mi;
          mi = t;
        }
        if (p.op == GPUOpTypeDiv) {
          const float wt = __fadd_rn(__fmul_rn(mr, mr), __fmul_rn(mi, mi));
          mr = __fdiv_rn(mr, wt);
          mi = __fdiv_rn(mi, wt);
          wtf = __fsqrt_rn(wt);
        }
      }
      float* base = rp + p.nrparm + iIF * p.incif + iCh * p.incf;
      for (int s = p.stokb; s < p.stokb + p.nstok; s++) {
        float* cv = base + s * p.incs;
        if (cv[2] <= 0.0f && p.op != GPUOpTypeRepl) continue;
        if (bad) {
          cv[0] = 0.0f;
          cv[1] = 0.0f;
          cv[2] = 0.0f;
        } else if (p.op == GPUOpTypeDiv) {
          const float vr = cv[0], vi = cv[1];
          cv[0] = __fadd_rn(__fmul_rn(mr, vr), __fmul_rn(mi, vi));
          cv[1] = __fsub_rn(__fmul_rn(mr, vi), __fmul_rn(mi, vr));
          cv[2] = __fmul_rn(cv[2], wtf);
        } else if (p.op == GPUOpTypeRepl) {
          cv[0] = mr;
          cv[1] = mi;
        } else {
          cv[0] = __fsub_rn(cv[0], mr);
          cv[1] = __fsub_rn(cv[1], mi);
        }
        mr = __fmul_rn(mr, p.stokFactor);
        mi = __fmul_rn(mi, p.stokFactor);
      }
    }
  }
}

int apply_params(const ObitDFTGrid* g, const GPUVisInfo* v, int opType, float stokFactor, int doFlip,
                 float* d_vis, int nvis, GridApplyParams* p) {
  if (!v) return fail(OBIT_DFT_EBADARG, "grid apply: null GPUVisInfo");
  if (opType < GPUOpTypeSub || opType > GPUOpTypeRepl) return fail(OBIT_DFT_EBADARG, "grid apply: bad opType");
  if (nvis < 0 || (nvis > 0 && !d_vis)) return fail(OBIT_DFT_EBADARG, "grid apply: bad records");
  if (!v->freqScale) return fail(OBIT_DFT_EBADARG, "grid apply: freqScale is required");
  if (v->lenvis <= 0 || v->nrparm < 0 || v->nchan <= 0 || v->nIF <= 0 || v->nstok <= 0)
    return fail(OBIT_DFT_EBADARG, "grid apply: bad record layout");
  if (v->ilocu < 0 || v->ilocv < 0 || v->ilocw < 0 || v->ilocu >= v->nrparm || v->ilocv >= v->nrparm ||
      v->ilocw >= v->nrparm)
    return fail(OBIT_DFT_EBADARG, "grid apply: u, v, w offsets outside the random parameters");
  if (v->chanb < 0 || v->chane < v->chanb || v->chane >= v->nchan || v->IFb < 0 || v->IFe < v->IFb ||
      v->IFe >= v->nIF || v->stokb < 0 || v->stoke < v->stokb || v->stoke >= v->nstok)
    return fail(OBIT_DFT_EBADARG, "grid apply: bad channel, IF or polarization selection");
  if (v->incf <= 0 || v->incif <= 0 || v->incs <= 0 || v->kincf <= 0 || v->kincif <= 0)
    return fail(OBIT_DFT_EBADARG, "grid apply: bad increments");
  const long long last = (long long)v->nrparm +
                         3LL * ((long long)v->IFe * v->incif + (long long)v->chane * v->incf +
                                (long long)v->stoke * v->incs) + 2;
  if (last >= v->lenvis) return fail(OBIT_DFT_EBADARG, "grid apply: selection beyond the record length");
  const GridHostPlan& h = g->hp;
  GridApplyParams q = {};
  q.plane = g->d_plane;
  q.pitch = h.pitch;
  q.nxp = h.nxp;
  q.nyp = h.ny;
  q.crpix0 = h.crpix0;
  q.crpix1 = h.crpix1;
  q.cdelt0 = h.cdelt0;
  q.cdelt1 = h.cdelt1;
  q.table = g->d_table;
  q.exact = g->kernel == OBIT_DFT_GRID_KERNEL_EXACT;
  q.flip = h.flip;
  q.do3Dmul = h.do3Dmul;
  q.doRot = h.doRot;
  q.doPC = h.doPC;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) q.um[i * 3 + j] = h.umat[i][j];
  q.ccrot = h.ccrot;
  q.ssrot = h.ssrot;
  q.d0 = h.dxyzc[0];
  q.d1 = h.dxyzc[1];
  q.d2 = h.dxyzc[2];
  q.vis = d_vis;
  q.nvis = nvis;
  q.lrec = v->lenvis;
  q.nrparm = v->nrparm;
  q.ilocu = v->ilocu;
  q.ilocv = v->ilocv;
  q.ilocw = v->ilocw;
  q.fscale = v->freqScale;
  q.kincf = v->kincf;
  q.kincif = v->kincif;
  q.chanb = v->chanb;
  q.nchan = v->chane - v->chanb + 1;
  q.ifb = v->IFb;
  q.nif = v->IFe - v->IFb + 1;
  q.incf = 3 * v->incf;
  q.incif = 3 * v->incif;
  q.incs = 3 * v->incs;
  q.stokb = v->stokb;
  q.nstok = v->stoke - v->stokb + 1;
  q.op = opType;
  q.stokFactor = stokFactor;
  q.doFlip = doFlip ? 1 : 0;
  q.nsel = q.nchan * q.nif;
  q.nchunk = (q.nsel + 31) / 32;
  *p = q;
  return OBIT_DFT_OK;
}

// freqScale in host memory is copied (in order on `st`) to a device buffer of
// the field; device or managed memory is read in place.
int resolve_fscale(ObitDFTGrid* g, const GPUVisInfo* v, cudaStream_t st, GridApplyParams* q) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, v->freqScale) != cudaSuccess) {
    cudaGetLastError();
    at.type = cudaMemoryTypeUnregistered;
  }
  if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return OBIT_DFT_OK;
  const size_t n = (size_t)v->IFe * v->kincif + (size_t)v->chane * v->kincf + 1;
  if (n > g->fscaleCount) {
    cudaFree(g->d_fscale);
    g->d_fscale = nullptr;
    g->fscaleCount = 0;
    CUDA_TRY(cudaMalloc(&g->d_fscale, sizeof(float) * n));
    g->fscaleCount = n;
  }
  CUDA_TRY(cudaMemcpyAsync(g->d_fscale, v->freqScale, sizeof(float) * n, cudaMemcpyHostToDevice, st));
  q->fscale = g->d_fscale;
  return OBIT_DFT_OK;
}

int launch_apply(const GridApplyParams& q, cudaStream_t st) {
  if (q.nvis == 0) return OBIT_DFT_OK;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long items = (long long)q.nvis * q.nchunk;
  const long long want = (items + kApplyWarps - 1) / kApplyWarps;
  const int grid = (int)std::min<long long>(want, (long long)nsm * 8);
  grid_apply_kernel<<<grid, kApplyWarps * 32, 0, st>>>(q);
  CUDA_TRY(cudaGetLastError());
  return OBIT_DFT_OK;
}

void release(ObitDFTGrid* g) {
  if (!g) return;
  cudaFree(g->d_plane);
  cudaFree(g->d_table);
  cudaFree(g->d_stage);
  cudaFree(g->d_fscale);
  if (g->haveStreams) {
    for (cudaStream_t st : g->hs) cudaStreamDestroy(st);
    for (cudaEvent_t ev : g->hev) cudaEventDestroy(ev);
  }
  delete g;
}

}  // namespace

namespace {

// Pixels of an image model (ObitSkyModelLoadImage, ObitSkyModel.c:2163-2260)
// into the zeroed, quadrant-swapped grid of twice the image: blanked pixels
// and those below minFlux (or above 1e20) are zero (ObitFArrayClip, then the
// blank-skipping ObitFArrayShiftAdd and ObitFArrayDeblank of ObitFArrayPad,
// ObitFArray.c:3512-3530), the rest times factor, pixel (x, y) at grid cell
// (x, y) + n - n/2.
__global__ void grid_image_kernel(const float* __restrict__ pix, int n, float fblank, float minFlux,
                                  float factor, float* __restrict__ grid) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= n) return;
  float v = pix[(size_t)y * n + x];
  if (v == fblank || v < minFlux || v > 1.0e20f) v = 0.0f;
  else v = __fmul_rn(factor, v);
  const int N = 2 * n, off = n - n / 2;
  const int gx = (x + off + n) % N, gy = (y + off + n) % N;
  grid[(size_t)gy * N + gx] = v;
}

// Device half of a field's set-up: the grid (component cells, or image
// pixels when `pixels` is given), the FFT, the plane and the kernel table.
int build_field(ObitDFTGrid* g, const ObitDFTCCField* field, const float* pixels, float fblank, float minFlux,
                float factor, cudaStream_t st) {
  GridHostPlan& h = g->hp;
  float* d_grid = nullptr;
  float2* d_fft = nullptr;
  float* d_UU = nullptr;
  float* d_pix = nullptr;
  float* d_rows = nullptr;   // flux, dx, dy of the rows
  int* d_keys = nullptr;     // keys in, keys out, counters
  float* d_vals = nullptr;   // values in, values out
  void* d_sort = nullptr;
  cufftHandle plan = 0;
  bool havePlan = false;
  auto cleanup = [&]() {
    cudaFree(d_grid);
    cudaFree(d_fft);
    cudaFree(d_UU);
    cudaFree(d_pix);
    cudaFree(d_rows);
    cudaFree(d_keys);
    cudaFree(d_vals);
    cudaFree(d_sort);
    if (havePlan) cufftDestroy(plan);
  };
  auto bail = [&](int code, const std::string& msg) {
    cleanup();
    return fail(code, msg);
  };
  const size_t nh = (size_t)h.nx / 2 + 1;
  const size_t npix = pixels ? (size_t)(h.nx / 2) * (h.nx / 2) : 0;
  const int nrow = pixels ? 0 : h.rowsDesc.count;
  size_t sortBytes = 0;
  cudaError_t e;
  if (nrow > 0 && cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, (const int*)nullptr, (int*)nullptr,
                                                  (const float*)nullptr, (float*)nullptr, nrow, 0, 31, st) !=
                      cudaSuccess)
    return bail(OBIT_DFT_ECUDA, "grid create: sort sizing failed");
  if ((e = cudaMalloc(&g->d_plane, sizeof(float2) * (size_t)h.rows * h.pitch)) != cudaSuccess ||
      (e = cudaMalloc(&g->d_table, sizeof(float) * h.table.size())) != cudaSuccess ||
      (e = cudaMalloc(&d_grid, sizeof(float) * (size_t)h.nx * h.ny)) != cudaSuccess ||
      (e = cudaMalloc(&d_fft, sizeof(float2) * nh * h.ny)) != cudaSuccess ||
      (e = cudaMalloc(&d_UU, sizeof(float) * std::max<size_t>(1, h.UU.size()))) != cudaSuccess ||
      (pixels && (e = cudaMalloc(&d_pix, sizeof(float) * npix)) != cudaSuccess) ||
      (nrow && (e = cudaMalloc(&d_rows, sizeof(float) * 3 * (size_t)nrow)) != cudaSuccess) ||
      (nrow && (e = cudaMalloc(&d_keys, sizeof(int) * (2 * (size_t)nrow + 2))) != cudaSuccess) ||
      (nrow && (e = cudaMalloc(&d_vals, sizeof(float) * 2 * (size_t)nrow)) != cudaSuccess) ||
      (nrow && (e = cudaMalloc(&d_sort, std::max<size_t>(16, sortBytes))) != cudaSuccess))
    return bail(OBIT_DFT_ECUDA, std::string("grid create: cudaMalloc: ") + cudaGetErrorString(e));
  const size_t r0 = (size_t)h.rowsDesc.first;
  if ((e = cudaMemcpyAsync(g->d_table, h.table.data(), sizeof(float) * h.table.size(), cudaMemcpyHostToDevice,
                           st)) != cudaSuccess ||
      (!h.UU.empty() && (e = cudaMemcpyAsync(d_UU, h.UU.data(), sizeof(float) * h.UU.size(),
                                             cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
      (pixels && (e = cudaMemcpyAsync(d_pix, pixels, sizeof(float) * npix, cudaMemcpyDefault, st)) !=
                     cudaSuccess) ||
      (nrow && (e = cudaMemcpyAsync(d_rows, field->flux + r0, sizeof(float) * nrow, cudaMemcpyDefault, st)) !=
                   cudaSuccess) ||
      (nrow && (e = cudaMemcpyAsync(d_rows + nrow, field->deltaX + r0, sizeof(float) * nrow, cudaMemcpyDefault,
                                    st)) != cudaSuccess) ||
      (nrow && (e = cudaMemcpyAsync(d_rows + 2 * (size_t)nrow, field->deltaY + r0, sizeof(float) * nrow,
                                    cudaMemcpyDefault, st)) != cudaSuccess) ||
      (nrow && (e = cudaMemsetAsync(d_keys + 2 * (size_t)nrow, 0, 2 * sizeof(int), st)) != cudaSuccess) ||
      (e = cudaMemsetAsync(d_grid, 0, sizeof(float) * (size_t)h.nx * h.ny, st)) != cudaSuccess)
    return bail(OBIT_DFT_ECUDA, std::string("grid create: copy: ") + cudaGetErrorString(e));
  if (pixels) {
    const int n = h.nx / 2;
    grid_image_kernel<<<dim3((unsigned)((n + 255) / 256), (unsigned)n), 256, 0, st>>>(d_pix, n, fblank, minFlux,
                                                                                    factor, d_grid);
  } else if (nrow) {
    RowGridParams rp;
    rp.flux = d_rows;
    rp.dx = d_rows + nrow;
    rp.dy = d_rows + 2 * (size_t)nrow;
    rp.n = nrow;
    rp.r = h.rowsDesc;
    rp.keys = d_keys;
    rp.vals = d_vals;
    rp.counters = d_keys + 2 * (size_t)nrow;
    grid_rows_kernel<<<(unsigned)((nrow + 255) / 256), 256, 0, st>>>(rp);
    if ((e = cudaGetLastError()) != cudaSuccess)
      return bail(OBIT_DFT_ECUDA, std::string("grid rows: ") + cudaGetErrorString(e));
    // stable radix sort by cell: each cell's rows stay in row order
    if (cub::DeviceRadixSort::SortPairs(d_sort, sortBytes, d_keys, d_keys + nrow, d_vals, d_vals + nrow, nrow, 0,
                                        31, st) != cudaSuccess)
      return bail(OBIT_DFT_ECUDA, "grid create: sort failed");
    grid_cells_kernel<<<(unsigned)((nrow + 255) / 256), 256, 0, st>>>(d_keys + nrow, d_vals + nrow, nrow, d_grid);
  }
  if ((e = cudaGetLastError()) != cudaSuccess)
    return bail(OBIT_DFT_ECUDA, std::string("grid fill: ") + cudaGetErrorString(e));
  if (nrow) {
    int counters[2] = {0, 0};
    if ((e = cudaMemcpyAsync(counters, d_keys + 2 * (size_t)nrow, sizeof(counters), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return bail(OBIT_DFT_ECUDA, std::string("grid create: ") + cudaGetErrorString(e));
    h.ncomp = counters[0];
    h.bad = counters[1];
    if (h.ncomp == 0) {  // nothing gridded: the reference skips the field
      cleanup();
      cudaFree(g->d_plane);
      cudaFree(g->d_table);
      g->d_plane = nullptr;
      g->d_table = nullptr;
      return OBIT_DFT_OK;
    }
  }
  // ObitSkyModelFTImage: forward real-to-half-complex transform, unnormalized
  if (cufftPlan2d(&plan, h.ny, h.nx, CUFFT_R2C) != CUFFT_SUCCESS)
    return bail(OBIT_DFT_ECUDA, "grid create: cufftPlan2d failed");
  havePlan = true;
  if (cufftSetStream(plan, st) != CUFFT_SUCCESS ||
      cufftExecR2C(plan, d_grid, reinterpret_cast<cufftComplex*>(d_fft)) != CUFFT_SUCCESS)
    return bail(OBIT_DFT_ECUDA, "grid create: cufftExecR2C failed");
  PlaneParams pp;
  pp.fft = d_fft;
  pp.plane = g->d_plane;
  pp.nx = h.nx;
  pp.ny = h.ny;
  pp.pitch = h.pitch;
  pp.nxp = h.nxp;
  pp.doGaus = h.doGaus;
  pp.b1 = h.b1;
  pp.b2 = h.b2;
  pp.b3 = h.b3;
  pp.dV = h.dV;
  pp.UU = d_UU;
  grid_plane_kernel<<<dim3((unsigned)((h.pitch + 255) / 256), (unsigned)h.rows), 256, 0, st>>>(pp);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return bail(OBIT_DFT_ECUDA, std::string("grid plane: ") + cudaGetErrorString(e));
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
    return bail(OBIT_DFT_ECUDA, std::string("grid create: ") + cudaGetErrorString(e));
  cleanup();
  return OBIT_DFT_OK;
}

int new_field(int kernel, ObitDFTGrid** out, ObitDFTGrid** g) {
  if (!out) return fail(OBIT_DFT_EBADARG, "grid create: null output");
  *out = nullptr;
  if (kernel != OBIT_DFT_GRID_KERNEL_REFERENCE && kernel != OBIT_DFT_GRID_KERNEL_EXACT)
    return fail(OBIT_DFT_EBADARG, "grid create: unknown kernel");
  *g = new ObitDFTGrid();
  (*g)->kernel = kernel;
  return OBIT_DFT_OK;
}

}  // namespace

extern "C" int obit_dft_grid_create(const ObitDFTCCField* field, const ObitDFTGridImage* image,
                                    const ObitDFTCCModel* model, float maxGrid, int kernel, void* stream,
                                    ObitDFTGrid** out) {
  ObitDFTGrid* g = nullptr;
  int rc = new_field(kernel, out, &g);
  if (rc) return rc;
  rc = obit::grid_host_plan(field, image, model, maxGrid, &g->hp);
  if (!rc && cudaGetDevice(&g->device) != cudaSuccess) rc = fail(OBIT_DFT_ECUDA, "grid create: no device");
  if (!rc && g->hp.rowsDesc.count > 0)  // no rows: nothing gridded, the reference skips the field
    rc = build_field(g, field, nullptr, 0.0f, 0.0f, 1.0f, (cudaStream_t)stream);
  if (rc) {
    release(g);
    return rc;
  }
  *out = g;
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_grid_create_image(const float* pixels, float fblank, const ObitDFTCCField* field,
                                          const ObitDFTGridImage* image, const ObitDFTCCModel* model, int kernel,
                                          void* stream, ObitDFTGrid** out) {
  if (!pixels) return fail(OBIT_DFT_EBADARG, "grid create: null image");
  ObitDFTGrid* g = nullptr;
  int rc = new_field(kernel, out, &g);
  if (rc) return rc;
  rc = obit::grid_host_plan_image(field, image, model, &g->hp);
  if (!rc && cudaGetDevice(&g->device) != cudaSuccess) rc = fail(OBIT_DFT_ECUDA, "grid create: no device");
  if (!rc) rc = build_field(g, field, pixels, fblank, model->minFlux, model->factor, (cudaStream_t)stream);
  if (rc) {
    release(g);
    return rc;
  }
  *out = g;
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_grid_apply(ObitDFTGrid* g, const GPUVisInfo* visInfo, int opType, float stokFactor,
                                   int doFlip, float* d_vis, int nvis, void* stream) {
  if (!g) return fail(OBIT_DFT_EBADARG, "grid apply: null field");
  GridApplyParams q;
  int rc = apply_params(g, visInfo, opType, stokFactor, doFlip, d_vis, nvis, &q);
  if (rc) return rc;
  if (g->hp.ncomp == 0 || nvis == 0) return OBIT_DFT_OK;
  CUDA_TRY(cudaSetDevice(g->device));
  rc = resolve_fscale(g, visInfo, (cudaStream_t)stream, &q);
  if (rc) return rc;
  return launch_apply(q, (cudaStream_t)stream);
}

extern "C" int obit_dft_grid_apply_host(ObitDFTGrid* g, const GPUVisInfo* visInfo, int opType,
                                        float stokFactor, int doFlip, float* h_vis, int nvis, void* stream) {
  if (!g) return fail(OBIT_DFT_EBADARG, "grid apply: null field");
  if (nvis > 0 && !h_vis) return fail(OBIT_DFT_EBADARG, "grid apply: null records");
  if (!visInfo) return fail(OBIT_DFT_EBADARG, "grid apply: null GPUVisInfo");
  if (nvis == 0 || g->hp.ncomp == 0) return OBIT_DFT_OK;
  CUDA_TRY(cudaSetDevice(g->device));
  const size_t lrec = (size_t)std::max(1, visInfo->lenvis);
  // chunks of about 64 MB, round-robin over the streams, each stream reusing
  // its own staging slot in order: the upload of one chunk, the kernel of
  // another and the download of a third overlap (pinned records), and the
  // device holds S chunks whatever the size of the host buffer
  constexpr int S = ObitDFTGrid::kHostStreams;
  const int per = (int)std::max<size_t>(1, std::min<size_t>((size_t)nvis, (64u << 20) / (sizeof(float) * lrec)));
  const size_t slot = (size_t)per * lrec;
  const size_t bytes = sizeof(float) * slot * (size_t)std::min(S, (nvis + per - 1) / per);
  if (bytes > g->stageBytes) {
    cudaFree(g->d_stage);
    g->d_stage = nullptr;
    g->stageBytes = 0;
    CUDA_TRY(cudaMalloc(&g->d_stage, bytes));
    g->stageBytes = bytes;
  }
  GridApplyParams q;
  int rc = apply_params(g, visInfo, opType, stokFactor, doFlip, g->d_stage, nvis, &q);
  if (rc) return rc;
  if (!g->haveStreams) {
    for (cudaStream_t& hs : g->hs) CUDA_TRY(cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking));
    for (cudaEvent_t& ev : g->hev) CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    g->haveStreams = true;
  }
  cudaStream_t st = (cudaStream_t)stream;
  rc = resolve_fscale(g, visInfo, st, &q);
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(g->hev[S], st));
  for (int i = 0; i < S; i++) CUDA_TRY(cudaStreamWaitEvent(g->hs[i], g->hev[S], 0));
  int k = 0;
  for (int r0 = 0; r0 < nvis; r0 += per, k++) {
    const int n = std::min(per, nvis - r0);
    cudaStream_t cs = g->hs[k % S];
    float* dv = g->d_stage + (size_t)(k % S) * slot;
    const size_t cb = sizeof(float) * (size_t)n * lrec;
    CUDA_TRY(cudaMemcpyAsync(dv, h_vis + (size_t)r0 * lrec, cb, cudaMemcpyHostToDevice, cs));
    GridApplyParams qc = q;
    qc.vis = dv;
    qc.nvis = n;
    rc = launch_apply(qc, cs);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(h_vis + (size_t)r0 * lrec, dv, cb, cudaMemcpyDeviceToHost, cs));
  }
  for (int i = 0; i < S; i++) {
    CUDA_TRY(cudaEventRecord(g->hev[i], g->hs[i]));
    CUDA_TRY(cudaStreamWaitEvent(st, g->hev[i], 0));
  }
  CUDA_TRY(cudaStreamSynchronize(st));
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_grid_info(const ObitDFTGrid* g, long long* info, int n) {
  if (!g || !info) return fail(OBIT_DFT_EBADARG, "grid info: null argument");
  const GridHostPlan& h = g->hp;
  const long long v[10] = {h.ncomp, h.bad, h.nx, h.ny, h.nxp, h.doGaus, h.do3Dmul, h.doPC, h.doRot, g->kernel};
  for (int i = 0; i < n && i < 10; i++) info[i] = v[i];
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_grid_plane(const ObitDFTGrid* g, float* h_plane, long long capacity) {
  if (!g || !h_plane) return fail(OBIT_DFT_EBADARG, "grid plane: null argument");
  const GridHostPlan& h = g->hp;
  if (!g->d_plane) return fail(OBIT_DFT_EBADARG, "grid plane: the field has no components");
  if (capacity < 2LL * h.nxp * h.ny) return fail(OBIT_DFT_EBADARG, "grid plane: buffer too small");
  CUDA_TRY(cudaSetDevice(g->device));
  CUDA_TRY(cudaMemcpy2D(h_plane, sizeof(float2) * h.nxp, g->d_plane, sizeof(float2) * h.pitch,
                        sizeof(float2) * h.nxp, h.ny, cudaMemcpyDeviceToHost));
  return OBIT_DFT_OK;
}

extern "C" int obit_dft_grid_destroy(ObitDFTGrid* g) {
  if (!g) return OBIT_DFT_OK;
  cudaSetDevice(g->device);
  release(g);
  return OBIT_DFT_OK;
}
