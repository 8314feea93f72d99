// Types shared by the DFT kernels (device) and the planner (host, plain C++):
// limits, model and operation kinds, the channel-block descriptor, the kernel
// parameter block and the shared-memory layout sizes.
#pragma once
#include <stddef.h>

#ifdef __CUDACC__
#define OBIT_HD __host__ __device__
#else
#define OBIT_HD
#endif

namespace obit {

constexpr int kThreads = 256;  // default CTA size
constexpr int kMaxNTerm = 4;   // spectral terms supported (ObitSkyModel nSpecTerm)
constexpr int kMaxDf = 8;      // distinct channel increments per launch
constexpr int kMaxPol = 4;
constexpr int kMaxBt = 32;     // blocks per tile (R >= 8)
constexpr int kDefaultWaitPolls = 1 << 22;  // bulk-copy wait before the timeout path

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
  int Bt, R;        // tile shape: blocks per tile, rows per tile (Bt * R == CTA size)
  int nBlockTiles;  // ceil(nblocks / Bt)
  int ndf;
  float df_hi[kMaxDf], df_lo[kMaxDf];
  const float* comps;  // ncomp records of cstride floats (reference field order)
  const float* compsLo;  // optional ncomp x 4 floats: low parts of X, Y, Z (FP64
                         // positions; fields 1-3 of comps hold the high parts)
  int ncomp, cstride, ct, nterm;
  // Mixed instances only: the untapered components of a Gaussian-family model
  // as a point-family sub-table (same stride, ordered by spectral index)
  const float* compsPt;
  int ncompPt;
  int nspec;           // planes (tabulated spectra)
  int rowBase;         // first row index of this launch within vis
  int* errFlag;        // set non-zero on an internal error (never traps)
  int waitPolls;       // polls of a component-tile copy before the timeout path
};

// A batched launch over many facets (one KParams each, same tile shape and
// model family): items [itemStart[f], itemStart[f + 1]) belong to facet f.
struct BatchParams {
  const KParams* facets;  // device array of nfacet parameter blocks
  const int* itemStart;   // device array of nfacet + 1 cumulative item counts
  int nfacet;
  int* counter;           // device work counter, zero at launch
};

// Point models (no per-channel amplitude factor) with K a multiple of 8 take
// the factored recurrence: channel k = 8a + b of a block gets
// G_b * H_a, G_b = A z0 s^b and H_a = s^(8a), so each evaluation is one
// packed complex multiply-accumulate.
OBIT_HD constexpr inline bool point_factored(int mode, int K) { return mode == kPoint && K >= 8 && K % 8 == 0; }

// Point models with one spectral index (PointSpec with one term, PointTSpec)
// take the same factored form when the planner allows it (spectral-factored
// instances): amplitude A exp(e0 + e1 k + e2 k^2) over a block; the linear part
// rides on a non-unit step w = s exp(e1), the quadratic part is split into the
// tile's common exp(alpha_t l2 k^2), applied per channel when the tile's sums
// are folded, and a residual (alpha - alpha_t) l2 k^2 replaced by its minimax
// line over the block.  alpha_t is the midpoint of the tile's first and last
// spectral index: the component table is ordered by spectral index, so the
// components of a tile have nearly equal indices and the residual is tiny.
OBIT_HD constexpr inline bool spec_factorable(int mode, int K) {
  return (mode == kPointSpec || mode == kPointTSpec) && K >= 8 && K % 8 == 0;
}
// Field of the spectral index: PointSpec's first term, PointTSpec's alpha
// (ObitSkyModel.c:2044-2063, ObitSkyModelMF.c:1497-1514).
constexpr int kSpecIndexField = 4;

//--------------------------------------------------------------------------
// Shared memory per CTA of the recurrence kernel (dynamic):
//   comps  : ct * cstride floats (component tile, zero-filled past ncomp)
//   uvw    : R * 3 floats (padded to a multiple of 4)
//   blk    : Bt BlockDesc (this tile's channel blocks)
//   P      : ct * R float2            (phase turns, split-FP32)
//   S      : ndf * ct * R float4      (step s and s^(K/4); s and s^4 when factored)
//   T      : ndf * ct * R float2      (s^8, factored point models)
//   Q      : ct * R floats            (Gaussian form, Gaussian models)
//   G      : ct * Bt * 4 * (max(K/4, 1) + 1) floats (spectral amplitudes, point
//            families with a spectrum: 16-byte entries, one padding entry per row)
//            Spectral-factored instances instead: F, ct * Bt float4 (amplitude
//            at the block's first channel, exp(e1), exp(4 e1), exp(8 e1)), and
//            Phi, Bt * K floats (the tile's per-channel exp(alpha_t l2 k^2))
//   Cmp    : 2 * K * R * Bt floats    (Kahan compensation of the totals, factored
//            point models: K/2 re and K/2 im pairs per thread, thread-minor)
//   lo     : ct * 4 floats            (low parts of X, Y, Z: instances for FP64
//            positions; reserved in every plan so that one plan serves both)
// The model stage of the epilogue (R * Bt * K float2) reuses the same space.
//--------------------------------------------------------------------------
OBIT_HD inline size_t smem_floats_main(int R, int Bt, int K, int ct, int cstride, int ndf, bool gauss,
                                       bool table, bool factored = false, bool fspec = false) {
  size_t n = (size_t)ct * cstride + 4 * (size_t)ct + (size_t)((R * 3 + 3) & ~3) +
             (size_t)Bt * (sizeof(BlockDesc) / 4) + 2 * (size_t)ct * R + 4 * (size_t)ndf * ct * R;
  if (gauss) n += (size_t)ct * R;
  if (fspec) n += (size_t)ct * Bt * 4 + (size_t)Bt * K;
  else if (table) n += (size_t)ct * Bt * 4 * ((K >= 4 ? K / 4 : 1) + 1);
  if (factored) n += 2 * (size_t)ndf * ct * R + 2 * (size_t)K * R * Bt;
  return n;
}
OBIT_HD inline size_t smem_floats_stage(int R, int Bt, int K) { return (size_t)R * Bt * K * 2; }

}  // namespace obit
