// Beam-corrected DFT (linear feeds; Stokes I, Q, U or V sky): the model of
// ObitCUDABeamModel's beam*Kernel family (ObitCUDABeamModel.cu:139-1226) with
// the Jones products of cudaJonesCor1_Lin_{I,Q,U,V} (CUDALinCorSum.h:104-455).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "dft_types.h"

namespace obit {

// Channels per block of the beam recurrence kernel.
constexpr int kBeamK = 8;

// Tensor-core form: records per CTA item (one per warp), channels per matrix
// tile (the 16 rows of an m16n8k8 product) and tiles per run.
constexpr int kBeamMmaWarps = 8;
constexpr int kBeamMmaRows = 16;
constexpr int kBeamMmaTiles = 16;
constexpr int kBeamMmaMaxChan = kBeamMmaRows * kBeamMmaTiles;

// A run of uniformly spaced channels of one IF within one Jones plane (at most
// kBeamMmaMaxChan): channel k has frequency ratio f0 + k df (df: increment
// class dfc of KParams), table index ifq0 + k kincf and record offset
// off0 + k incf.
struct BeamSeg {
  float f0_hi, f0_lo;
  int dfc;
  int off0;
  int ifq0;
  int nch;
  int jplane;
  int pad;
};

struct BeamKParams {
  // Records, layout, channel blocks (at most kBeamK channels, never spanning a
  // change of Jones plane), tile shape R x Bt, component table and tile ct,
  // error flag: the fields the DFT kernels use, same meaning.
  KParams k;
  int ilocb, iloca1, iloca2;     // BASELINE offset, or ANTENNA1 / ANTENNA2 (ilocb < 0)
  int ncorr;                     // modelled correlations of XX, YY, XY, YX (1, 2 or 4)
  float polFact[4];              // per record correlation
  // per-channel form (the plain comparator): selection and tables
  int nrparm, chanb, nchanSel, ifb, nifSel, kincf, kincif, incif;
  const double* fscale;          // device, per (channel, IF) table index: nu / nu_uvref
  const double* lnspec;          // device or null: log-frequency term per table index
  const int* plane;              // device or null: tabulated-spectrum plane per table index
  const int* jchan;              // device: Jones plane per table index
  const int* antType;            // device: antenna type per antenna (0-rel)
  int numAnt, numAntType, numJChan;
  const float* jones;            // device: [type][component][plane] x 8 floats (XX, XY, YX, YY)
  int jonesComps;                // components per type in the Jones table (>= ncomp)
  int mode;                      // ModelKind
  int stokType;                  // sky Stokes: 1 I, 2 Q, 3 U, 4 V
  int circular;                  // 1: circular feeds (RR, LL, RL, LR), 0: linear
  float c2p, s2p;                // cos, sin of twice the parallactic angle (linear Q, U)
  int flavor;                    // kFlavorRecur (blocks) or kFlavorPlain (one thread per channel)
  // tensor-core form (uniformly spaced channels): runs of
  // channels, their count, and 1 to launch it instead of the block form
  const BeamSeg* segs;
  int nseg;
  int mma;
  // coefficient fragments of the tensor-core form, written by its prologue:
  // [plane][type pair][component group of 4][column 8][component in group 4]
  // float4 {b0 hi, b1 hi, b0 lo, b1 lo}; ncompPad components per (plane, pair),
  // a multiple of the component tile, zero past the model
  float4* coefTab;
  int ncompPad;
  // spectral amplitudes of the tensor-core form (families with a spectrum),
  // written by its prologue: [run][component group of 4][matrix
  // tile 16][lane group 8][component in group 4] float2 {A(16 m + g),
  // A(16 m + g + 8)}, zero past the run and the model
  float2* ampTab;
};

// Correlation slots the recurrence kernel accumulates: XX and YY, or all four.
inline int beam_nq(const BeamKParams& p) { return p.ncorr > 2 ? 4 : 2; }

// Dynamic shared memory of a launch with component tile p.k.ct.
size_t beam_smem_bytes(const BeamKParams& p);

// Largest component tile (<= 128, a multiple of 8) whose shared memory fits
// one CTA per SM; sets p->k.ct.  Returns 0 or an error code with err.
int beam_fit_tile(BeamKParams* p, std::string* err);

// One launch over all records of kp (stream-ordered, asynchronous).  The
// tensor-core form runs its prologues first unless `prologue` is false (the
// caller ran launch_beam_prologue for this call and ordered the stream after
// it).
int launch_beam(const BeamKParams& kp, cudaStream_t stream, std::string* err, bool prologue = true);

// Tensor-core form.  Whether the model family has it; the bytes of its
// coefficient-fragment and amplitude tables (p.ncompPad, p.nseg set; no
// amplitude table for models without a spectrum); the dynamic shared memory of a
// launch with component tile p.k.ct; the largest tile (<= 128, a multiple of 4)
// that fits one CTA per SM, set in p->k.ct (0 when none fits: the caller keeps
// the block form); the launch (the prologue kernels, then the kernel).
bool beam_mma_supported(int mode);
size_t beam_mma_coef_bytes(const BeamKParams& p);
size_t beam_mma_amp_bytes(const BeamKParams& p);
size_t beam_mma_smem_bytes(const BeamKParams& p);
int beam_mma_fit_tile(BeamKParams* p);
int launch_beam_mma(const BeamKParams& kp, cudaStream_t stream, std::string* err, bool prologue = true);
// The tensor-core form's prologues alone (the coefficient fragments and the
// spectral amplitudes), for callers that launch the kernel on several streams.
int launch_beam_prologue(const BeamKParams& kp, cudaStream_t stream, std::string* err);

}  // namespace obit
