// Host-side planning for the DFT kernels: channel blocks, tile shape, shared
// memory (plan_layout, plain C++ in dft_planner.cpp), and the device side of a
// plan and the launch (dft_plan.cu).  No torch types.
#pragma once
#include <cuda_runtime_api.h>

#include <string>
#include <vector>

#include "dft_types.h"

namespace obit {

// Everything the planner needs to describe one visibility layout + model.
struct LayoutDesc {
  int lrec = 0, nrparm = 0, ilocu = 0, ilocv = 1, ilocw = 2;
  int nchan = 1, nif = 1, nstok = 1;
  int incs = 3, incf = 3, incif = 3;  // floats
  int kincf = 1, kincif = 1;          // frequency-table increments
  int chanb = 0, chane = 0;           // selected channels (0-rel, inclusive)
  int ifb = 0, ife = 0;               // selected IFs
  int stokb = 0, stoke = 0;           // selected polarizations
  std::vector<double> fscale;         // nu/nu_uvref per (chan, IF) table index
  std::vector<double> lnspec;         // Spec: ln(nu/nu_model); TSpec: ln(nu/nu_plane)
  std::vector<int> specIndex;         // TSpec plane per (chan, IF)
  std::vector<int> blockKey;          // optional, per (chan, IF): blocks never span a change
                                      // (the beam kernel's Jones plane)
};

struct ModelDesc {
  int kind = kPoint;  // ModelKind
  int nterm = 0;
  int lcomp = 4;      // floats per component in the source table
  int ncomp = 0;
  int nspec = 0;      // planes for tabulated spectra
  // Planning only (not kept by the plan): the spectral index of each component
  // in the order of the device table the kernel will read, or NULL.  Point
  // families with one spectral index may take the spectral-factored kernel only
  // when it is given (the table must be ordered by it; see spec_factorable).
  const float* specIndex = nullptr;
  // Mixed Gaussian models (Gaussian family with one spectral index): the
  // first ncompPt rows of the device table are its untapered components in the
  // matching point family's field order (same stride, ordered by spectral
  // index, which specIndex then lists); the ncomp rows after them are the
  // Gaussian components.  0: an ordinary table.
  int ncompPt = 0;
};

// Bound on the per-term relative amplitude error of the spectral-factored form
// (|alpha - alpha_tile| |l2| n^2 / 8 over every tile and block); plans above it
// keep the chain form.  A tenth of the 1e-5 parity bound (relative to the sum
// of |A|); 20,000 indices over [-1.5, 0.5] in 128-component tiles with 1 MHz
// channels at 1.4 GHz give 2e-7.
constexpr double kSpecResidualTol = 1e-6;

struct ApplyDesc {
  int op = kOpSub;
  int flipMask = 0;
  int cumulative = 1;
  float stokFactor = 1.0f;
  float polFact[kMaxPol] = {1.f, 1.f, 1.f, 1.f};
};

struct TuneDesc {
  int flavor = kFlavorRecur;
  int K = 0;    // channels per thread; 0 = chosen by the planner
  int ct = 0;   // components per shared-memory tile (shrunk to fit shared memory); 0 = planner's
               // choice: 160 where it fits shared memory (and the spectral-factored bound)
               // as it is, else 128 shrunk to fit
  int Bt = 0;   // blocks per tile (power of two); 0 = chosen by the planner
  int threads = 0;  // CTA size, 128 or 256; 0 = chosen by the planner
  int specFactor = 1;  // 0: point families with a spectrum keep the chain form
};

// A compiled plan: block table on the device plus the fixed kernel fields.
struct Plan {
  KParams kp{};                    // vis / nvis / rowBase / comps filled at launch
  std::vector<BlockDesc> blocks;   // host copy
  BlockDesc* d_blocks = nullptr;   // device copy (owned)
  size_t smemBytes = 0;
  int threads = 256;               // CTA size
  int gridCap = 0;                 // CTAs resident across the device
  TuneDesc tune;
  ModelDesc model;
  bool specFactored = false;       // spectral-factored instance (spec_factorable)
  bool mixed = false;              // mixed instance (ModelDesc.ncompPt > 0)
  bool linear = true;              // every block has a uniform channel increment
  double maxNonLin = 0.0;          // largest deviation from a linear frequency run
};

// Padded component stride (floats): multiple of 4 so tiles are 16-byte aligned.
int comp_stride(const ModelDesc& m);

// Host part of planning: validate, cut the selected channels into blocks,
// choose channels per thread, tile shape and component tile.  Fills
// plan->blocks and every KParams field except the pointers and row range.
// No CUDA calls.  Returns 0, an error code (3) with a message in err, or 4
// when a mixed table (ModelDesc.ncompPt > 0) cannot run mixed on this layout
// (blocks too short for the factored form, or the point rows fail the
// residual bound): the caller then plans the unsplit table.
int plan_layout(const LayoutDesc& L, const ModelDesc& M, const ApplyDesc& A, const TuneDesc& T,
                Plan* plan, std::string* err);

// Whether a kernel instantiation exists for (flavor, K).
bool kernel_exists(int flavor, int K);

// Build the plan: plan_layout plus the device block table and launch limits.
// Returns 0 or an error code with a message in err.
int build_plan(const LayoutDesc& L, const ModelDesc& M, const ApplyDesc& A, const TuneDesc& T,
               Plan* plan, std::string* err);
// Device side of a laid-out plan: kernel attributes, launch limits and the
// block table, copied on `stream` into dst (a device buffer of at least
// kp.nblocks descriptors) or, when dst is NULL, into a table allocated here
// and owned by the plan.
int finalize_plan(Plan* plan, BlockDesc* dst, cudaStream_t stream, std::string* err);
void free_plan(Plan* plan);

// Launch on `stream` over rows [rowBase, rowBase + nvis) of d_vis.
int launch_plan(const Plan& plan, float* d_vis, int rowBase, int nvis, const float* d_comps,
                int* d_err, cudaStream_t stream, std::string* err);

// Supported channel-block lengths.
bool valid_K(int K);

// Raise (never lower) kernel fn's dynamic shared-memory limit on the current
// device to at least `bytes`; the limit is shared by every plan of fn.
int raise_smem_limit(const void* fn, size_t bytes, std::string* err);

// Batched recurrence kernel (dft_batch_kernels.cu): whether K is instantiated;
// set the shared-memory attribute and report the resident CTAs across the
// device; launch `grid` persistent CTAs over the batch on `stream`.
bool batch_kernel_exists(int K);
int batch_prepare(int K, int mode, int threads, size_t smemBytes, int* gridCap, std::string* err);
int launch_batch(int K, int mode, const BatchParams& bp, int grid, int threads, size_t smemBytes,
                 cudaStream_t stream, std::string* err);

}  // namespace obit
