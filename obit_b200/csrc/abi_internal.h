// Internal helpers shared by the C-ABI entry points (obit_dft_capi.cu,
// obit_dft_static.cu): translation of the reference-layout descriptors
// (GPUVisInfo, GPUModelInfo) plus the optional FP64 frequency side table and
// CPU polarization rules into the planner's descriptions, and the padded copy
// of a component table.
#pragma once
#include <cuda_runtime_api.h>

#include <string>
#include <vector>

#include "dft_plan.h"
#include "obit_dft.h"

namespace obit {

// FP64 channel frequencies supplied with obit_dft_set_freq.
struct FreqSide {
  bool have = false;
  std::vector<double> freqArr, specFreq;
  double uvRef = 0.0, modelRef = 0.0;
};

// The reference CPU DFT's polarization rules (obit_dft_set_poln).
struct PolnRules {
  bool cpuRules = false;
  float stokFactor = 1.0f;
  int doFlip = 0;
};

// Model description taken from GPUModelInfo.
struct ModelCfg {
  ModelDesc model;
  int opType = 0, doSwap = 0;
  float stokFact[4] = {1.f, 1.f, 1.f, 1.f};
  std::vector<int> specIndex;  // coarse plane per (channel, IF), tabulated spectra
};

// GPUModelInfo -> ModelCfg.  ncomp/lcomp give the component count and record
// length (the caller resolves GPUInfo.nmodel / modelSize); validates the
// record length for the type; copies specIndex (host pointer, else device).
// A device specIndex is read with a blocking copy on the legacy default stream,
// or, when `order` is given, on that stream (then synchronized), so that the
// read follows work the caller queued there.
int model_from_info(const GPUModelInfo* m, int ncomp, int lcomp, const GPUVisInfo* v, ModelCfg* mc,
                    std::string* err, const cudaStream_t* order = nullptr);

// GPUVisInfo (+ FP64 side table) -> LayoutDesc, including the frequency ratio
// and log-frequency tables; reads the FP32 freqScale from the device when no
// FP64 table is set (on the legacy default stream, or on *order as above).
int layout_from_info(const GPUVisInfo* v, const ModelCfg& mc, const FreqSide& fs, LayoutDesc* L,
                     std::string* err, const cudaStream_t* order = nullptr);

// Operation and polarization handling.
int apply_from_info(const ModelCfg& mc, const PolnRules& pr, const LayoutDesc& L, ApplyDesc* A,
                    std::string* err);

// Padded copy (rows of comp_stride floats, zero-filled) of a device component
// table of md.ncomp rows of md.lcomp floats, ordered on `stream`.
int copy_comps(float* dst, const float* src, const ModelDesc& md, cudaStream_t stream,
               std::string* err);

// Status of a kernel error flag read back by the host (0: none).  Codes:
// 2 a component-tile copy did not land within the wait limit (the CTA left
// after its copy landed: the context stays usable, OBIT_DFT_EKERNEL);
// 3 a record's antenna number outside the beam's antenna table (EKERNEL);
// 5 a copy was still in flight after the second wait window when the CTA left:
// the CUDA context must be treated as unusable (OBIT_DFT_ECUDA).
int kernel_flag_status(int flag, std::string* msg);

// Thread-local last-error message of the C ABI.
void set_last_error(const std::string& msg);
const char* last_error();

}  // namespace obit
