// Beam-corrected DFT (Stokes I, linear feeds): the model of ObitCUDABeamModel's
// beam*Kernel family (ObitCUDABeamModel.cu:139-1226) with the Jones product of
// cudaJonesCor1_Lin_I (CUDALinCorSum.h:104-134).
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace obit {

struct BeamKParams {
  float* vis;                    // device records, nvis x lrec floats
  int nvis, lrec, nrparm, ilocu, ilocv, ilocw;
  int ilocb, iloca1, iloca2;     // BASELINE offset, or ANTENNA1 / ANTENNA2 (ilocb < 0)
  int incs, incf, incif;         // float increments between correlations, channels, IFs
  int ncorr;                     // modelled correlations of XX, YY, XY, YX (1, 2 or 4)
  int op;                        // OpKind
  float polFact[4];              // per record correlation
  int chanb, nchanSel, ifb, nifSel, kincf, kincif;  // selection and table increments
  const double* fscale;          // device, per (channel, IF) table index: nu / nu_uvref
  const double* lnspec;          // device or null: log-frequency term per table index
  const int* plane;              // device or null: tabulated-spectrum plane per table index
  const int* jchan;              // device: Jones plane per table index
  const int* antType;            // device: antenna type per antenna (0-rel)
  int numAnt, numAntType, numJChan;
  const float* jones;            // device: [type][component][plane] x 8 floats (XX, XY, YX, YY)
  int jonesComps;                // components per type in the Jones table (>= ncomp)
  const float* comps;            // device: ncomp records of cstride floats
  int ncomp, cstride, ct, nterm, mode;
  int* errFlag;                  // set to 3 for a record whose antennas are outside the table
  int stokType;                  // sky Stokes: 1 I, 2 Q, 3 U, 4 V
  float c2p, s2p;                // cos, sin of twice the parallactic angle (Q, U)
};

// Shared memory of one launch: the component tile and its Jones coefficients
// for every (type, type) pair and plane, 8 floats each.
inline size_t beam_smem_bytes(const BeamKParams& p) {
  return sizeof(float) * ((size_t)p.ct * p.cstride + (size_t)p.numAntType * p.numAntType * p.ct * p.numJChan * 8);
}

// One launch over all records of kp (stream-ordered, asynchronous).
int launch_beam(const BeamKParams& kp, cudaStream_t stream, std::string* err);

}  // namespace obit
