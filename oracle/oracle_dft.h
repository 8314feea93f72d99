/*
 * Test infrastructure: CPU oracles for the Obit DFT sky-model predict/subtract.
 *
 * Nothing in the product links this header.  It describes one buffer of
 * Obit random-group visibility records plus a CLEAN-component table, the
 * same inputs ThreadSkyModelFTDFT reads from ObitSkyModel / ObitUVDesc
 * (ObitSystem/Obit/src/ObitSkyModel.c:2354-2857) and ThreadSkyModelMFFTDFT
 * reads from ObitSkyModelMF (ObitSystem/Obit/src/ObitSkyModelMF.c:1971-2440).
 *
 * Two implementations consume it:
 *   oracle_dft.c  (A) every FP32 input promoted to double; phase, sin/cos,
 *                     exp and the component sum in FP64.  Judge of max/RMS error.
 *   refcpu_dft.c  (B) the reference CPU loop restated with its FP32 phase
 *                     rounding, linked against the reference's own
 *                     ObitSinCosVec / ObitExpVec (built from the reference
 *                     sources into oracle/_ref/).  Timed CPU baseline.
 */
#ifndef OBIT_ORACLE_DFT_H
#define OBIT_ORACLE_DFT_H
#ifdef __cplusplus
extern "C" {
#endif

/* Component model types: numbering of GPUModType,
 * ObitSystem/Obit/include/ObitCUDASkyModelInfoDef.h:44-52. */
enum {
  ORACLE_POINT = 0,
  ORACLE_POINT_SPEC = 1,
  ORACLE_POINT_TSPEC = 2,
  ORACLE_GAUSS = 3,
  ORACLE_GAUSS_SPEC = 4,
  ORACLE_GAUSS_TSPEC = 5
};

typedef struct OracleJob {
  /* visibility record geometry (ObitUVDesc: lrec, nrparm, ilocu/v/w) */
  int nvis, lrec, nrparm, ilocu, ilocv, ilocw;
  /* increments between Stokes, channels and IFs, in floats (desc->incs...) */
  int incs, incf, incif;
  int nchan, nif;
  /* increments into the per-(channel, IF) frequency tables */
  int kincf, kincif;
  /* selection; starts are 0-relative (startChannelPB-1 etc.) */
  int startChannel, numberChannel, startIF, numberIF, startPoln, numberPoln;
  /* component table: ncomp rows of lcomp floats, reference layout */
  int modType, nterm, lcomp, ncomp;
  const float *comps;
  /* operation */
  int doDivide, doReplace;
  /* per-polarization handling: model for the j-th selected polarization is
   * (flip bit j ? i : 1) * polFact[j] * stokFactor^(number of earlier
   * polarizations actually written), the CPU reference's rule
   * (ObitSkyModel.c:2787-2849); polFact carries GPUModelInfo.stokFact. */
  int flipMask;
  float stokFactor;
  float polFact[4];
  /* frequency tables indexed ichan*kincf + iIF*kincif */
  const double *fscale;   /* nu / nu_uv_reference, used by the FP64 oracle */
  const float *fscale32;  /* the FP32 desc->fscale, used by restatement B */
  const double *lnspec;   /* Spec: ln(nu/nu_model_ref); TSpec: ln(nu/nu_plane) */
  const int *specIndex;   /* TSpec: coarse plane per (channel, IF) */
  /* optional FP64 X, Y, Z per component (3 doubles each) used for the phase in
   * place of the FP32 fields 1-3 of the table (the FP64 oracle only) */
  const double *xyz;
} OracleJob;

/* One component's FP64 amplitude (flux x spectrum x taper) and phase
 * X u + Y v + Z w at scaled (u, v, w), for the log-frequency term L and the
 * coarse plane of the (channel, IF) (the per-component step of the model
 * functions below). */
void oracle_comp_term(const OracleJob *job, int ic, double u, double v, double w, double L,
                      int plane, double *amp, double *phase);

/* (A) FP64 model: for every row and selected (channel, IF) writes the raw
 * complex component sum S = sum_c amp_c exp(i phase_c) (no flip, no
 * polarization factor) to model[(row*nfreq + ifq)*2 + {0,1}] and the L1 norm
 * sum_c |amp_c| to l1[row*nfreq + ifq], where nfreq = nchan*nif and
 * ifq = ichan*kincf + iIF*kincif.  Unselected entries are left untouched.
 * Returns 0, or -1 for an unsupported model type. */
int oracle_model_fp64(const OracleJob *job, const float *vis, double *model,
                      double *l1, int nthreads);

/* (A) FP64 model applied to vis in place (subtract / divide / replace) with
 * the CPU reference's weight and polarization rules; arithmetic in double,
 * results rounded to float. Returns 0, or -1 for an unsupported model type. */
int oracle_apply_fp64(const OracleJob *job, float *vis, int nthreads);

/* (B) reference-faithful restatement; in oracle/_ref/libobit_refcpu.so only. */
int refcpu_apply(const OracleJob *job, float *vis, int nthreads);

/* Beam-corrected DFT (oracle_beam.c): antenna types, the Jones plane of each
 * (channel, IF) and the Jones table of ObitCUDABeamModel (GPUBeamAntInfo,
 * ObitSystem/Obit/include/ObitCUDABeamModelInfoDef.h:178-205). */
typedef struct OracleBeam {
  int numAnt, numAntType, numJChan;
  const int *antType;   /* [numAnt] type of each antenna (0-rel) */
  const int *jchan;     /* [nchan*nif] Jones plane per (channel, IF) table index */
  int ilocb;            /* BASELINE offset in the record, or -1 */
  int iloca1, iloca2;   /* ANTENNA1 / ANTENNA2 offsets when ilocb < 0 */
  const float *jones;   /* [numAntType][ncomp][numJChan][8]: XX, XY, YX, YY complex */
  int stokType;         /* 1..4 = I, Q, U, V sky */
  double c2p, s2p;      /* cos, sin of twice the parallactic angle (linear Q, U) */
  int circular;         /* 1: circular feeds (RR, LL, RL, LR), 0: linear */
} OracleBeam;

/* Applies the beam-corrected FP64 model (Stokes I, linear feeds) to the
 * records in place: job->numberPoln correlations from the first (XX, YY, XY,
 * YX), the job's channel / IF selection and operation.  l1 (may be NULL)
 * receives per (row, table index, model correlation XX/XY/YX/YY) the sum over
 * components of |amp| |coefficient|.  Returns 0, or < 0 for a bad job. */
void oracle_beam_jones(int ntype, int nx, int ny, int nplane, const float *pixels, float fblank,
                       int hwidth, int projection, const double crval[2], const double crpix[2],
                       const double cdelt[2], double crota, const double *planeFreq, double refSizeFact,
                       double parAng, const float *pos, int ncomp, float *jones);
int oracle_beam_apply(const OracleJob *job, const OracleBeam *beam, float *vis, double *l1,
                      int nthreads);

/* The four model coefficients (XX, XY, YX, YY) of one Jones pair for Stokes
 * 1..4 (the step oracle_beam_apply takes per component). */
void oracle_beam_coeffs(int stokType, double c2p, double s2p, const float *J1, const float *J2,
                        double *cr, double *ci);

/* The reference's gridded-model loop (refcpu_grid.c): the interpolator's plane
 * (ny rows of nxp complex values), its kernel table ((ntab + 1) x 25), the
 * field geometry and the record layout, selection and operation.  Increments
 * and offsets in floats. */
typedef struct RefGridJob {
  const float *plane;
  int nxp, ny;
  const float *table;
  int ntab;
  float crpix0, crpix1, cdelt0, cdelt1;
  float flip;
  int do3Dmul;
  float umat[9];
  int doRot;
  float ccrot, ssrot;
  int doPC;
  float dxyzc[3];
  int lrec, nrparm, ilocu, ilocv, ilocw;
  const float *fscale;
  int kincf, kincif;
  int chanb, nchan, ifb, nif, incf, incif, incs, stokb, nstok;
  int doDivide, doReplace, doFlip;
  float stokFactor;
} RefGridJob;

int refcpu_grid_apply(const RefGridJob *job, float *vis, long nvis, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
