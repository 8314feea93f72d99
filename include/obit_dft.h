/*
 * obit_dft.h - C ABI of the B200 DFT sky-model predict / subtract library
 * (libobit_dft.so).  Plain C: pointers, ints and floats, no C++ or torch types.
 *
 * Two levels are exported:
 *
 *  1. The reference's CUDA-layer entry points, same names and argument, so the
 *     library links in place of ObitCUDASkyModel.o under the unmodified
 *     ObitGPUSkyModel.c:
 *       ObitCUDASkyModelDFTInit / SetMod / Calc / Shutdown (GPUInfo*)
 *     replacing ObitSystem/Obit/include/ObitCUDASkyModel.h:44-54 (defined at
 *     ObitSystem/Obit/src/ObitCUDASkyModel.cu:727-783).  The structures below
 *     keep the field order and types of ObitCUDASkyModelInfoDef.h:42-195 so a
 *     GPUInfo filled by ObitGPUSkyModelDFTInit / DFTSetMod
 *     (ObitSystem/Obit/src/ObitGPUSkyModel.c:207-491) is read as is.
 *
 *  2. Status-returning forms of the same four calls plus additions the
 *     reference has no equivalent for (FP64 frequency side table, CPU-reference
 *     polarization rules, kernel choice, a device-resident call and a
 *     multi-facet batch).  Every call returns OBIT_DFT_OK (0) or an error code;
 *     obit_dft_last_error() gives the calling thread's last message.  Nothing
 *     in the library calls exit(), abort() or cudaDeviceReset().
 */
#ifndef OBIT_DFT_H
#define OBIT_DFT_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference-layout types (ObitCUDASkyModelInfoDef.h:42-195) ---------- */

/* Sky model component types supported on the GPU
 * (ObitCUDASkyModelInfoDef.h:44-52). */
enum gpuModType {
  GPUModTypePoint = 0,  /* point */
  GPUModTypePointSpec,  /* point, spectrum as polynomial in ln(nu/nu0) */
  GPUModTypePointTSpec, /* point, tabulated spectrum per coarse plane */
  GPUModTypeGauss,      /* elliptical Gaussian */
  GPUModTypeGaussSpec,  /* Gaussian, polynomial spectrum */
  GPUModTypeGaussTSpec  /* Gaussian, tabulated spectrum */
};
typedef enum gpuModType GPUModType;

/* Operation applied to the data (ObitCUDASkyModelInfoDef.h:58-63). */
enum gpuOpType {
  GPUOpTypeSub = 0, /* data -= model */
  GPUOpTypeDiv,     /* data /= model, weight *= |model| */
  GPUOpTypeRepl     /* data = model */
};
typedef enum gpuOpType GPUOpType;

/* Visibility layout (ObitCUDASkyModelInfoDef.h:66-123).  Increments incf,
 * incif, incs are in correlations (3 floats each), as ObitGPUSkyModel.c fills
 * them (desc->incf/3 ...). */
typedef struct {
  int nvis;   /* records in the buffer */
  int nprod;  /* correlations per record */
  int nrparm; /* random parameters per record */
  int lenvis; /* floats per record */
  int nchan;
  int ilocu, ilocv, ilocw, iloct, ilocb, ilocsu; /* random-parameter offsets */
  int chanb, chane; /* selected channels, 0-relative inclusive */
  int incf;         /* correlations between channels */
  int nIF;
  int IFb, IFe;     /* selected IFs */
  int incif;        /* correlations between IFs */
  int nstok;
  int stokb, stoke; /* selected polarizations */
  int incs;         /* correlations between polarizations */
  int stype;        /* 0 IQUV, 1 RR/LL/RL/LR, 2 XX/YY/XY/YX */
  int kincif;       /* IF increment in freqScale */
  int kincf;        /* channel increment in freqScale */
  float *freqRat;   /* host: uv reference freq / model (or coarse-plane) freq */
  float *d_freqRat; /* device copy of freqRat */
  float *freqScale; /* device: nu/nu_uvref per (channel, IF), nchan*nIF floats */
} GPUVisInfo;

/* Model description (ObitCUDASkyModelInfoDef.h:125-146). */
typedef struct {
  int nterm;          /* spectral terms */
  int size;           /* floats per component */
  int doSwap;         /* multiply the model of polarization 3 (LR) by i */
  GPUModType type;
  GPUOpType opType;
  int *specIndex;     /* host: coarse plane per (channel, IF), tabulated spectra */
  int *d_specIndex;   /* device copy of specIndex */
  int nmodel[4];      /* components per polarization */
  float *model[4];    /* device component tables per polarization */
  float stokFact[4];  /* multiplier per polarization */
} GPUModelInfo;

/* Per-instance state (ObitCUDASkyModelInfoDef.h:148-195).  stream/cycleDone
 * are arrays of cudaStream_t / cudaEvent_t, declared as void* so that this
 * header needs no CUDA include; the layout is the same. */
typedef struct {
  int nvis;
  int nchan;
  int nrparm;
  int lenvis;
  int modelSize;
  int nstream;
  int prtLv;
  int oldnVisPIO;
  int cuda_device;
  int bufferSize;
  int nmodel[4];
  float *d_model[4];
  float *d_freq;
  float *h_data;   /* pinned host buffer of nvis records */
  float **d_data;  /* nstream device buffers of (nvis+3)*lenvis/nstream floats */
  GPUVisInfo *d_visInfo, *h_visInfo;
  GPUModelInfo *d_modelInfo, *h_modelInfo;
  void **stream;
  void **cycleDone;
} GPUInfo;

/* ---- level 1: the reference's CUDA-layer symbols ------------------------ */

/* Replaces ObitCUDASkyModelDFTInit (ObitCUDASkyModel.h:44-45,
 * ObitCUDASkyModel.cu:727-731): binds library state to this GPUInfo on
 * gpuInfo->cuda_device.  Call after the GPUInfo fields are filled. */
void ObitCUDASkyModelDFTInit(GPUInfo *gpuInfo);

/* Replaces ObitCUDASkyModelDFTSetMod (ObitCUDASkyModel.h:47-48,
 * ObitCUDASkyModel.cu:733-744): takes the component table now in
 * gpuInfo->d_model[0] (nmodel[0] rows of modelSize floats) and the model
 * description in h_modelInfo. */
void ObitCUDASkyModelDFTSetMod(GPUInfo *gpuInfo);

/* Replaces ObitCUDASkyModelDFTCalc (ObitCUDASkyModel.h:50-51,
 * ObitCUDASkyModel.cu:746-765): applies the model to the nvis records in the
 * pinned buffer gpuInfo->h_data, in place, synchronously. */
void ObitCUDASkyModelDFTCalc(GPUInfo *gpuInfo);

/* Replaces ObitCUDASkyModelDFTShutdown (ObitCUDASkyModel.h:53-54,
 * ObitCUDASkyModel.cu:767-783): releases this GPUInfo's library state.  Unlike
 * the reference it does not reset the device. */
void ObitCUDASkyModelDFTShutdown(GPUInfo *gpuInfo);

/* ---- level 2: status-returning API -------------------------------------- */

enum {
  OBIT_DFT_OK = 0,
  OBIT_DFT_EBADARG = 1,     /* invalid argument or descriptor */
  OBIT_DFT_ECUDA = 2,       /* CUDA runtime error */
  OBIT_DFT_EUNSUPPORTED = 3,/* model type / layout not supported */
  OBIT_DFT_EKERNEL = 4      /* a kernel reported an internal error */
};

/* Kernel flavors for obit_dft_set_kernel. */
enum {
  OBIT_DFT_RECUR = 0, /* split-FP32 phase + complex channel recurrence (default) */
  OBIT_DFT_PLAIN = 1, /* FP64 phase, one sin/cos per component-visibility */
  OBIT_DFT_RECUR_CHAIN = 2 /* the recurrence, with point components that carry a
                              spectral index kept on the chain form (no
                              spectral-factored form); a comparator */
};

/* Status forms of the four calls above. */
int obit_dft_init(GPUInfo *gpuInfo);
int obit_dft_set_mod(GPUInfo *gpuInfo);
int obit_dft_calc(GPUInfo *gpuInfo);
int obit_dft_shutdown(GPUInfo *gpuInfo);

/* FP64 component positions (no reference counterpart; the reference's device
 * table holds FP32 X, Y, Z, which at 1e7-radian phases -- VLBI baselines, a
 * field far from the phase centre -- limit the phase itself to about a radian).
 * xyz: X, Y, Z of each component in FP64, in the units of fields 1-3 of the
 * component table (ObitSkyModel.c:1965-1982), at least as many as the model
 * set by the last SetMod.  Fields 1-3 of the library's device copy become the
 * nearest floats and the remainders a side table, so the split-FP32 phase
 * carries the FP64 positions; the plain kernel adds them in FP64.  NULL drops
 * the side table; the next SetMod drops it too.  The multi-facet batch and
 * obit_dft_calc_noalloc take FP32 positions only.  The void form records
 * failures for obit_dft_last_error like the four calls above. */
int obit_dft_set_mod_d(GPUInfo *gpuInfo, const double *xyz, int ncomp);
void ObitCUDASkyModelDFTSetModD(GPUInfo *gpuInfo, const double *xyz, int ncomp);

/* Beam-corrected DFT, linear feeds, Stokes I, Q, U or V sky (the model of
 * ObitCUDABeamModel's beam*Kernel family, ObitCUDABeamModel.cu:139-1226, with
 * the Jones products of cudaJonesCor1_Lin_{I,Q,U,V}, CUDALinCorSum.h:104-455).  No
 * level-2 counterpart of this shape: the reference's ObitCUDABeamModelDFT*
 * calls take a GPUBeamInfo of device beam-image interpolators
 * (ObitCUDABeamModelInfoDef.h:148-275) and fill the Jones table from them on
 * the GPU; here the caller passes the Jones table itself.  For a record of
 * baseline (a1, a2) -- from BASELINE = 256 a1 + a2 (+ subarray fraction) or
 * ANTENNA1 / ANTENNA2, as GetAnts (ObitCUDABeamModel.cu:82-99) -- and a
 * (channel, IF) of Jones plane jc, component c contributes its DFT term times
 *   XX: P(0,0) + P(1,1)   XY: P(1,3) + P(0,2)   YX: P(2,0) + P(3,1)   YY: P(2,2) + P(3,3),
 * P(i, j) = J1[i] conj(J2[j]), J1 = jones[type(a1)][c][jc], J2 = jones[type(a2)][c][jc],
 * for Stokes I; Q and U combine D = P00 - P11 (XY: P02 - P13, YX: P20 - P31, YY:
 * P22 - P33) and S = P10 + P01 (P12 + P03, P30 + P21, P32 + P23) as c2p D - s2p S
 * and c2p S + s2p D with c2p, s2p = cos, sin of twice the parallactic angle; V is
 * i (P01 - P13), i (P03 - P12), i (P21 - P30), i (P23 - P32) -- the combinations
 * the reference's GPU kernels and its CPU ObitSkyModelVMBeamJonesCorSum use.
 * The records' first correlations XX, YY (, XY, YX with four) are modelled;
 * each one with positive weight (any, when replacing) is subtracted from,
 * divided into (weight unchanged) or replaced by its model times stokFact of
 * its position, independently of the others; every selected channel of every
 * selected IF is processed.  Once set, obit_dft_calc and obit_dft_calc_device
 * apply the beam-corrected model; NULL returns to the plain sky model; the
 * multi-facet batch and obit_dft_calc_noalloc do not take a beam; an FP64 side
 * table set by obit_dft_set_mod_d enters the beam path's phases as it does the
 * plain model's.  A record
 * whose antennas fall outside antType is left untouched and the call reports
 * OBIT_DFT_EKERNEL (code 3). */
typedef struct ObitDFTBeam {
  int numAnt;            /* antennas: records number them 1..numAnt */
  int numAntType;        /* antenna types */
  int numJChan;          /* Jones planes */
  const int *antType;    /* host [numAnt]: type of each antenna, 0..numAntType-1 */
  const int *jchan;      /* host [nchan*nIF]: Jones plane of each (channel, IF), freqScale order */
  int ilocb;             /* BASELINE random parameter offset, or -1 */
  int iloca1, iloca2;    /* ANTENNA1 / ANTENNA2 offsets when ilocb < 0 */
  int stokType;          /* Stokes of the sky model: 1 I, 2 Q, 3 U, 4 V */
  const float *jones;    /* device, 16-byte aligned: [numAntType][jonesComps][numJChan] 2x2
                            complex matrices of 8 floats (XX, XY, YX, YY as re, im) */
  int jonesComps;        /* components per type in jones, at least the model's */
  float parAng;          /* parallactic angle, radians (Stokes Q and U, linear feeds) */
  int circular;          /* 1: circular feeds, records RR, LL, RL, LR and Jones matrices
                            in the R, L basis; 0: linear feeds (XX, YY, XY, YX) */
} ObitDFTBeam;
int obit_dft_set_beam(GPUInfo *gpuInfo, const ObitDFTBeam *beam);

/* The beam kernel the next call will use (building the plan if needed):
 * info[0] = form (0: blocks of at most 8 channels on the FP32 pipe, 1: the
 * tensor-core form -- point families on uniformly spaced channels with the
 * default flavor; OBIT_DFT_RECUR_CHAIN keeps the block form -- 2: one thread
 * per channel, OBIT_DFT_PLAIN), info[1] = components per tile, info[2] =
 * channel runs (form 1) or blocks per record (forms 0 and 2).  Writes
 * min(n, 3) entries; OBIT_DFT_EBADARG when no beam is set.  Form 1 keeps
 * per-plan device tables of the split Jones coefficients and the spectral
 * amplitudes, rewritten at the start of every call (once per obit_dft_calc,
 * before its first chunk), so a Jones table refilled in place between calls
 * is read afresh; calls on one GPUInfo that overlap on the GPU share them. */
int obit_dft_beam_info(GPUInfo *gpuInfo, int *info, int n);

/* Beam images from which the Jones table is interpolated: for every antenna
 * type the 8 images of GetJonesKernel's interpolators
 * (ObitCUDABeamModel.cu:1228-1299): P1 re, P1 im, P2 re, P2 im, X1 re, X1 im,
 * X2 re, X2 im -- the parallel hands (XX or RR, YY or LL) and the cross terms
 * (XY or RL, YX or LR) -- each nplane planes (the Jones planes) of ny rows of
 * nx pixels, on one pixel grid. */
typedef struct ObitDFTBeamImages {
  int numAntType;        /* antenna types */
  int nx, ny, nplane;    /* pixels per row, rows, planes */
  const float *pixels;   /* device: [numAntType][8][nplane][ny][nx] */
  float fblank;          /* value of blanked pixels */
  int hwidth;            /* Lagrange interpolation half-width, 1..4 (2 hwidth + 1 taps per axis) */
  int projection;        /* 0: linear offsets; about crval 1 -SIN, 2 -TAN, 3 -ARC, 4 -NCP,
                            5 -GLS, 6 -MER, 7 -AIT, 8 -STG (CUDASkyGeom.h:91-250) */
  double crval[2];       /* reference position of the grid (deg) */
  float crpix[2];        /* reference pixel (1-relative) */
  float cdelt[2];        /* pixel increments (deg) */
  const float *planeFreq;/* host [nplane]: frequency (Hz) of each plane */
  float refSizeFact;     /* primary-beam factor of InvBeam (ObitCUDABeamModel.cu:66-72):
                            antenna size x 1.052 x DG2RAD / VELIGHT, per Hz per degree */
  float crota;           /* rotation of the grid's y axis (deg, CROTA2); enters the -MER and
                            -AIT scale factors only, as in CUDAPositionXYpixLM */
} ObitDFTBeamImages;

/* Fill a Jones table in the layout of ObitDFTBeam.jones ([numAntType][ncomp]
 * [nplane] 2x2 complex matrices of 8 floats, device, 16-byte aligned) by
 * interpolating the beam images at each component's position, as
 * GetJonesKernel does: the pixel of the position rotated by the parallactic
 * angle parAng (radians), a Lagrange interpolation of each image in each
 * plane (taps on blanked pixels dropped; blank when the remaining weight is
 * at most 0.9), each value times the inverse primary-beam gain of the
 * component's offset, and the unit matrix where the position is off the
 * grid, the gain factor is 10 or more, a parallel hand's real part exceeds
 * 1.3, or an interpolant is blank (the reference tests P1's real part twice
 * where P2's is meant, and lets blanks through the cross terms).  pos:
 * device [ncomp][2], each component's offset from the pointing centre (deg)
 * in the grid's coordinates.  Antenna types whose images lie on different
 * grids (the reference holds a descriptor per type, GetJonesKernel reading
 * type t's from interpolator 8 t) take one call per type with numAntType = 1,
 * that type's pixels and grid, and jones advanced by t x ncomp x nplane x 8
 * floats; every type has the same nplane.  Asynchronous on `stream`. */
int obit_dft_beam_jones(const ObitDFTBeamImages *images, const float *pos, int ncomp, float parAng,
                        float *jones, void *stream);

/* FP64 frequency side table (no reference counterpart; the reference passes
 * only FP32 freqScale).  freqArr: nchan*nIF channel frequencies in Hz indexed
 * like freqScale (ObitUVDesc.freqArr, ObitUVDesc.c:506-617); uvRefFreq: the
 * data reference frequency (desc->freq); modelRefFreq: reference frequency of
 * polynomial spectra (image CRVAL of the frequency axis; 0 = uvRefFreq);
 * specFreq/nSpec: coarse-plane frequencies of tabulated spectra (may be NULL).
 * With it the phase is formed from FP64 frequencies; without it from the FP32
 * freqScale the reference supplies. */
int obit_dft_set_freq(GPUInfo *gpuInfo, const double *freqArr, int nfreq, double uvRefFreq,
                      double modelRefFreq, const double *specFreq, int nSpec);

/* Polarization rules of the reference CPU DFT (ObitSkyModel.c:2787-2849)
 * instead of the per-polarization stokFact of GPUModelInfo: the model is
 * multiplied by stokFactor after each polarization actually written, and by
 * i for every polarization when doFlip.  cpuRules = 0 restores stokFact. */
int obit_dft_set_poln(GPUInfo *gpuInfo, int cpuRules, float stokFactor, int doFlip);

/* Kernel flavor, channels per thread (recurrence: 2, 4, 8, 16, 32; plain:
 * 1, 2, 4, 8, 16) and components per shared-memory tile; 0 keeps the current
 * value. */
int obit_dft_set_kernel(GPUInfo *gpuInfo, int flavor, int chanPerThread, int compsPerTile);

/* CTA tile shape: channel blocks per tile (1, 2, 4, ..., 32; 0 = planner's
 * choice) and threads per CTA (128 or 256; 0 = planner's choice: 256, or 128
 * when the records have at most two channel blocks).  Rows per tile are
 * threads / blocks (at least 8). */
int obit_dft_set_tile(GPUInfo *gpuInfo, int blocksPerTile, int threadsPerCTA);

/* Device-resident form of Calc: applies the model to nvis records already in
 * device memory at d_vis (lenvis floats each), asynchronously on `stream`
 * (a cudaStream_t; NULL = default stream).  No host copies. */
int obit_dft_calc_device(GPUInfo *gpuInfo, float *d_vis, int nvis, void *stream);

/* The plan the next call will use (building it if needed): info[0..10] =
 * flavor, channels per thread, components per tile, blocks per tile, rows per
 * tile, threads per CTA, channel blocks per row, channel-increment classes;
 * info[8] = 1 when point components with one spectral index take the
 * spectral-factored recurrence (0: the chain form); info[9] = 1 when a
 * Gaussian model with one spectral index runs mixed (its untapered components
 * as spectral-factored points, the rest in the chain form, one launch), and
 * info[10] the number of those point components.  Writes min(n, 11)
 * entries. */
int obit_dft_plan_info(GPUInfo *gpuInfo, int *info, int n);

/* No counterpart in the reference.  The same model application as
 * obit_dft_calc_device, for callers that cannot let a library allocate device
 * memory: processes whose device memory is all owned by their own pool (a
 * caching allocator, or a job sized to fill HBM), and latency-bound callers
 * that cannot take cudaFree's implicit device synchronization.  The caller passes
 * only inputs and outputs: the descriptors (host structs; visInfo->freqScale,
 * modelInfo->model[0] and the records d_vis are device memory, specIndex
 * host or device), an optional FP64 frequency table as for obit_dft_set_freq
 * (freqArr NULL uses the FP32 freqScale), and nvis records at d_vis updated in
 * place on `stream`.  Polarizations follow GPUModelInfo (stokFact, doSwap).
 * Scratch lives in a fixed 8 MiB device array inside the library (error flag,
 * channel blocks, padded component table): larger models are rejected with
 * OBIT_DFT_EUNSUPPORTED.  No cudaMalloc/cudaFree is called.  Device
 * descriptors (freqScale, a device specIndex) are read in order on `stream`.
 * The call is synchronous -- it waits for `stream` and returns after the update
 * is complete -- and must never be made while a stream is capturing.  All calls
 * share the array: calls that overlap on the GPU race and must be serialized. */
int obit_dft_calc_noalloc(const GPUVisInfo *visInfo, const GPUModelInfo *modelInfo,
                          const double *freqArr, double uvRefFreq, double modelRefFreq,
                          const double *specFreq, int nSpec, float *d_vis, int nvis,
                          void *stream);

/* ---- multi-facet batch ---------------------------------------------------
 * The reference applies a multi-facet model one field (and one buffer) at a
 * time: ObitSkyModel loops over the mosaic's images and calls
 * ObitGPUSkyModelDFTCalc / ObitCUDASkyModelDFTCalc per buffer
 * (ObitSystem/Obit/src/ObitGPUSkyModel.c:502-518).  The batch below has no
 * counterpart there: it applies many facets -- each its own device-resident
 * records, layout, frequencies and component table, with uneven row and
 * component counts -- in one persistent kernel launch per model family,
 * captured once in a CUDA graph and replayed.  Facets of one model family
 * share one tile shape (channels per thread, components per tile, blocks and
 * rows per CTA), chosen by obit_dft_batch_autotune or set explicitly. */

/* One facet.  visInfo/modelInfo are read at creation as for the single-facet
 * calls (modelInfo->model[0] is the device component table of nmodel[0] rows
 * of `size` floats, copied at creation; visInfo->freqScale is read unless
 * freqArr is given); d_vis holds nvis records updated in place by each run.
 * cpuRules/stokFactor/doFlip as for obit_dft_set_poln. */
typedef struct {
  const GPUVisInfo *visInfo;
  const GPUModelInfo *modelInfo;
  const double *freqArr; /* optional nchan*nIF FP64 channel frequencies (Hz) */
  double uvRefFreq;      /* data reference frequency (with freqArr) */
  double modelRefFreq;   /* polynomial-spectrum reference (0 = uvRefFreq) */
  const double *specFreq;/* coarse-plane frequencies, tabulated spectra */
  int nSpec;
  int cpuRules;
  float stokFactor;
  int doFlip;
  float *d_vis;
  int nvis;
} ObitDFTFacet;

typedef struct ObitDFTBatch ObitDFTBatch;

/* Plans every facet on the current device (tile shape: the planner's default
 * for the first facet of each model family until tuned or set), copies the
 * component tables and builds the facet parameter blocks and work list. */
int obit_dft_batch_create(const ObitDFTFacet *facets, int nfacet, ObitDFTBatch **out);

/* Times candidate tile shapes per model family on a scratch copy of a row
 * sample of every facet (the facets' records are not modified) and keeps the
 * fastest.  best (may be NULL) receives, for the family of the most work,
 * {K, compsPerTile, blocksPerTile, rowsPerTile, threads, candidates tried}. */
int obit_dft_batch_autotune(ObitDFTBatch *batch, void *stream, int *best);

/* Fixes the tile shape of every model family (0 keeps the planner's choice
 * for that field); invalidates the captured graph. */
int obit_dft_batch_set_tile(ObitDFTBatch *batch, int chanPerThread, int compsPerTile,
                            int blocksPerTile, int threadsPerCTA);

/* Applies every facet's model to its records: one graph launch on `stream`
 * holding, per model family, a counter reset and one persistent batch kernel.
 * The graph is captured at the first run after creation or a tile change.
 * Asynchronous; obit_dft_batch_check reads the kernels' error flag. */
int obit_dft_batch_run(ObitDFTBatch *batch, void *stream);

/* Streamed form of obit_dft_batch_run for records in host memory: facet i's
 * nvis records (the count given at creation) are read from and written back to
 * h_vis[i] (pinned memory, for the copies to overlap the kernels).  The rows
 * pass through a device staging area of stagingBytes, in waves that fill one
 * half of it each: one graph launch on `stream` copies wave w in, applies the
 * batch kernels to it and copies it out, wave w + 1's upload overlapping wave
 * w's kernels on a second stream.  The graph is captured at the first call and
 * again when h_vis, stagingBytes or the tile shape change.  info (may be NULL)
 * receives {waves, bytes uploaded per run}.  Asynchronous: the host records
 * are complete once `stream` is; obit_dft_batch_check reads the kernels'
 * error flag.  The staging area must hold two records of the widest facet. */
int obit_dft_batch_run_host(ObitDFTBatch *batch, float *const *h_vis, long long stagingBytes, void *stream,
                            long long *info);

/* Comparator: the same work as one kernel launch per facet on `stream`, with
 * each facet's own planner-default plan of kernel `flavor`
 * (OBIT_DFT_RECUR or OBIT_DFT_PLAIN). */
int obit_dft_batch_run_per_facet(ObitDFTBatch *batch, int flavor, void *stream);

/* Synchronizes the device, reads and clears the batch's error flag. */
int obit_dft_batch_check(ObitDFTBatch *batch);

/* Batch facts: info[0] facets, [1] model families (kernel launches per run),
 * [2] work items, [3] component-visibility evaluations per run, then for the
 * family of the most work [4] K, [5] compsPerTile, [6] blocksPerTile,
 * [7] rowsPerTile, [8] threads, [9] grid.  Writes min(n, 10) entries. */
int obit_dft_batch_info(ObitDFTBatch *batch, long long *info, int n);

/* Releases the batch's device memory, graph and streams. */
int obit_dft_batch_destroy(ObitDFTBatch *batch);

/* ---- records resident across CLEAN major cycles ----------------------------
 * No counterpart in the reference, which re-reads the data and copies every
 * buffer to the GPU and back each major cycle (ObitDConCleanVisMF.c:907,
 * ObitGPUSkyModel.c:510-517).  The records are uploaded once; each cycle
 * resets a device work copy to them, applies its models to that copy with the
 * device-resident calls (obit_dft_calc_device, obit_dft_batch_run on facets
 * pointing into it, obit_dft_grid_apply), and downloads the residual.  Device
 * memory: twice the records. */
typedef struct ObitDFTResident ObitDFTResident;

/* Uploads nvis records of lenvis floats from h_vis (pinned for speed) on the
 * current device; returns when they are resident. */
int obit_dft_resident_create(const float *h_vis, int nvis, int lenvis, void *stream, ObitDFTResident **out);

/* Resets the work copy to the uploaded records (device-to-device, ordered on
 * `stream`). */
int obit_dft_resident_reset(ObitDFTResident *r, void *stream);

/* Device pointer of the work copy (nvis records), for the device-resident
 * calls; NULL for a NULL handle. */
float *obit_dft_resident_records(ObitDFTResident *r);

/* Copies the work copy to h_out (nvis x lenvis floats) after the work queued
 * on `stream`; returns when h_out holds it. */
int obit_dft_resident_download(ObitDFTResident *r, float *h_out, void *stream);

/* Releases the device copies. */
int obit_dft_resident_destroy(ObitDFTResident *r);

/* Reads and clears the kernels' device error flag (synchronizes the device):
 * OBIT_DFT_OK or OBIT_DFT_EKERNEL. */
int obit_dft_check(GPUInfo *gpuInfo);

/* Diagnostic, no counterpart in the reference: polls of a component-tile copy
 * before a kernel gives up, sets the error flag and leaves its remaining
 * records untouched (default 4194304; a negative value restores it).  0 makes
 * every wait give up at once, which exercises the timeout path -- the call
 * then reports OBIT_DFT_EKERNEL and the CUDA context stays usable.  A lowered
 * limit runs a separate kernel instance, available for 32-channel
 * point+spectrum plans. */
int obit_dft_set_wait_limit(GPUInfo *gpuInfo, int polls);

/* Last error message of the calling thread ("" if none). */
const char *obit_dft_last_error(void);

/* Library version (major*10000 + minor*100 + patch). */
int obit_dft_version(void);

#ifdef __cplusplus
}
#endif
#endif /* OBIT_DFT_H */
