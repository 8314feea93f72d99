/*
 * obit_dft_comps.h - CLEAN-component tables to the DFT component table
 * (host code in libobit_dft.so).  Plain C.
 *
 * Replaces the host step Obit runs before every DFT pass:
 *   ObitSkyModelLoadComps     ObitSystem/Obit/src/ObitSkyModel.c:1682-2121
 *   ObitTableCCUtilMergeSel   ObitSystem/Obit/src/ObitTableCCUtil.c:1238-1361
 * with the field geometry of ObitUVDescShiftPhase / ObitSkyGeomShiftSIN
 * (ObitUVDesc.c:735-790, ObitSkyGeom.c:177-205) and the 3-D re-projection
 * matrix of ObitUVDescShift3DMatrix (ObitUVDesc.c:882-978).  The caller reads
 * the CC tables and image headers (Obit's table and FITS layers are not part
 * of this library) and passes their columns and keywords below.
 *
 * Per field: the selected rows (startComp..endComp, deselected rows skipped)
 * are merged -- rows at the same (DeltaX, DeltaY) summed, except for tables
 * with polynomial spectra, which the reference does not merge -- and sorted by
 * decreasing |flux|; each merged component becomes one row of the output in
 * the reference field order ([flux * factor, X, Y, Z] then Gaussian and
 * spectral terms, as the DFT entry points of obit_dft.h read it).  Fields are
 * appended in order.  The model type of the output is the highest among the
 * fields; point fields in a Gaussian model carry zero Gaussian terms.
 * Supported: point, Gaussian, point / Gaussian with polynomial spectrum,
 * -SIN projection, 3-D images, and 2-D images whose centre is the uv phase
 * centre with no rotation or pixel offset; tabulated spectra through
 * obit_dft_load_comps_mf below.  Uniform spheres, exponential disks, -NCP
 * and shifted 2-D images are rejected with OBIT_DFT_EUNSUPPORTED.
 */
#ifndef OBIT_DFT_COMPS_H
#define OBIT_DFT_COMPS_H
#ifdef __cplusplus
extern "C" {
#endif

/* One field (image) of the model: its CC-table columns and image keywords. */
typedef struct {
  int nrow;                 /* rows in the column arrays */
  const float *flux;        /* FLUX, Jy */
  const float *deltaX;      /* DELTAX, deg */
  const float *deltaY;      /* DELTAY, deg */
  const float *deltaZ;      /* DELTAZ column or NULL */
  const float *parms;       /* PARMS, nrow x nparms (NULL when nparms is 0):
                               [0..2] major, minor FWHM (deg), PA (deg); [3] type
                               (ObitSkyModelCompType); [4..] spectral terms */
  int nparms;
  const int *status;        /* row status or NULL (< 0: deselected) */
  int startComp, endComp;   /* 1-relative; endComp <= 0: to the last row */
  double crvalRA, crvalDec; /* image reference position, deg */
  float rotation;           /* CROTA of the declination axis, deg */
  int do3D;                 /* image descriptor: 1 = 3-D image */
  float xPxOff, yPxOff;     /* 2-D images: reference pixel offsets, pixels */
  float cdeltX, cdeltY;     /* deg per pixel */
  float xShift, yShift;     /* image XSHIFT / YSHIFT keywords */
  int ncpProjection;        /* 1 = -NCP (unsupported), 0 = -SIN */
} ObitDFTCCField;

/* The sky model's own settings (ObitSkyModel members). */
typedef struct {
  double uvRA, uvDec;       /* uv phase centre, deg */
  float uvRotation;         /* uv rotation (CROTA of its declination axis), deg */
  float factor;             /* multiplies every flux (Factor) */
  float minFlux;            /* keep |flux| > minFlux */
  float minDFT;             /* keep |flux| > minDFT */
  int noNeg;                /* stop a field at its first merged flux <= 0 (Stokes I) */
  int do3D;                 /* sky-model 3-D flag: 1 ignores 2-D pixel offsets */
} ObitDFTCCModel;

/* Builds the component table.  With table NULL only sizes are returned:
 * *nrowOut = the rows to allocate (selected CC rows in all fields, an upper
 * bound), *lcomp = floats per row.  Otherwise table (capacity floats) receives
 * *nrowOut rows of *lcomp floats, of which the first *ncomp are components and
 * the rest zero; *modType is the model type (ObitSkyModelCompType numbering:
 * 0 point, 1 Gaussian, 10 point + spectrum, 11 Gaussian + spectrum) and
 * *nterm the spectral terms per row.  Returns OBIT_DFT_OK or an error code
 * with obit_dft_last_error() set. */
int obit_dft_load_comps(const ObitDFTCCField *fields, int nfield, const ObitDFTCCModel *model,
                        float *table, long long capacity, int *nrowOut, int *ncomp, int *lcomp,
                        int *modType, int *nterm);

/* The same, plus FP64 positions (no reference counterpart): when xyz and
 * table are both given, xyz (3 doubles per table row) receives X,
 * Y, Z of each component row written, computed with every step of the
 * geometry above (field shift, rotation, 3-D re-projection) in FP64, for
 * obit_dft_set_mod_d.  The table itself is the one obit_dft_load_comps
 * writes. */
int obit_dft_load_comps_d(const ObitDFTCCField *fields, int nfield, const ObitDFTCCModel *model,
                          float *table, long long capacity, int *nrowOut, int *ncomp, int *lcomp,
                          int *modType, int *nterm, double *xyz);

/* Settings of a multi-frequency sky model (ObitSkyModelMF members) whose
 * components carry tabulated spectra: one flux per coarse frequency plane. */
typedef struct {
  int nSpec;                /* coarse planes (the model image's NSPEC) */
  const double *specFreq;   /* [nSpec] plane frequencies, Hz; the fit's reference is specFreq[0] */
  int noSIfit;              /* 1: no spectral-index fit (polarized data, ObitSkyModelMF.c:1164-1168) */
  int doAlphaCorr;          /* 1: plane fluxes times (nu / priorAlphaRefF)^priorAlpha */
  float priorAlpha;
  double priorAlphaRefF;    /* Hz */
} ObitDFTCCModelMF;

/* ObitSkyModelMFLoadComps (ObitSkyModelMF.c:1130-1635): the component table
 * of point or Gaussian components with tabulated spectra (types 20 and 21,
 * PARMS[4 .. 4 + nSpec - 1] the per-plane fluxes).  Rows at the same position
 * merge with each plane's flux summed (CCMergeSpec); each output row is
 * [flux x factor, X, Y, Z, (g1, g2, g3,) alpha, S_0 .. S_nSpec-1] with S_k the
 * plane flux times factor (and the prior-alpha correction) and alpha the
 * spectral index fitted to the planes as ObitSpectrumFitSingleArg does for
 * two terms (weighted least squares of S_0 (nu / nu_0)^alpha, nu_0 =
 * specFreq[0], every plane's sigma 1e-4 Jy, exactly-zero planes left out;
 * the fit is kept only if its reduced chi^2 is below 1.5 times the constant
 * model's, and alpha outside [-2, 2] becomes 0).  Positions and selection as
 * obit_dft_load_comps.  *modType is 20 or 21; *lcomp = 5 (8 for Gaussians) +
 * nSpec.  Fields of other types, or of both TSpec types, are rejected with
 * OBIT_DFT_EUNSUPPORTED. */
int obit_dft_load_comps_mf(const ObitDFTCCField *fields, int nfield, const ObitDFTCCModel *model,
                           const ObitDFTCCModelMF *mf, float *table, long long capacity, int *nrowOut,
                           int *ncomp, int *lcomp, int *modType);

#ifdef __cplusplus
}
#endif
#endif /* OBIT_DFT_COMPS_H */
