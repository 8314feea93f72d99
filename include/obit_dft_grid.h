/*
 * obit_dft_grid.h - gridded model Fourier transform on the GPU
 * (libobit_dft.so).  Plain C.
 *
 * The reference's second way of predicting a CLEAN model, chosen per pass by
 * ObitSkyModelChose (ObitSystem/Obit/src/ObitSkyModel.c:3560-3620) and run on
 * its host threads:
 *   ObitSkyModelGridFTComps   ObitSkyModel.c:4243-4371  per field: the field's
 *     CLEAN components summed into a grid twice the image size
 *     (ObitTableCCUtilGrid, ObitTableCCUtil.c:106-302), FFT to a half plane
 *     (ObitSkyModelFTImage, :4475-4498), the Gaussian taper of a Gaussian
 *     model, conjugate columns (ObitCArrayAddConjg, ObitCArray.c:1660-1726)
 *     and a Lagrange interpolator (ObitCInterpolate.c:128-206, 699-830)
 *   ObitSkyModelFTGrid        ObitSkyModel.c:2878-2943, ThreadSkyModelFTGrid
 *     :2970-3232  per record and channel: u, v, w scaled to the channel,
 *     re-projected (3-D fields) or rotated, the half-plane conjugation, the
 *     interpolated model, the field-offset phase, then subtract / divide /
 *     replace over the selected polarizations.
 * Here the grid, FFT (cuFFT), taper and conjugate columns are built once per
 * field on the device, and one kernel applies the field to device-resident
 * records.
 *
 * Supported: point and Gaussian components (spectral terms are ignored, as
 * the reference's gridded path ignores them; every Gaussian of a field must
 * have one size), -SIN fields that are 3-D images, and 2-D images centred on
 * the uv phase centre with no rotation or pixel offset.  Exponential disks,
 * uniform spheres, -NCP and shifted 2-D images are rejected with
 * OBIT_DFT_EUNSUPPORTED.  Rows are read from startComp to endComp without
 * regard to their status, as the reference reads them.
 */
#ifndef OBIT_DFT_GRID_H
#define OBIT_DFT_GRID_H
#include "obit_dft.h"
#include "obit_dft_comps.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Image keywords of a field besides those of ObitDFTCCField. */
typedef struct {
  int nx, ny;            /* pixels along the RA and declination axes (inaxes) */
  float crpixX, crpixY;  /* reference pixel, 1-relative */
} ObitDFTGridImage;

/* Interpolation weights. */
enum {
  OBIT_DFT_GRID_KERNEL_REFERENCE = 0, /* the reference's table: 201 rows every 0.005
                                         cell, selected one row high, so that the
                                         model is the one at a point 0.005 cell
                                         (+- 0.0025) below the requested one */
  OBIT_DFT_GRID_KERNEL_EXACT = 1      /* 25-point Lagrange weights at the requested
                                         point itself, on a window centred on it (no
                                         counterpart); a point within 12 cells of the
                                         plane's edge, whose window would leave the
                                         plane, is blanked as off the plane */
};

typedef struct ObitDFTGrid ObitDFTGrid;

/* ObitSkyModelGridFTComps for one field on the current device: selects and
 * grids the components (factor, minFlux, noNeg of `model`; maxGrid the
 * largest |flux| gridded), FFTs, tapers and adds the conjugate columns, all
 * ordered on `stream` (a cudaStream_t; NULL = default stream).  *out receives
 * the field; it holds nothing to apply when no component was gridded
 * (obit_dft_grid_info).  kernel: OBIT_DFT_GRID_KERNEL_*. */
int obit_dft_grid_create(const ObitDFTCCField *field, const ObitDFTGridImage *image,
                         const ObitDFTCCModel *model, float maxGrid, int kernel, void *stream,
                         ObitDFTGrid **out);

/* ObitSkyModelLoadImage (ObitSkyModel.c:2163-2260), the image model
 * (OBIT_SkyModel_Image, which the reference always grids): a model image of
 * image->nx x image->ny pixels (square; row-major, nx per row; host or device
 * memory) instead of components.  Pixels below model->minFlux (or above 1e20)
 * and blanked pixels (value fblank) are zero, the rest times model->factor
 * (ObitFArrayClip and ObitFArrayPad); the image is centred in the grid of
 * twice its size by pixel nx / 2, then transformed and interpolated as the
 * component model is (no taper).  field gives the image's geometry only
 * (crval, rotation, do3D, pixel offsets, cdelt, shifts, projection); its rows
 * are not read.  The reference's primary-beam correction of the image
 * (doPBCor, ObitPBUtilImageCor) calls ObitPBUtilRelPB with its reference
 * frequency and minimum gain swapped (ObitPBUtil.c:566 against
 * ObitPBUtil.h:54-55), which clamps every gain to 1: the image is used as
 * it is there too. */
int obit_dft_grid_create_image(const float *pixels, float fblank, const ObitDFTCCField *field,
                               const ObitDFTGridImage *image, const ObitDFTCCModel *model, int kernel,
                               void *stream, ObitDFTGrid **out);

/* ThreadSkyModelFTGrid on nvis records at d_vis (device, lenvis floats each,
 * updated in place, asynchronously on `stream`).  visInfo gives the layout and
 * selection (its freqScale, the FP32 nu / nu_uvref per (channel, IF) as
 * ObitUVDesc.fscale, in device memory or in host memory, which is then copied
 * in order on `stream`); opType GPUOpTypeSub / Div / Repl;
 * stokFactor and doFlip as ObitSkyModel's: the model is multiplied by
 * stokFactor after each polarization written and by i when doFlip.  A model
 * point outside the plane zeroes the data and weight of every selected
 * polarization with positive weight (any, when replacing). */
int obit_dft_grid_apply(ObitDFTGrid *grid, const GPUVisInfo *visInfo, int opType, float stokFactor,
                        int doFlip, float *d_vis, int nvis, void *stream);

/* The same on records in host memory: h_vis (pinned, for the copies to
 * overlap) passes through three device slots of about 64 MB held by the field,
 * in chunks on three streams of the field, the upload, kernel and download of
 * different chunks overlapping, all ordered after the work queued on `stream`;
 * any number of records (device memory does not grow with nvis); returns when
 * h_vis holds the result. */
int obit_dft_grid_apply_host(ObitDFTGrid *grid, const GPUVisInfo *visInfo, int opType,
                             float stokFactor, int doFlip, float *h_vis, int nvis, void *stream);

/* Facts of a field: info[0] components gridded, [1] components off a cell
 * centre by more than 0.1 cell (the reference's warning count), [2] grid nx,
 * [3] grid ny, [4] plane columns (nx / 2 + 1 + 12 conjugate columns), [5] 1
 * when Gaussian-tapered, [6] 1 when u, v, w are re-projected (3-D field off
 * the phase centre), [7] 1 when the field-offset phase is applied, [8] 1 when
 * u, v are rotated, [9] kernel.  Writes min(n, 10) entries. */
int obit_dft_grid_info(const ObitDFTGrid *grid, long long *info, int n);

/* Copies the interpolator's plane (ny rows of nx / 2 + 13 complex values, re
 * and im floats) to host memory h_plane of `capacity` floats. */
int obit_dft_grid_plane(const ObitDFTGrid *grid, float *h_plane, long long capacity);

/* Releases the field's device memory. */
int obit_dft_grid_destroy(ObitDFTGrid *grid);

/* Mode choice of ObitSkyModelChose (ObitSkyModel.c:3560-3620).  modelMode:
 * 0 fastest, 1 DFT, 2 grid, 3 mixed (returned unchanged unless 0); modelType:
 * 0 components, 1 image, 2 point.  ncc, nx, ny: selected components and image
 * size of each of nfield fields; nvis records; nchan channels times IFs.
 * Returns 1 (DFT) or 2 (grid) for mode 0: the reference's time model
 * (1e-5 s per visibility interpolated, 0.8e-6 s per grid cell at 4 cells per
 * image pixel -- 2 above 2048 pixels --, 1e-4 s per component gridded, all
 * times channels and halved, against 6.6e-7 s per visibility-component
 * DFT). */
int obit_dft_choose_mode(int modelMode, int modelType, const int *ncc, const int *nx, const int *ny,
                         int nfield, long long nvis, int nchan);

/* The same choice from this library's own rates on a B200 (no counterpart):
 * the DFT costs ncc x nvis x nchan / dftRate seconds per field, the gridded
 * model nvis x nchan / gridRate plus gridSetup seconds per field; returns 1
 * (DFT) or 2 (grid) for the cheaper in total (2 for image models, 1 for point
 * models).  A rate or set-up of 0 takes the value measured on one B200 with
 * the default kernels: 4.5e12 component-visibility evaluations/s, 3.5e9 model
 * visibilities/s, 0.01 s per field.  The gridded model's accuracy is the
 * reference's table offset (see OBIT_DFT_GRID_KERNEL_REFERENCE) unless the
 * exact kernel is used; the DFT is exact to 1e-7 of the model's L1 norm. */
int obit_dft_choose_mode_measured(int modelType, const int *ncc, const int *nx, const int *ny, int nfield,
                                  long long nvis, int nchan, double dftRate, double gridRate,
                                  double gridSetup);

#ifdef __cplusplus
}
#endif
#endif /* OBIT_DFT_GRID_H */
