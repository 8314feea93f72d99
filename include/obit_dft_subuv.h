/* The caller of the model path: ObitSkyModelSubUV's pass structure
 * (ObitSystem/Obit/src/ObitSkyModel.c:850-1087) over this library's GPU paths,
 * native.  Data I/O, calibration and the selection of the reference's ObitUV
 * layer stay with the caller, which hands over one buffer of records.
 */
#ifndef OBIT_DFT_SUBUV_H
#define OBIT_DFT_SUBUV_H
#include "obit_dft_comps.h"
#include "obit_dft_grid.h"
#include "obit_gpu_skymodel.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Applies the CLEAN model of `fields` (CC tables with their image geometry,
 * `images` the fields' image sizes) to uv->buffer (uv->numVisBuff records)
 * in place, with the operation, factor and channel / IF / polarization
 * selection of `sky` (its modType and nSpecTerm are taken from the loaded
 * table; modelRefFreq as for ObitGPUSkyModelDFTInit).
 *   mode      0 chooses as ObitSkyModelChose (ObitSkyModel.c:3560-3620), or
 *             from this library's measured B200 rates when measured = 1
 *             (obit_dft_choose_mode_measured); 1 forces the DFT, 2 the
 *             gridded model, 3 OBIT_SkyModel_Mixed: per field, the DFT of
 *             the components above model->minDFT, then the gridded model of
 *             those of at most maxGrid (ObitSkyModel.c:1421-1424, 1512-1515;
 *             the caller sets the two thresholds as the reference's
 *             minDFT and maxGrid);
 *   DFT       every field's components in one table (ObitSkyModelLoadComps,
 *             here obit_dft_load_comps) applied in one pass (nload = -1,
 *             ObitSkyModel.c:986-987) through the ObitGPUSkyModel mirror
 *             (include/obit_gpu_skymodel.h), with the FP64 channel
 *             frequencies when uv->freqArr is given;
 *   gridded   each field in its own pass, in field order (:974-995),
 *             obit_dft_grid_create / obit_dft_grid_apply_host with maxGrid
 *             and kernel (OBIT_DFT_GRID_KERNEL_*); images must be given.
 * *modeUsed (1, 2 or 3) and *ncompUsed (DFT: merged component rows;
 * gridded: rows gridded over the fields; Mixed: both) are written when not
 * NULL.  Returns 0, or a status code of include/obit_dft.h with the message in
 * err (and in obit_dft_last_error for the library's own failures). */
int obit_dft_sub_uv(const ObitDFTCCField *fields, int nfield, const ObitDFTGridImage *images,
                    const ObitDFTCCModel *model, const ObitDFTSkyModel *sky, ObitDFTUVData *uv, int mode,
                    int measured, float maxGrid, int kernel, int *modeUsed, int *ncompUsed, ObitDFTErr *err);

/* The same pass structure for image models (OBIT_SkyModel_Image, which the
 * reference always grids: ObitSkyModelLoadImage, ObitSkyModel.c:1427-1428,
 * 2163-2260): per field, in field order, the model image pixels[f]
 * (images[f].nx x images[f].ny floats, square, row-major; host or device
 * memory) with blanking value fblank, the field's geometry from fields[f]
 * (its CC rows are not read), gridded and applied to uv->buffer with the
 * operation and selection of `sky`.  *npixUsed (pixels gridded over the
 * fields) is written when not NULL.  Returns 0 or a status code with the
 * message in err. */
int obit_dft_sub_uv_image(const float *const *pixels, float fblank, const ObitDFTCCField *fields, int nfield,
                          const ObitDFTGridImage *images, const ObitDFTCCModel *model, const ObitDFTSkyModel *sky,
                          ObitDFTUVData *uv, int kernel, long long *npixUsed, ObitDFTErr *err);

#ifdef __cplusplus
}
#endif
#endif
