// Test infrastructure (never linked into the product): the reference's pixel
// geometry of beam images, CUDAPositionXYpix / CUDAPositionXYpixLM
// (ObitSystem/Obit/include/CUDASkyGeom.h:91-286: linear offsets and the -SIN,
// -TAN, -ARC, -NCP, -GLS, -MER, -AIT and -STG projections), compiled for the
// host from the reference's own header where it lies (oracle/Makefile, target
// refgeom) so that the oracle's projections (oracle_beam.c) are checked
// against the reference's code rather than a restatement of it.
#include <math.h>
#include <string.h>

#include <cuda_runtime_api.h>  // types named by the reference's headers

#define __device__
#define __forceinline__ inline
#define __sincosf sincosf
#define HAVE_GPU 1
#define IS_CUDA 1
#include "CUDASkyGeom.h"

// Pixel (1-relative) of position coord (deg) on a grid whose first axis type
// is ctype (e.g. "RA---TAN"), rotated by rotar (rad); returns the reference's
// status (0 placed, 1 outside the projection, 2 or 3 bad values).
extern "C" long ref_position_xypix(const double coord[2], const char* ctype, const double crval[2],
                                   const float crpix[2], const float cdelt[2], const float crota[2],
                                   float rotar, float pixel[2]) {
  static CUDAImageDesc desc;
  memset(&desc, 0, sizeof(desc));
  strncpy(desc.ctype[0], ctype, IMLEN_KEYWORD - 1);
  for (int a = 0; a < 2; a++) {
    desc.crval[a] = crval[a];
    desc.crpix[a] = crpix[a];
    desc.cdelt[a] = cdelt[a];
    desc.crota[a] = crota[a];
  }
  double c[2] = {coord[0], coord[1]};
  return CUDAPositionXYpix(c, &desc, rotar, pixel);
}
