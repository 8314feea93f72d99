// Test infrastructure (never linked into the product): the reference's pixel
// geometry of beam images, CUDAPositionXYpix / CUDAPositionXYpixLM
// (ObitSystem/Obit/include/CUDASkyGeom.h:91-286: linear offsets and the -SIN,
// -TAN, -ARC, -NCP, -GLS, -MER, -AIT and -STG projections), and its beam-image
// interpolator, CUDABeamInterpPixel / SetConvKernal
// (ObitSystem/Obit/include/CUDABeamInterp.h:81-258), compiled for the host
// from the reference's own headers where they lie (oracle/Makefile, target
// refgeom) so that the oracle's projections and interpolation (oracle_beam.c)
// are checked against the reference's code rather than a restatement of it.
#include <math.h>
#include <string.h>

#include <cuda_runtime_api.h>  // types named by the reference's headers

#define __device__
#define __forceinline__ inline
#define __sincosf sincosf
#define HAVE_GPU 1
#define IS_CUDA 1
#define MAX(a, b) (((a) > (b)) ? (a) : (b))  // GLib's, which the reference headers expect
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#include "CUDASkyGeom.h"
#include "CUDABeamInterp.h"

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

// The reference's interpolation of one plane of an image (nx x ny x nplane
// floats, host memory) at pixel (1-relative; pixel[2] = plane number,
// 1-relative), with half-width hwidth: the interpolator is set up as the
// reference's host code sets it (Lagrange denominators as reciprocals, in
// single precision); returns fblank where the reference does.
extern "C" float ref_beam_interp_pixel(const float* data, int nx, int ny, int nplane, float fblank, int hwidth,
                                       const float pixel[3]) {
  CUDAFArray arr;
  memset(&arr, 0, sizeof(arr));
  arr.d_array = const_cast<float*>(data);
  arr.h_array = arr.d_array;
  arr.fblank = fblank;
  arr.ndim = 3;
  arr.naxis[0] = nx;
  arr.naxis[1] = ny;
  arr.naxis[2] = nplane;
  CUDABeamInterp in;
  memset(&in, 0, sizeof(in));
  in.nx = nx;
  in.ny = ny;
  in.hwidth = hwidth;
  const int iwid = 2 * hwidth + 1;
  for (int j = 0; j < iwid; j++) {
    float d = 1.0f;
    for (int i = 0; i < iwid; i++)
      if (i != j) d *= (float)(j - i);
    in.denom[j] = 1.0f / d;
  }
  in.h_myArray = &arr;
  in.d_myArray = &arr;
  float px[3] = {pixel[0], pixel[1], pixel[2]};
  return CUDABeamInterpPixel(&in, px);
}
