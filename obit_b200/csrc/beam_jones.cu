// Jones matrices of every (antenna type, component, beam plane) interpolated
// from beam images: the computation of GetJonesKernel
// (ObitCUDABeamModel.cu:1228-1299) with its pixel geometry (CUDAPositionXYpix,
// CUDASkyGeom.h:91-286; linear and -SIN grids) and Lagrange interpolator
// (CUDABeamInterpPixel / SetConvKernal, CUDABeamInterp.h), written anew.
// One thread per (component, antenna type); the position, its pixel, the
// interpolation kernels and the primary-beam factor's offset are computed
// once, then every plane's 8 images are interpolated with the same taps.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>

#include "abi_internal.h"
#include "obit_dft.h"

namespace obit {
namespace {

constexpr int kMaxTaps = 9;  // 2 hwidth + 1, hwidth <= 4

struct JonesParams {
  int numAntType, nx, ny, nplane, ncomp, hwidth, projection;
  float fblank, refSizeFact, parAng;
  double crval0, crval1;
  float crpix0, crpix1, cdelt0, cdelt1;
  const float* pixels;
  const float* pos;
  float* jones;
  float planeFreq[64];
};
constexpr int kMaxPlanes = 64;

// Pixel (1-relative) of a position (deg), or false when it cannot be
// projected: CUDAPositionXYpixLM (linear: offsets from crval with the 0 h
// wrap; -SIN: direction cosines about crval), then the rotation by parAng
// and the grid's increments and reference pixel (CUDAPositionXYpix).
__device__ bool pixel_of(const JonesParams& p, double x, double y, float& px, float& py) {
  const double d2r = 1.745329252e-2;
  double dx = x - p.crval0;
  if (dx > 180.0) x -= 360.0;
  if (dx < -180.0) x += 360.0;
  double l = x - p.crval0, m = y - p.crval1;
  if (p.projection == 1) {
    const double ra0 = p.crval0 * d2r, dec0 = p.crval1 * d2r, ra = x * d2r, dec = y * d2r;
    const double cd = cos(dec), sd = sin(dec), ca = cos(ra - ra0);
    const double sint = sd * sin(dec0) + cd * cos(dec0) * ca;
    if (sint < 0.0) return false;
    l = sin(ra - ra0) * cd / d2r;
    m = (sd * cos(dec0) - cd * sin(dec0) * ca) / d2r;
  }
  float sr, cr;
  sincosf(p.parAng, &sr, &cr);
  const double lr = l * cr + m * sr;
  const double mr = m * cr - l * sr;
  px = (float)(lr / p.cdelt0 + p.crpix0);
  py = (float)(mr / p.cdelt1 + p.crpix1);
  return true;
}

// Lagrange weights of the iwid taps about pixel (1-relative) on an axis of n
// pixels; start: first tap (0-relative).
__device__ void lagrange_taps(float pix, int n, int hw, int& start, float* w) {
  const int iwid = 2 * hw + 1;
  const int ipos = (int)(pix + 0.5f);
  int cen = ipos - hw;
  cen = max(1, min(cen, n - iwid + 1)) - 1;
  start = cen;
  const float xx = pix - (float)cen;  // 1 at the first tap
  for (int j = 0; j < iwid; j++) {
    float prod = 1.0f, den = 1.0f;
    for (int i = 0; i < iwid; i++)
      if (i != j) {
        prod *= xx - (float)(i + 1);
        den *= (float)(j - i);
      }
    w[j] = prod / den;
  }
}

// Inverse square root of the cos^2 primary-beam gain at offset ang (deg):
// InvBeam (ObitCUDABeamModel.cu:66-72), 100 past the 10 % point.
__device__ float inv_beam(float fact, float freq, float ang) {
  const double arg = (double)fact * freq * ang;
  if (arg > 1.02) return 100.0f;
  return (float)((1.0 - 4.0 * arg * arg) / cos(3.141592653589793 * arg));
}

__device__ __forceinline__ void set_unit(float* J) {
  J[0] = 1.f; J[1] = 0.f; J[2] = 0.f; J[3] = 0.f;
  J[4] = 0.f; J[5] = 0.f; J[6] = 1.f; J[7] = 0.f;
}

__global__ void beam_jones_kernel(const __grid_constant__ JonesParams p) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (c >= p.ncomp || t >= p.numAntType) return;
  float* Jc = p.jones + ((size_t)t * p.ncomp + c) * p.nplane * 8;
  const double x = p.pos[2 * c], y = p.pos[2 * c + 1];
  float px, py;
  const bool onGrid = pixel_of(p, x, y, px, py) && px >= 1.0f && px <= (float)p.nx && py >= 1.0f &&
                      py <= (float)p.ny;
  if (!onGrid) {
    for (int k = 0; k < p.nplane; k++) set_unit(Jc + 8 * k);
    return;
  }
  const int iwid = 2 * p.hwidth + 1;
  int xs, ys;
  float wx[kMaxTaps], wy[kMaxTaps];
  lagrange_taps(px, p.nx, p.hwidth, xs, wx);
  lagrange_taps(py, p.ny, p.hwidth, ys, wy);
  const float ang = sqrtf((float)(x * x + y * y));
  const size_t img = (size_t)p.nplane * p.ny * p.nx;
  const float* base = p.pixels + (size_t)t * 8 * img;
  for (int k = 0; k < p.nplane; k++) {
    float v[8];
    bool blank = false;
    for (int q = 0; q < 8; q++) {
      const float* d = base + q * img + (size_t)k * p.ny * p.nx;
      float sum = 0.f, sumwt = 0.f;
      for (int j = 0; j < iwid; j++) {
        const float* row = d + (size_t)(ys + j) * p.nx + xs;
        for (int i = 0; i < iwid; i++) {
          const float val = row[i];
          if (val != p.fblank) {
            const float wt = wx[i] * wy[j];
            sumwt += wt;
            sum += val * wt;
          }
        }
      }
      if (sumwt > 0.90f) v[q] = sum / sumwt;
      else blank = true;
    }
    const float g = inv_beam(p.refSizeFact, p.planeFreq[k], ang);
    float* J = Jc + 8 * k;
    if (blank || !(g < 10.0f) || !(fabsf(g * v[0]) <= 1.3f) || !(fabsf(g * v[2]) <= 1.3f)) {
      set_unit(J);
      continue;
    }
    // cudaMatxSet2C order: P1, X1, X2, P2 (XX, XY, YX, YY)
    J[0] = g * v[0]; J[1] = g * v[1];
    J[2] = g * v[4]; J[3] = g * v[5];
    J[4] = g * v[6]; J[5] = g * v[7];
    J[6] = g * v[2]; J[7] = g * v[3];
  }
}

}  // namespace
}  // namespace obit

extern "C" int obit_dft_beam_jones(const ObitDFTBeamImages* im, const float* pos, int ncomp, float parAng,
                                   float* jones, void* stream) {
  using namespace obit;
  set_last_error("");
  auto bad = [](int code, const char* msg) {
    set_last_error(msg);
    return code;
  };
  if (!im || !pos || !jones || !im->pixels || !im->planeFreq) return bad(OBIT_DFT_EBADARG, "NULL beam-image argument");
  if (ncomp < 0) return bad(OBIT_DFT_EBADARG, "negative component count");
  if (im->numAntType < 1 || im->nplane < 1) return bad(OBIT_DFT_EBADARG, "no antenna types or planes");
  if (im->nplane > kMaxPlanes) return bad(OBIT_DFT_EUNSUPPORTED, "more than 64 beam planes");
  if (im->hwidth < 1 || im->hwidth > 4) return bad(OBIT_DFT_EBADARG, "interpolation half-width must be 1..4");
  if (im->nx < 2 * im->hwidth + 1 || im->ny < 2 * im->hwidth + 1)
    return bad(OBIT_DFT_EBADARG, "beam images smaller than the interpolation kernel");
  if (im->projection != 0 && im->projection != 1) return bad(OBIT_DFT_EUNSUPPORTED, "projection must be 0 or 1");
  if (!(im->cdelt[0] != 0.0f) || !(im->cdelt[1] != 0.0f)) return bad(OBIT_DFT_EBADARG, "zero pixel increment");
  if (((uintptr_t)jones & 15u) != 0) return bad(OBIT_DFT_EBADARG, "Jones table not 16-byte aligned");
  if (ncomp == 0) return OBIT_DFT_OK;
  JonesParams p{};
  p.numAntType = im->numAntType;
  p.nx = im->nx;
  p.ny = im->ny;
  p.nplane = im->nplane;
  p.ncomp = ncomp;
  p.hwidth = im->hwidth;
  p.projection = im->projection;
  p.fblank = im->fblank;
  p.refSizeFact = im->refSizeFact;
  p.parAng = parAng;
  p.crval0 = im->crval[0];
  p.crval1 = im->crval[1];
  p.crpix0 = im->crpix[0];
  p.crpix1 = im->crpix[1];
  p.cdelt0 = im->cdelt[0];
  p.cdelt1 = im->cdelt[1];
  p.pixels = im->pixels;
  p.pos = pos;
  p.jones = jones;
  for (int k = 0; k < im->nplane; k++) p.planeFreq[k] = im->planeFreq[k];
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) return bad(OBIT_DFT_ECUDA, cudaGetErrorString(ce));
  const dim3 grid((unsigned)((ncomp + 127) / 128), (unsigned)im->numAntType);
  beam_jones_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(p);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    set_last_error(std::string("beam Jones kernel launch: ") + cudaGetErrorString(ce));
    return OBIT_DFT_ECUDA;
  }
  return OBIT_DFT_OK;
}
