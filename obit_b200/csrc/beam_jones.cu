// Jones matrices of every (antenna type, component, beam plane) interpolated
// from beam images: the computation of GetJonesKernel
// (ObitCUDABeamModel.cu:1228-1299) with its pixel geometry (CUDAPositionXYpix,
// CUDASkyGeom.h:91-286; linear grids and the eight projections) and Lagrange interpolator
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
  float fblank, refSizeFact, parAng, crota;
  double crval0, crval1;
  float crpix0, crpix1, cdelt0, cdelt1;
  const float* pixels;
  const float* pos;
  float* jones;
  float planeFreq[64];
};
constexpr int kMaxPlanes = 64;

// Offsets (deg) of a position (deg) from the grid's reference position in
// the grid's projection, or false where it cannot be projected: the linear
// offsets after the 0 h wrap, or for projections 1..8 (-SIN, -TAN, -ARC,
// -NCP, -GLS, -MER, -AIT, -STG) the projected coordinates of the standard
// AIPS definitions scaled back to degrees, as CUDAPositionXYpixLM
// (CUDASkyGeom.h:91-250) forms them; crota (deg) enters only the -MER and
// -AIT scale factors.
__device__ bool grid_offsets(const JonesParams& p, double x, double y, double& l, double& m) {
  const double d2r = 1.745329252e-2, halfPi = 6.28318530717959 / 4.0, eps = 1.0e-5;
  const double dx = x - p.crval0;
  if (dx > 180.0) x -= 360.0;
  if (dx < -180.0) x += 360.0;
  l = x - p.crval0;
  m = y - p.crval1;
  if (p.projection == 0) return true;
  const double ra0 = p.crval0 * d2r, dec0 = p.crval1 * d2r, ra = x * d2r, dec = y * d2r;
  const double cd = cos(dec), sd = sin(dec), cd0 = cos(dec0), sd0 = sin(dec0);
  const double da = ra - ra0, ca = cos(da);
  const double cosAlt = sd * sd0 + cd * cd0 * ca;  // cosine of the angle from the reference
  const double mNorth = sd * cd0 - cd * sd0 * ca;   // north component of the direction
  double L = sin(da) * cd, M = 0.0;
  switch (p.projection) {
    case 1:  // -SIN: orthographic
      if (cosAlt < 0.0) return false;
      M = mNorth;
      break;
    case 2:  // -TAN: gnomonic
      if (cosAlt <= 0.0) return false;
      L /= cosAlt;
      M = mNorth / cosAlt;
      break;
    case 3: {  // -ARC: zenithal equidistant
      const double th = acos(fmin(1.0, fmax(-1.0, cosAlt)));
      const double f = th != 0.0 ? th / sin(th) : 1.0;
      L *= f;
      M = mNorth * f;
      break;
    }
    case 4:  // -NCP: north celestial pole
      if (dec0 == 0.0) return false;
      M = (cd0 - cd * ca) / sd0;
      break;
    case 5:  // -GLS: global sinusoid
      if (fabs(dec) > halfPi || fabs(dec0) > halfPi) return false;
      L = da * cd;
      M = dec - dec0;
      break;
    case 6: {  // -MER: Mercator, scaled to the grid's increment along y
      const double r = p.crota * d2r;
      double step = p.cdelt1 * cos(r) + p.cdelt0 * sin(r);
      if (step == 0.0) step = 1.0;
      const double y0 = (p.crval1 / 2.0 + 45.0) * d2r;
      const double ly0 = log(tan(y0)), ly1 = log(tan(y0 + step / 2.0 * d2r));
      const double gy = step * d2r / (ly1 - ly0);
      double gx = cos(p.crval1 * d2r);
      if (gx <= 0.0) gx = 1.0;
      const double t = tan(dec / 2.0 + halfPi / 2.0);
      if (t < eps) return false;
      L = gx * da;
      M = gy * log(t) - gy * ly0;
      break;
    }
    case 7: {  // -AIT: Hammer-Aitoff, scaled to the grid's increments
      const double half = da / 2.0;
      if (fabs(half) > halfPi) return false;
      const double r = p.crota * d2r, cr = cos(r), sr = sin(r);
      const double yc = p.crval1 * d2r;
      double sy = p.cdelt1 * cr + p.cdelt0 * sr;
      if (sy == 0.0) sy = 1.0;
      sy *= d2r;
      double ny = sin(yc + sy) / sqrt((1.0 + cos(yc + sy)) / 2.0) - sin(yc) / sqrt((1.0 + cos(yc)) / 2.0);
      if (ny == 0.0) ny = 1.0;
      const double gy = sy / ny;
      double sx = p.cdelt0 * cr - p.cdelt1 * sr;
      if (sx == 0.0) sx = 1.0;
      sx *= d2r;
      double nx = 2.0 * cos(yc) * sin(sx / 2.0);
      if (nx == 0.0) nx = 1.0;
      const double gx = sx * sqrt((1.0 + cos(yc) * cos(sx / 2.0)) / 2.0) / nx;
      const double y0 = gy * sin(yc) / sqrt((1.0 + cos(yc)) / 2.0);
      const double z = sqrt((1.0 + cd * cos(half)) / 2.0);
      if (fabs(z) < eps) return false;
      L = 2.0 * gx * cd * sin(half) / z;
      M = gy * sd / z - y0;
      break;
    }
    case 8: {  // -STG: stereographic
      if (fabs(dec) > halfPi) return false;
      const double den = 1.0 + cosAlt;
      if (fabs(den) < eps) return false;
      L *= 2.0 / den;
      M = mNorth * 2.0 / den;
      break;
    }
    default:
      return false;
  }
  l = L / d2r;
  m = M / d2r;
  return true;
}

// Pixel (1-relative) of a position (deg), or false when it cannot be
// projected: the grid offsets rotated by the parallactic angle, then the
// grid's increments and reference pixel (CUDAPositionXYpix,
// CUDASkyGeom.h:266-286).
__device__ bool pixel_of(const JonesParams& p, double x, double y, float& px, float& py) {
  double l, m;
  if (!grid_offsets(p, x, y, l, m)) return false;
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
  if (im->projection < 0 || im->projection > 8) return bad(OBIT_DFT_EUNSUPPORTED, "projection must be 0..8");
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
  p.crota = im->crota;
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
