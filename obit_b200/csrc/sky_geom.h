// Field geometry shared by the component loader and the gridded model: the
// phase-centre shift terms of a -SIN field and the 3-D re-projection matrices,
// at the reference's single- and double-precision rounding points.  Included
// only by host files compiled without floating-point contraction.
#pragma once
#include <cmath>

namespace obit {
namespace geom {

constexpr double kGeomPi = 3.14159265358979323846;

// ObitSkyGeomShiftSIN (ObitSkyGeom.c:177-205): FP64 direction cosines of the
// field centre in the map frame, FP32 phase-shift terms 2 pi (l, m, n - 1).
inline void shift_sin(double ra, double dec, float rotate, double xra, double xdec, float dxyzc[3]) {
  // the reference's DG2RAD macro expands unparenthesized: rotate * pi / 180
  const float maprr = (float)(rotate * kGeomPi / 180.0);
  const double d2r = kGeomPi / 180.0;
  const double xxshft = std::cos(d2r * xdec) * std::sin(d2r * (xra - ra));
  const double yyshft = std::sin(d2r * xdec) * std::cos(d2r * dec) -
                        std::cos(d2r * xdec) * std::sin(d2r * dec) * std::cos(d2r * (xra - ra));
  const float xshift = (float)(std::cos((double)maprr) * xxshft + std::sin((double)maprr) * yyshft);
  const float yshift = (float)(-std::sin((double)maprr) * xxshft + std::cos((double)maprr) * yyshft);
  const float x2 = xshift * xshift, y2 = yshift * yshift;  // single-precision squares
  const double dz = std::sqrt(1.0 - (double)x2 - (double)y2);
  dxyzc[0] = (float)(2.0 * kGeomPi * (double)xshift);
  dxyzc[1] = (float)(2.0 * kGeomPi * (double)yshift);
  dxyzc[2] = (float)(2.0 * kGeomPi * (dz - 1.0));
}

// The same shift terms with no single-precision rounding (FP64 positions).
inline void shift_sin_d(double ra, double dec, float rotate, double xra, double xdec, double dxyzc[3]) {
  const double maprr = (double)rotate * kGeomPi / 180.0;
  const double d2r = kGeomPi / 180.0;
  const double xxshft = std::cos(d2r * xdec) * std::sin(d2r * (xra - ra));
  const double yyshft = std::sin(d2r * xdec) * std::cos(d2r * dec) -
                        std::cos(d2r * xdec) * std::sin(d2r * dec) * std::cos(d2r * (xra - ra));
  const double xshift = std::cos(maprr) * xxshft + std::sin(maprr) * yyshft;
  const double yshift = -std::sin(maprr) * xxshft + std::cos(maprr) * yyshft;
  const double dz = std::sqrt(1.0 - xshift * xshift - yshift * yshift);
  dxyzc[0] = 2.0 * kGeomPi * xshift;
  dxyzc[1] = 2.0 * kGeomPi * yshift;
  dxyzc[2] = 2.0 * kGeomPi * (dz - 1.0);
}

// rm of ObitUVDescShift3DMatrix: rotation by r with rm[0][1] = sign sin r.
inline void rot_matrix(double r, double sign, double rm[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) rm[i][j] = 0.0;
  rm[2][2] = 1.0;
  rm[0][0] = std::cos(r);
  rm[1][1] = rm[0][0];
  rm[1][0] = -sign * std::sin(r);
  rm[0][1] = sign * std::sin(r);
}

// out[j][i] = sum_k rm2[k][i] (sum_l x[l][i'] ...): the two products of
// ObitUVDescShift3DMatrix, t[j][i] = sum_k x[k][i] rm1[j][k], then
// out[j][i] = sum_k rm2[k][i] t[j][k], FP64 sums in the reference's order.
template <typename T>
void matrix_chain(const double x[3][3], const double rm1[3][3], const double rm2[3][3], T out[3][3]) {
  double t[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      t[j][i] = 0.0;
      for (int k = 0; k < 3; k++) t[j][i] += x[k][i] * rm1[j][k];
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++) s += rm2[k][i] * t[j][k];
      out[j][i] = (T)s;
    }
}

// ObitUVDescShift3DMatrix, 3-D image branch (ObitUVDesc.c:913-978): the uv
// re-projection matrix R(map +) X R(uv -), FP64 products in the reference's
// summation order, stored as T.
template <typename T>
void urot3d(double ra, double dec, double xra, double xdec, float mrot, float urot, T U[3][3]) {
  const double d2r = kGeomPi / 180.0;
  const double sa = std::sin(d2r * (xra - ra)), ca = std::cos(d2r * (xra - ra));
  const double sd = std::sin(d2r * xdec), cd = std::cos(d2r * xdec);
  const double sd0 = std::sin(d2r * dec), cd0 = std::cos(d2r * dec);
  double x[3][3], r1[3][3], r2[3][3];
  x[0][0] = ca;
  x[1][0] = -sd * sa;
  x[2][0] = cd * sa;
  x[0][1] = sd0 * sa;
  x[1][1] = cd * cd0 + sd * sd0 * ca;
  x[2][1] = sd * cd0 - cd * sd0 * ca;
  x[0][2] = -cd0 * sa;
  x[1][2] = cd * sd0 - sd * cd0 * ca;
  x[2][2] = sd * sd0 + cd * cd0 * ca;
  rot_matrix(d2r * (double)mrot, 1.0, r1);
  rot_matrix(d2r * (double)urot, -1.0, r2);
  matrix_chain(x, r1, r2, U);
}

// The image-plane matrix of the same call (ObitUVDesc.c:978-1020): the
// backward product R(uv +) X' R(map -), used to turn a field offset into the
// re-projected frame.
template <typename T>
void prot3d(double ra, double dec, double xra, double xdec, float mrot, float urot, T P[3][3]) {
  const double d2r = kGeomPi / 180.0;
  const double sa = std::sin(d2r * (xra - ra)), ca = std::cos(d2r * (xra - ra));
  const double sd = std::sin(d2r * xdec), cd = std::cos(d2r * xdec);
  const double sd0 = std::sin(d2r * dec), cd0 = std::cos(d2r * dec);
  double x[3][3], r1[3][3], r2[3][3];
  x[0][0] = ca;
  x[1][0] = sd0 * sa;
  x[2][0] = -cd0 * sa;
  x[0][1] = -sd * sa;
  x[1][1] = cd * cd0 + sd * sd0 * ca;
  x[2][1] = sd0 * cd - cd0 * sd * ca;
  x[0][2] = cd * sa;
  x[1][2] = cd0 * sd - sd0 * cd * ca;
  x[2][2] = sd * sd0 + cd * cd0 * ca;
  rot_matrix(d2r * (double)urot, 1.0, r1);
  rot_matrix(d2r * (double)mrot, -1.0, r2);
  matrix_chain(x, r1, r2, P);
}

}  // namespace geom
}  // namespace obit
