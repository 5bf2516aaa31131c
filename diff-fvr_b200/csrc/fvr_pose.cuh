// FP64 rigid-pose helpers shared by the parallel-beam and cone-beam kernels.
#pragma once

#include "fvr_common.cuh"

namespace fvr {

constexpr double kDeg = 0.017453292519943295769236907684886;

struct Mat3 {
  double m[3][3];
};

__device__ __forceinline__ Mat3 mat_mul(const Mat3& a, const Mat3& b) {
  Mat3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
  return r;
}

// a . b^T
__device__ __forceinline__ Mat3 mat_mul_bt(const Mat3& a, const Mat3& b) {
  Mat3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[j][0] + a.m[i][1] * b.m[j][1] + a.m[i][2] * b.m[j][2];
  return r;
}

__device__ __forceinline__ Mat3 rot_z(double c, double s) { return Mat3{{{c, -s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}}}; }
__device__ __forceinline__ Mat3 rot_y(double c, double s) { return Mat3{{{c, 0.0, s}, {0.0, 1.0, 0.0}, {-s, 0.0, c}}}; }
__device__ __forceinline__ Mat3 rot_x(double c, double s) { return Mat3{{{1.0, 0.0, 0.0}, {0.0, c, -s}, {0.0, s, c}}}; }
__device__ __forceinline__ Mat3 drot_z(double c, double s) {
  return Mat3{{{-s, -c, 0.0}, {c, -s, 0.0}, {0.0, 0.0, 0.0}}};
}
__device__ __forceinline__ Mat3 drot_y(double c, double s) {
  return Mat3{{{-s, 0.0, c}, {0.0, 0.0, 0.0}, {-c, 0.0, -s}}};
}
__device__ __forceinline__ Mat3 drot_x(double c, double s) {
  return Mat3{{{0.0, 0.0, 0.0}, {0.0, -s, -c}, {0.0, c, -s}}};
}

// Rz(90 deg) exactly as src/fvr/torch_engine.py:194-198 forms it: the angle
// 90 * (pi/180) is rounded to float32 (1.5707963705062866, i.e. pi/2 + 4.37e-8)
// and its cos/sin are taken in float32, giving cos = -4.371138828673793e-08
// (= -(fl32(pi/2) - pi/2) rounded to float32) and sin = 1.
__device__ __forceinline__ Mat3 lateral_rot() { return rot_z(-4.371138828673793e-08, 1.0); }

// sin/cos of an angle in degrees: sincospi(deg / 180) needs no large-argument
// range reduction and is exact at multiples of 90 degrees.
__device__ __forceinline__ void sincos_deg(double deg, double* s, double* c) { sincospi(deg / 180.0, s, c); }

// R = Rz(yaw) Ry(pitch) Rx(roll), angles in degrees (torch_engine.py:139-174).
__device__ __forceinline__ Mat3 euler_R(double yaw, double pitch, double roll) {
  double sz, cz, sy, cy, sx, cx;
  sincos_deg(yaw, &sz, &cz);
  sincos_deg(pitch, &sy, &cy);
  sincos_deg(roll, &sx, &cx);
  return mat_mul(rot_z(cz, sz), mat_mul(rot_y(cy, sy), rot_x(cx, sx)));
}

// R and dR/d(yaw, pitch, roll) (per radian) from one set of sines / cosines.
__device__ __forceinline__ void euler_R_jac(double yaw, double pitch, double roll, Mat3* R, Mat3 dR[3]) {
  double sz, cz, sy, cy, sx, cx;
  sincos_deg(yaw, &sz, &cz);
  sincos_deg(pitch, &sy, &cy);
  sincos_deg(roll, &sx, &cx);
  const Mat3 Z = rot_z(cz, sz), Y = rot_y(cy, sy), X = rot_x(cx, sx);
  const Mat3 YX = mat_mul(Y, X);
  *R = mat_mul(Z, YX);
  dR[0] = mat_mul(drot_z(cz, sz), YX);
  dR[1] = mat_mul(Z, mat_mul(drot_y(cy, sy), X));
  dR[2] = mat_mul(Z, mat_mul(Y, drot_x(cx, sx)));
}

// d<G, R>/d(yaw, pitch, roll), per degree.
__device__ __forceinline__ void euler_vjp(double yaw, double pitch, double roll, const Mat3& G, double out[3]) {
  double sz, cz, sy, cy, sx, cx;
  sincos_deg(yaw, &sz, &cz);
  sincos_deg(pitch, &sy, &cy);
  sincos_deg(roll, &sx, &cx);
  const Mat3 Z = rot_z(cz, sz), Y = rot_y(cy, sy), X = rot_x(cx, sx);
  const Mat3 dz = mat_mul(drot_z(cz, sz), mat_mul(Y, X));
  const Mat3 dy = mat_mul(Z, mat_mul(drot_y(cy, sy), X));
  const Mat3 dx = mat_mul(Z, mat_mul(Y, drot_x(cx, sx)));
  double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      a += G.m[i][j] * dz.m[i][j];
      b += G.m[i][j] * dy.m[i][j];
      c += G.m[i][j] * dx.m[i][j];
    }
  out[0] = a * kDeg;
  out[1] = b * kDeg;
  out[2] = c * kDeg;
}

}  // namespace fvr
