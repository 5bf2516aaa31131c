/*
 * Oracle (test infrastructure only): plain-C, OpenMP restatement of the
 * parallel-beam zero-IFFT spectral NCC loss and its pose gradient, in double
 * precision.  Used as the timed CPU baseline and as a fast full-size checker;
 * never linked into the product.
 *
 * Restates, per candidate and view:
 *   src/fvr/torch_engine.py:139-174  R = Rz(yaw) Ry(pitch) Rx(roll) (degrees)
 *   src/fvr/torch_engine.py:194-211  lateral R . Rz(90deg) (float32 cos/sin),
 *                                    u = R[0]*(W-1,H-1,D-1)/2, v = R[1]*(...)
 *   src/fvr/triton_slice.py:664-715  zero-padding trilinear gather
 *   src/fvr/torch_engine.py:227-234  phase ramp -2pi(ku tx + kv ty)/(R sp + 1e-6)
 *   src/fvr/torch_engine.py:269-290  HP filter, NCC, loss = 1 - mean ncc
 * and the adjoint the reference gets from autograd (per-sample chain rule:
 * forward pass for the moments, second pass for the gradient).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define DEG 0.017453292519943295769236907684886

static void mat_mul(const double a[3][3], const double b[3][3], double r[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}

static void euler(double yaw, double pitch, double roll, double R[3][3], double dR[3][3][3]) {
  double cz = cos(yaw * DEG), sz = sin(yaw * DEG), cy = cos(pitch * DEG), sy = sin(pitch * DEG);
  double cx = cos(roll * DEG), sx = sin(roll * DEG);
  double Z[3][3] = {{cz, -sz, 0}, {sz, cz, 0}, {0, 0, 1}}, Y[3][3] = {{cy, 0, sy}, {0, 1, 0}, {-sy, 0, cy}};
  double X[3][3] = {{1, 0, 0}, {0, cx, -sx}, {0, sx, cx}};
  double dZ[3][3] = {{-sz, -cz, 0}, {cz, -sz, 0}, {0, 0, 0}}, dY[3][3] = {{-sy, 0, cy}, {0, 0, 0}, {-cy, 0, -sy}};
  double dX[3][3] = {{0, 0, 0}, {0, -sx, -cx}, {0, cx, -sx}};
  double t[3][3], u[3][3];
  mat_mul(Y, X, t);
  mat_mul(Z, t, R);
  if (!dR) return;
  mat_mul(dZ, t, dR[0]);
  mat_mul(dY, X, u);
  mat_mul(Z, u, dR[1]);
  mat_mul(Y, dX, u);
  mat_mul(Z, u, dR[2]);
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dR[k][i][j] *= DEG;
}

static void lateral(double L[3][3]) {
  float a = 90.0f * (float)DEG;
  double c = (double)cosf(a), s = (double)sinf(a);
  double M[3][3] = {{c, -s, 0}, {s, c, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) L[i][j] = M[i][j];
}

/* zero-padding trilinear value and derivatives of the complex spectrum */
static void sample(const double* spec, int D, int H, int W, double px, double py, double pz, double s[2],
                   double d[3][2]) {
  double fx = floor(px), fy = floor(py), fz = floor(pz);
  double tx = px - fx, ty = py - fy, tz = pz - fz;
  long ix = (long)fx, iy = (long)fy, iz = (long)fz;
  size_t plane = (size_t)D * H * W;
  s[0] = s[1] = 0;
  for (int k = 0; k < 3; ++k) d[k][0] = d[k][1] = 0;
  for (int c = 0; c < 8; ++c) {
    int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
    long z = iz + dz, y = iy + dy, x = ix + dx;
    if (z < 0 || z >= D || y < 0 || y >= H || x < 0 || x >= W) continue;
    size_t idx = ((size_t)z * H + y) * W + x;
    double vr = spec[idx], vi = spec[plane + idx];
    double wx = dx ? tx : 1 - tx, wy = dy ? ty : 1 - ty, wz = dz ? tz : 1 - tz;
    double sx = dx ? 1 : -1, sy = dy ? 1 : -1, sz = dz ? 1 : -1;
    double w = wx * wy * wz;
    s[0] += w * vr;
    s[1] += w * vi;
    d[0][0] += sx * wy * wz * vr;
    d[0][1] += sx * wy * wz * vi;
    d[1][0] += wx * sy * wz * vr;
    d[1][1] += wx * sy * wz * vi;
    d[2][0] += wx * wy * sz * vr;
    d[2][1] += wx * wy * sz * vi;
  }
}

/*
 * spec   : planar [2][D][H][W] centred spectrum (double)
 * poses  : [C][6] (yaw, pitch, roll deg; tx, ty, tz)
 * ftarg  : [R*R][2] target spectrum (already high-passed); hp: [R*R] or NULL
 * g      : upstream dL/dloss; grad: [C][6] or NULL (loss only)
 * returns the loss 1 - mean_c ncc_c; ncc: [C] or NULL
 */
double fvr_oracle_sncc(const double* spec, int D, int H, int W, const double* poses, int C, int view,
                       const double* ftarg, const double* hp, int R, double spacing0, double g, double* ncc,
                       double* grad, int threads) {
  const double sc[3] = {0.5 * (W > 1 ? W - 1 : 1), 0.5 * (H > 1 ? H - 1 : 1), 0.5 * (D > 1 ? D - 1 : 1)};
  const double kap = -2.0 * M_PI / (R * spacing0 + 1e-6);
  double* lin = (double*)malloc(sizeof(double) * R);
  /* the float32 values of torch.linspace(-1, 1, R): a float32 step, each value
   * rounded once to float32 from the exact start + step i (lower half) or
   * end - step (R - 1 - i) (upper half) */
  const float step = R > 1 ? 2.0f / (float)(R - 1) : 0.0f;
  for (int i = 0; i < R; ++i)
    lin[i] = R == 1 ? -1.0
                    : (double)(float)(i < R / 2 ? -1.0 + (double)step * i : 1.0 - (double)step * (R - 1 - i));
  double et = 0;
  for (int q = 0; q < R * R; ++q) et += ftarg[2 * q] * ftarg[2 * q] + ftarg[2 * q + 1] * ftarg[2 * q + 1];
  double nsum = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nsum)
#endif
  for (int c = 0; c < C; ++c) {
    const double* p = poses + 6 * c;
    double Rp[3][3], dR[3][3][3], Rt[3][3], Lm[3][3];
    euler(p[0], p[1], p[2], Rp, dR);
    if (view) {
      lateral(Lm);
      mat_mul(Rp, Lm, Rt);
    } else {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[i][j] = Rp[i][j];
    }
    double u[3], v[3];
    for (int k = 0; k < 3; ++k) {
      u[k] = Rt[0][k] * sc[k];
      v[k] = Rt[1][k] * sc[k];
    }
    double cross = 0, ep = 0;
    for (int pass = 0; pass < (grad ? 2 : 1); ++pass) {
      double a = 0, b = 0, gc = -g / C;
      if (pass == 1) {
        double s_ = sqrt(ep * et);
        a = 1.0 / (s_ + 1e-8);
        b = s_ > 0 ? -cross * et / (2.0 * s_ * (s_ + 1e-8) * (s_ + 1e-8)) : 0.0;
      }
      double du[3] = {0, 0, 0}, dv[3] = {0, 0, 0}, dtx = 0, dty = 0;
      for (int i = 0; i < R; ++i) {
        for (int j = 0; j < R; ++j) {
          int q = i * R + j;
          double ku = lin[i], kv = lin[j];
          double s[2], d[3][2];
          sample(spec, D, H, W, sc[0] + ku * u[0] + kv * v[0], sc[1] + ku * u[1] + kv * v[1],
                 sc[2] + ku * u[2] + kv * v[2], s, d);
          double ph = kap * (ku * p[3] + kv * p[4]);
          double cs = cos(ph), sn = sin(ph), h = hp ? hp[q] : 1.0;
          double shr = h * (s[0] * cs - s[1] * sn), shi = h * (s[0] * sn + s[1] * cs);
          double tr = ftarg[2 * q], ti = ftarg[2 * q + 1];
          if (pass == 0) {
            cross += shr * tr + shi * ti;
            ep += shr * shr + shi * shi;
          } else {
            double Gr = gc * (a * tr + 2 * b * shr), Gi = gc * (a * ti + 2 * b * shi);
            /* dL/dS = h e^{-i ph} G ; dL/dph = Re(conj(G) i S_hat) */
            double lr = h * (cs * Gr + sn * Gi), li = h * (cs * Gi - sn * Gr);
            double dph = Gi * shr - Gr * shi;
            dtx += dph * kap * ku;
            dty += dph * kap * kv;
            for (int k = 0; k < 3; ++k) {
              double e = lr * d[k][0] + li * d[k][1];
              du[k] += ku * e;
              dv[k] += kv * e;
            }
          }
        }
      }
      if (pass == 1) {
        double gR[3][3] = {{du[0] * sc[0], du[1] * sc[1], du[2] * sc[2]},
                           {dv[0] * sc[0], dv[1] * sc[1], dv[2] * sc[2]},
                           {0, 0, 0}};
        if (view) { /* dL/dR_pose = dL/dR_total . L^T */
          double t[3][3];
          for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y) t[x][y] = gR[x][0] * Lm[y][0] + gR[x][1] * Lm[y][1] + gR[x][2] * Lm[y][2];
          for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y) gR[x][y] = t[x][y];
        }
        for (int k = 0; k < 3; ++k) {
          double acc = 0;
          for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y) acc += gR[x][y] * dR[k][x][y];
          grad[6 * c + k] = acc;
        }
        grad[6 * c + 3] = dtx;
        grad[6 * c + 4] = dty;
        grad[6 * c + 5] = 0;
      }
    }
    double n = cross / (sqrt(ep * et) + 1e-8);
    if (ncc) ncc[c] = n;
    nsum += n;
  }
  free(lin);
  return 1.0 - nsum / C;
}
