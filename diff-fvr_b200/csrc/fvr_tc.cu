// Parallel-beam (torch-engine convention) kernels, sm_100a.
//
//  * stencil layout build from a centred complex spectrum (+ f16 brick scales)
//  * drop-in fourier_slice_3d forward / adjoint on the reference's planar
//    [B_vol, 2, D, H, W] layout        (src/fvr/triton_slice.py:37-339)
//  * fused zero-IFFT spectral NCC: slice gather + phase ramp + high-pass +
//    NCC moments (+ pose-gradient moments) in one pass over the samples
//                                      (src/fvr/torch_engine.py:176-234, 269-307)
//  * image path: modulated slice written in ifftshift order for the 2D IFFT,
//    and the per-sample slice adjoint  (src/fvr/torch_engine.py:236-241)
//  * FP64 pose maps: Euler (yaw Z, pitch Y, roll X) -> slice axes and the
//    Euler Jacobian of the pose gradient (src/fvr/torch_engine.py:139-211)
#include "fvr_stencil.cuh"

namespace fvr {

// ----------------------------------------------------------------------------
// stencil build
// ----------------------------------------------------------------------------

// master spectrum: planar [2][D][H][W] (the reference's f_vol_5d[0]) or
// interleaved [D][H][W][2]
template <typename MT>
__device__ __forceinline__ float2 master_load(const MT* m, int64_t idx, int64_t plane) {
  return plane ? make_float2(ldf(m + idx), ldf(m + plane + idx)) : make_float2(ldf(m + 2 * idx), ldf(m + 2 * idx + 1));
}

template <typename MT>
__device__ __forceinline__ void entry_values(const MT* m, int64_t plane, int D, int H, int W, int ez, int ey, int ex,
                                             float (&re)[8], float (&im)[8]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int z = ez - 1 + (c >> 2), y = ey - 1 + ((c >> 1) & 1), x = ex - 1 + (c & 1);
    if (z >= 0 && z < D && y >= 0 && y < H && x >= 0 && x < W) {
      float2 v = master_load(m, (static_cast<int64_t>(z) * H + y) * W + x, plane);
      re[c] = v.x;
      im[c] = v.y;
    } else {
      re[c] = 0.f;
      im[c] = 0.f;
    }
  }
}

template <typename MT>
__global__ void stencil_brick_max_kernel(const MT* __restrict__ m, int64_t plane, int D, int H, int W,
                                         unsigned int* bmax) {
  const int64_t n = static_cast<int64_t>(D + 1) * (H + 1) * (W + 1);
  const int bx = (W + 1 + kBrick - 1) / kBrick, by = (H + 1 + kBrick - 1) / kBrick;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int ex = static_cast<int>(e % (W + 1));
    const int ey = static_cast<int>((e / (W + 1)) % (H + 1));
    const int ez = static_cast<int>(e / (static_cast<int64_t>(W + 1) * (H + 1)));
    float re[8], im[8];
    entry_values(m, plane, D, H, W, ez, ey, ex, re, im);
    float mx = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) mx = fmaxf(mx, fmaxf(fabsf(re[c]), fabsf(im[c])));
    const int64_t b = (static_cast<int64_t>(ez / kBrick) * by + ey / kBrick) * bx + ex / kBrick;
    atomicMax(bmax + b, __float_as_uint(mx));  // non-negative floats order like their bits
  }
}

// scale = 2^e with max/scale <= 2^15 (half max is 65504); exact to apply.
__global__ void stencil_scale_kernel(const unsigned int* bmax, float* scales, int64_t nb) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= nb) return;
  const float mx = __uint_as_float(bmax[i]);
  float sc = 1.f;
  if (mx > 0.f && isfinite(mx)) {
    int e;
    frexpf(mx, &e);  // mx = f * 2^e, f in [0.5, 1)
    sc = ldexpf(1.f, e - 15);
  }
  scales[i] = sc;
}

template <typename MT, int DT>
__global__ void stencil_build_kernel(const MT* __restrict__ m, int64_t plane, int D, int H, int W,
                                     void* __restrict__ out, const float* __restrict__ scales) {
  const int64_t n = static_cast<int64_t>(D + 1) * (H + 1) * (W + 1);
  const int bx = (W + 1 + kBrick - 1) / kBrick, by = (H + 1 + kBrick - 1) / kBrick;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int ex = static_cast<int>(e % (W + 1));
    const int ey = static_cast<int>((e / (W + 1)) % (H + 1));
    const int ez = static_cast<int>(e / (static_cast<int64_t>(W + 1) * (H + 1)));
    float re[8], im[8];
    entry_values(m, plane, D, H, W, ez, ey, ex, re, im);
    if constexpr (DT == FVR_F32) {
      float4* p = static_cast<float4*>(out) + e * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) p[i] = make_float4(re[2 * i], im[2 * i], re[2 * i + 1], im[2 * i + 1]);
    } else {
      uint32_t w[8];
      if constexpr (DT == FVR_BF16) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(re[c]));
          const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(im[c]));
          w[c] = lo | (hi << 16);
        }
      } else {
        const float inv = 1.f / scales[(static_cast<int64_t>(ez / kBrick) * by + ey / kBrick) * bx + ex / kBrick];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t lo = __half_as_ushort(__float2half_rn(re[c] * inv));
          const uint32_t hi = __half_as_ushort(__float2half_rn(im[c] * inv));
          w[c] = lo | (hi << 16);
        }
      }
      uint4* p = static_cast<uint4*>(out) + e * 2;
      p[0] = make_uint4(w[0], w[1], w[2], w[3]);
      p[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
}

// ----------------------------------------------------------------------------
// drop-in planar gather  (triton_slice.py:46-143, 145-271)
// ----------------------------------------------------------------------------

template <typename VT>
__device__ __forceinline__ float planar_at(const VT* ch, int D, int H, int W, int z, int y, int x) {
  if (z < 0 || z >= D || y < 0 || y >= H || x < 0 || x >= W) return 0.f;
  return ldf(ch + (static_cast<int64_t>(z) * H + y) * W + x);
}

template <typename VT>
__device__ __forceinline__ void planar_corners(const VT* base, int64_t vol_dhw, int D, int H, int W, float px,
                                               float py, float pz, Sample8& v, float& tx, float& ty, float& tz) {
  const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  tx = px - fx;
  ty = py - fy;
  tz = pz - fz;
  // clamp the integer base far outside the volume (all corners then read as 0)
  const float lo = -2.f;
  const int ix = static_cast<int>(fminf(fmaxf(fx, lo), static_cast<float>(W)));
  const int iy = static_cast<int>(fminf(fmaxf(fy, lo), static_cast<float>(H)));
  const int iz = static_cast<int>(fminf(fmaxf(fz, lo), static_cast<float>(D)));
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int z = iz + (c >> 2), y = iy + ((c >> 1) & 1), x = ix + (c & 1);
    v.re[c] = planar_at(base, D, H, W, z, y, x);
    v.im[c] = planar_at(base + vol_dhw, D, H, W, z, y, x);
  }
}

template <typename VT>
__global__ void __launch_bounds__(256) slice3d_fwd_kernel(const VT* __restrict__ vol, int D, int H, int W,
                                                          const float* __restrict__ u, const float* __restrict__ v,
                                                          int N, const float* __restrict__ fx,
                                                          const float* __restrict__ fy, int K, float cx, float cy,
                                                          float cz, VT* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int bn = blockIdx.y;
  if (q >= K) return;
  const int b = bn / N, n = bn - b * N;
  const float a = __ldg(fx + q), bb = __ldg(fy + q);
  const float px = fmaf(bb, __ldg(v + 3 * n + 0), fmaf(a, __ldg(u + 3 * n + 0), cx));
  const float py = fmaf(bb, __ldg(v + 3 * n + 1), fmaf(a, __ldg(u + 3 * n + 1), cy));
  const float pz = fmaf(bb, __ldg(v + 3 * n + 2), fmaf(a, __ldg(u + 3 * n + 2), cz));
  const int64_t dhw = static_cast<int64_t>(D) * H * W;
  Sample8 s;
  float tx, ty, tz;
  planar_corners(vol + static_cast<int64_t>(b) * 2 * dhw, dhw, D, H, W, px, py, pz, s, tx, ty, tz);
  Interp o;
  trilerp<false>(s, tx, ty, tz, o);
  VT* dst = out + static_cast<int64_t>(bn) * 2 * K;
  stf(dst + q, o.sr);
  stf(dst + K + q, o.si);
}

// Per (pose, tile) partial sums of dL/du, dL/dv (6 values) in fp64.
template <typename VT, typename GT>
__global__ void __launch_bounds__(256) slice3d_bwd_kernel(const VT* __restrict__ vol, int B, int D, int H, int W,
                                                          const GT* __restrict__ go, const float* __restrict__ u,
                                                          const float* __restrict__ v, int N,
                                                          const float* __restrict__ fx, const float* __restrict__ fy,
                                                          int K, float cx, float cy, float cz,
                                                          double* __restrict__ partial) {
  __shared__ double red[6 * 8];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y;
  float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (q < K) {
    const float a = __ldg(fx + q), bb = __ldg(fy + q);
    const float px = fmaf(bb, __ldg(v + 3 * n + 0), fmaf(a, __ldg(u + 3 * n + 0), cx));
    const float py = fmaf(bb, __ldg(v + 3 * n + 1), fmaf(a, __ldg(u + 3 * n + 1), cy));
    const float pz = fmaf(bb, __ldg(v + 3 * n + 2), fmaf(a, __ldg(u + 3 * n + 2), cz));
    const int64_t dhw = static_cast<int64_t>(D) * H * W;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    for (int b = 0; b < B; ++b) {
      Sample8 s;
      float tx, ty, tz;
      planar_corners(vol + static_cast<int64_t>(b) * 2 * dhw, dhw, D, H, W, px, py, pz, s, tx, ty, tz);
      Interp o;
      trilerp<true>(s, tx, ty, tz, o);
      const GT* g = go + (static_cast<int64_t>(b) * N + n) * 2 * K;
      const float gr = ldf(g + q), gi = ldf(g + K + q);
      gx = fmaf(gr, o.dxr, fmaf(gi, o.dxi, gx));
      gy = fmaf(gr, o.dyr, fmaf(gi, o.dyi, gy));
      gz = fmaf(gr, o.dzr, fmaf(gi, o.dzi, gz));
    }
    acc[0] = gx * a;
    acc[1] = gy * a;
    acc[2] = gz * a;
    acc[3] = gx * bb;
    acc[4] = gy * bb;
    acc[5] = gz * bb;
  }
  double tot;
  block_reduce_to_f64<6>(acc, red, &tot);
  if (threadIdx.x < 6) partial[(static_cast<int64_t>(n) * gridDim.x + blockIdx.x) * 6 + threadIdx.x] = tot;
}

__global__ void slice3d_bwd_finalize_kernel(const double* __restrict__ partial, int N, int tiles, float* gu,
                                            float* gv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * 6) return;
  const int n = i / 6, m = i - n * 6;
  double s = 0.0;
  for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(n) * tiles + t) * 6 + m];
  if (m < 3)
    gu[n * 3 + m] = static_cast<float>(s);
  else
    gv[n * 3 + m - 3] = static_cast<float>(s);
}

// ----------------------------------------------------------------------------
// FP64 pose maps  (torch_engine.py:139-211)
// ----------------------------------------------------------------------------

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

// Rz(90 deg) exactly as the reference forms it: angle and cos/sin in float32,
// so the off-axis zeros are -4.37e-8 (torch_engine.py:194-198).
__device__ __forceinline__ Mat3 lateral_rot() {
  const float a = __fmul_rn(90.0f, 0.0174532925199432957692f);
  const double c = static_cast<double>(cosf(a)), s = static_cast<double>(sinf(a));
  return rot_z(c, s);
}

struct EulerJac {
  Mat3 R, dz, dy, dx;  // R and dR/d(yaw, pitch, roll) per degree
};

__device__ __forceinline__ EulerJac euler_jac(double yaw, double pitch, double roll) {
  double sz, cz, sy, cy, sx, cx;
  sincos(yaw * kDeg, &sz, &cz);
  sincos(pitch * kDeg, &sy, &cy);
  sincos(roll * kDeg, &sx, &cx);
  const Mat3 Z = rot_z(cz, sz), Y = rot_y(cy, sy), X = rot_x(cx, sx);
  EulerJac j;
  j.R = mat_mul(Z, mat_mul(Y, X));
  j.dz = mat_mul(drot_z(cz, sz), mat_mul(Y, X));
  j.dy = mat_mul(Z, mat_mul(drot_y(cy, sy), X));
  j.dx = mat_mul(Z, mat_mul(Y, drot_x(cx, sx)));
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      j.dz.m[a][b] *= kDeg;
      j.dy.m[a][b] *= kDeg;
      j.dx.m[a][b] *= kDeg;
    }
  return j;
}

// axes[c] = (u_xyz, v_xyz, tx, ty): u = R[0,:]*scale, v = R[1,:]*scale.
__global__ void tc_axes_kernel(const float* __restrict__ poses, int C, int lateral, double sx, double sy, double sz,
                               float* __restrict__ axes) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const float* p = poses + 6 * c;
  EulerJac j = euler_jac(p[0], p[1], p[2]);
  Mat3 R = lateral ? mat_mul(j.R, lateral_rot()) : j.R;
  float* a = axes + 8 * c;
  a[0] = static_cast<float>(R.m[0][0] * sx);
  a[1] = static_cast<float>(R.m[0][1] * sy);
  a[2] = static_cast<float>(R.m[0][2] * sz);
  a[3] = static_cast<float>(R.m[1][0] * sx);
  a[4] = static_cast<float>(R.m[1][1] * sy);
  a[5] = static_cast<float>(R.m[1][2] * sz);
  a[6] = p[3];
  a[7] = p[4];
}

// ----------------------------------------------------------------------------
// fused zero-IFFT spectral NCC  (torch_engine.py:176-234, 269-290)
// ----------------------------------------------------------------------------

enum {
  M_CROSS = 0,
  M_EP,
  M_ET,
  M_PHU,
  M_PHV,
  M_AU,       // 3
  M_AV = 8,   // 3
  M_BU = 11,  // 3
  M_BV = 14,  // 3
  M_NGRAD = 17
};
constexpr int kSnccThreads = 256;
constexpr int kSnccSpt = 4;  // samples per thread per tile
constexpr int kSnccTile = kSnccThreads * kSnccSpt;

struct SnccArgs {
  Stencil st;
  const float* axes;    // [C][8]
  const float2* ftarg;  // [R*R] complex target spectrum (already high-passed)
  const float* hp;      // [R*R] or null
  const float* lin;     // [R] torch.linspace(-1, 1, R)
  int R;
  float kpi;  // kappa / pi, phase/pi = kpi * (ku*tx + kv*ty)
  float cx, cy, cz;
  double* partial;  // [C][tiles][NM]
};

template <int DT, bool GRAD>
__global__ void __launch_bounds__(kSnccThreads) tc_sncc_moments_kernel(SnccArgs a) {
  constexpr int NM = GRAD ? M_NGRAD : 3;
  __shared__ double red[NM * (kSnccThreads / 32)];
  const int c = blockIdx.y;
  const float* ax = a.axes + 8 * c;
  const float ux = __ldg(ax + 0), uy = __ldg(ax + 1), uz = __ldg(ax + 2);
  const float vx = __ldg(ax + 3), vy = __ldg(ax + 4), vz = __ldg(ax + 5);
  const float tx = __ldg(ax + 6), ty = __ldg(ax + 7);
  const int R = a.R;
  const int K = R * R;
  float acc[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m) acc[m] = 0.f;
#pragma unroll
  for (int s = 0; s < kSnccSpt; ++s) {
    const int q = blockIdx.x * kSnccTile + s * kSnccThreads + threadIdx.x;
    if (q >= K) break;
    const int i = q / R, j = q - (q / R) * R;
    const float ku = __ldg(a.lin + i), kv = __ldg(a.lin + j);
    const float px = fmaf(kv, vx, fmaf(ku, ux, a.cx));
    const float py = fmaf(kv, vy, fmaf(ku, uy, a.cy));
    const float pz = fmaf(kv, vz, fmaf(ku, uz, a.cz));
    Interp o;
    stencil_sample<DT, GRAD, false>(a.st, px, py, pz, o);
    float sn, cs;
    sincospif(a.kpi * fmaf(ku, tx, kv * ty), &sn, &cs);
    const float h = a.hp ? __ldg(a.hp + q) : 1.f;
    const float2 T = __ldg(a.ftarg + q);
    const float shr = h * (o.sr * cs - o.si * sn);
    const float shi = h * (o.sr * sn + o.si * cs);
    acc[M_CROSS] = fmaf(shr, T.x, fmaf(shi, T.y, acc[M_CROSS]));
    acc[M_EP] = fmaf(shr, shr, fmaf(shi, shi, acc[M_EP]));
    acc[M_ET] = fmaf(T.x, T.x, fmaf(T.y, T.y, acc[M_ET]));
    if constexpr (GRAD) {
      // dL/dphi direction: Re(conj(T) i S_hat) = T.y*shr - T.x*shi
      const float ph = T.y * shr - T.x * shi;
      acc[M_PHU] = fmaf(ku, ph, acc[M_PHU]);
      acc[M_PHV] = fmaf(kv, ph, acc[M_PHV]);
      // M_T = h e^{-i phi} T ;  A_k = <M_T, dS/dp_k>
      const float mtr = h * (cs * T.x + sn * T.y);
      const float mti = h * (cs * T.y - sn * T.x);
      const float a0 = mtr * o.dxr + mti * o.dxi;
      const float a1 = mtr * o.dyr + mti * o.dyi;
      const float a2 = mtr * o.dzr + mti * o.dzi;
      // B_k = h^2 <S, dS/dp_k>
      const float h2 = h * h;
      const float b0 = h2 * (o.sr * o.dxr + o.si * o.dxi);
      const float b1 = h2 * (o.sr * o.dyr + o.si * o.dyi);
      const float b2 = h2 * (o.sr * o.dzr + o.si * o.dzi);
      acc[M_AU + 0] = fmaf(ku, a0, acc[M_AU + 0]);
      acc[M_AU + 1] = fmaf(ku, a1, acc[M_AU + 1]);
      acc[M_AU + 2] = fmaf(ku, a2, acc[M_AU + 2]);
      acc[M_AV + 0] = fmaf(kv, a0, acc[M_AV + 0]);
      acc[M_AV + 1] = fmaf(kv, a1, acc[M_AV + 1]);
      acc[M_AV + 2] = fmaf(kv, a2, acc[M_AV + 2]);
      acc[M_BU + 0] = fmaf(ku, b0, acc[M_BU + 0]);
      acc[M_BU + 1] = fmaf(ku, b1, acc[M_BU + 1]);
      acc[M_BU + 2] = fmaf(ku, b2, acc[M_BU + 2]);
      acc[M_BV + 0] = fmaf(kv, b0, acc[M_BV + 0]);
      acc[M_BV + 1] = fmaf(kv, b1, acc[M_BV + 1]);
      acc[M_BV + 2] = fmaf(kv, b2, acc[M_BV + 2]);
    }
  }
  double tot;
  block_reduce_to_f64<NM>(acc, red, &tot);
  if (threadIdx.x < NM) a.partial[(static_cast<int64_t>(c) * gridDim.x + blockIdx.x) * NM + threadIdx.x] = tot;
}

// Sum tiles (fp64, fixed order) -> mom[c][NM]; loss = 1 - mean_c ncc_c.
__global__ void __launch_bounds__(256) tc_sncc_finalize_kernel(const double* __restrict__ partial, int C, int tiles,
                                                               int NM, double* __restrict__ mom,
                                                               float* __restrict__ loss, float* __restrict__ ncc_out) {
  __shared__ double red[8];
  double nsum = 0.0;
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    double v[M_NGRAD];
    for (int m = 0; m < NM; ++m) {
      double s = 0.0;
      for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(c) * tiles + t) * NM + m];
      v[m] = s;
      mom[static_cast<int64_t>(c) * NM + m] = s;
    }
    const double ncc = v[M_CROSS] / (sqrt(v[M_EP] * v[M_ET]) + 1e-8);
    if (ncc_out) ncc_out[c] = static_cast<float>(ncc);
    nsum += ncc;
  }
  nsum = warp_sum(nsum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) s += red[w];
    *loss = static_cast<float>(1.0 - s / static_cast<double>(C));
  }
}

// Pose gradient from per-candidate slice-axis gradients.
//  mode 0: spectral NCC moments mom[c][17] and upstream dL/dloss (*g)
//  mode 1: adjoint partials part[c][tiles][8] = (dU[3], dV[3], PHU, PHV)
__global__ void tc_pose_grad_kernel(int mode, const double* __restrict__ src, int tiles, const float* __restrict__ g,
                                    const float* __restrict__ poses, int C, int lateral, double sx, double sy,
                                    double sz, double kappa, float* __restrict__ grad, int accumulate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double du[3], dv[3], dtx, dty;
  if (mode == 0) {
    const double* v = src + static_cast<int64_t>(c) * M_NGRAD;
    const double gl = static_cast<double>(*g);
    const double s = sqrt(v[M_EP] * v[M_ET]);
    const double aa = 1.0 / (s + 1e-8);
    const double bb = s > 0.0 ? -v[M_CROSS] * v[M_ET] / (2.0 * s * (s + 1e-8) * (s + 1e-8)) : 0.0;
    const double gc = -gl / static_cast<double>(C);
    for (int k = 0; k < 3; ++k) {
      du[k] = gc * (aa * v[M_AU + k] + 2.0 * bb * v[M_BU + k]);
      dv[k] = gc * (aa * v[M_AV + k] + 2.0 * bb * v[M_BV + k]);
    }
    dtx = gc * aa * kappa * v[M_PHU];
    dty = gc * aa * kappa * v[M_PHV];
  } else {
    double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < tiles; ++i)
      for (int m = 0; m < 8; ++m) t[m] += src[(static_cast<int64_t>(c) * tiles + i) * 8 + m];
    for (int k = 0; k < 3; ++k) {
      du[k] = t[k];
      dv[k] = t[3 + k];
    }
    dtx = kappa * t[6];
    dty = kappa * t[7];
  }
  const float* p = poses + 6 * c;
  EulerJac j = euler_jac(p[0], p[1], p[2]);
  Mat3 gR{{{du[0] * sx, du[1] * sy, du[2] * sz}, {dv[0] * sx, dv[1] * sy, dv[2] * sz}, {0.0, 0.0, 0.0}}};
  if (lateral) {  // R_total = R_pose . R_lat  ->  dL/dR_pose = dL/dR_total . R_lat^T
    const Mat3 L = lateral_rot();
    Mat3 t;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) t.m[a][b] = gR.m[a][0] * L.m[b][0] + gR.m[a][1] * L.m[b][1] + gR.m[a][2] * L.m[b][2];
    gR = t;
  }
  double gyaw = 0.0, gpitch = 0.0, groll = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      gyaw += gR.m[a][b] * j.dz.m[a][b];
      gpitch += gR.m[a][b] * j.dy.m[a][b];
      groll += gR.m[a][b] * j.dx.m[a][b];
    }
  float* o = grad + 6 * c;
  const float r[6] = {static_cast<float>(gyaw), static_cast<float>(gpitch), static_cast<float>(groll),
                      static_cast<float>(dtx), static_cast<float>(dty), 0.f};
  for (int k = 0; k < 6; ++k) o[k] = accumulate ? o[k] + r[k] : r[k];
}

// ----------------------------------------------------------------------------
// image path: modulated slice and its adjoint  (torch_engine.py:176-241)
// ----------------------------------------------------------------------------

struct SliceArgs {
  Stencil st;
  const float* axes;
  const float* lin;
  int R;
  float kpi;
  float cx, cy, cz;
  int shift;  // 1: write/read position ifftshift(q) (image path), 0: natural order
};

__device__ __forceinline__ int shifted_pos(int i, int j, int R, int shift) {
  if (shift) {
    // ifftshift: element (i, j) lands at ((i - R/2) mod R, (j - R/2) mod R)
    const int h = R / 2;
    i = i - h;
    if (i < 0) i += R;
    j = j - h;
    if (j < 0) j += R;
  }
  return i * R + j;
}

template <int DT>
__global__ void __launch_bounds__(256) tc_slice_kernel(SliceArgs a, float2* __restrict__ out) {
  const int c = blockIdx.y;
  const int R = a.R;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= R * R) return;
  const float* ax = a.axes + 8 * c;
  const int i = q / R, j = q - (q / R) * R;
  const float ku = __ldg(a.lin + i), kv = __ldg(a.lin + j);
  const float px = fmaf(kv, __ldg(ax + 3), fmaf(ku, __ldg(ax + 0), a.cx));
  const float py = fmaf(kv, __ldg(ax + 4), fmaf(ku, __ldg(ax + 1), a.cy));
  const float pz = fmaf(kv, __ldg(ax + 5), fmaf(ku, __ldg(ax + 2), a.cz));
  Interp o;
  stencil_sample<DT, false, false>(a.st, px, py, pz, o);
  float sn, cs;
  sincospif(a.kpi * fmaf(ku, __ldg(ax + 6), kv * __ldg(ax + 7)), &sn, &cs);
  out[static_cast<int64_t>(c) * R * R + shifted_pos(i, j, R, a.shift)] =
      make_float2(o.sr * cs - o.si * sn, o.sr * sn + o.si * cs);
}

// Given G = dL/dS_hat per sample, per-candidate partials
// (dU[3], dV[3], PHU, PHV) with dL/dS = e^{-i phi} G and
// dL/dphi = Re(conj(G) i S_hat).
template <int DT>
__global__ void __launch_bounds__(256) tc_slice_adjoint_kernel(SliceArgs a, const float2* __restrict__ G,
                                                               double* __restrict__ partial) {
  __shared__ double red[8 * 8];
  const int c = blockIdx.y;
  const int R = a.R;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (q < R * R) {
    const float* ax = a.axes + 8 * c;
    const int i = q / R, j = q - (q / R) * R;
    const float ku = __ldg(a.lin + i), kv = __ldg(a.lin + j);
    const float px = fmaf(kv, __ldg(ax + 3), fmaf(ku, __ldg(ax + 0), a.cx));
    const float py = fmaf(kv, __ldg(ax + 4), fmaf(ku, __ldg(ax + 1), a.cy));
    const float pz = fmaf(kv, __ldg(ax + 5), fmaf(ku, __ldg(ax + 2), a.cz));
    Interp o;
    stencil_sample<DT, true, false>(a.st, px, py, pz, o);
    float sn, cs;
    sincospif(a.kpi * fmaf(ku, __ldg(ax + 6), kv * __ldg(ax + 7)), &sn, &cs);
    const float2 g = __ldg(G + static_cast<int64_t>(c) * R * R + shifted_pos(i, j, R, a.shift));
    const float shr = o.sr * cs - o.si * sn, shi = o.sr * sn + o.si * cs;
    const float ph = g.y * shr - g.x * shi;
    const float dr = cs * g.x + sn * g.y, di = cs * g.y - sn * g.x;  // e^{-i phi} G
    const float e0 = dr * o.dxr + di * o.dxi;
    const float e1 = dr * o.dyr + di * o.dyi;
    const float e2 = dr * o.dzr + di * o.dzi;
    acc[0] = ku * e0;
    acc[1] = ku * e1;
    acc[2] = ku * e2;
    acc[3] = kv * e0;
    acc[4] = kv * e1;
    acc[5] = kv * e2;
    acc[6] = ku * ph;
    acc[7] = kv * ph;
  }
  double tot;
  block_reduce_to_f64<8>(acc, red, &tot);
  if (threadIdx.x < 8) partial[(static_cast<int64_t>(c) * gridDim.x + blockIdx.x) * 8 + threadIdx.x] = tot;
}

// relu mask of the saved image, as complex: G = (img > 0) * g
__global__ void relu_mask_kernel(const float* __restrict__ img, const float* __restrict__ g, float* __restrict__ out,
                                 int64_t n) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  out[i] = img[i] > 0.f ? g[i] : 0.f;
}

// complex * real table (per image), e.g. the high-pass filter of a target spectrum
__global__ void cmul_table_kernel(float2* __restrict__ x, const float* __restrict__ t, int64_t per, int64_t n) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float w = t[i % per];
  x[i] = make_float2(x[i].x * w, x[i].y * w);
}

// HP = 1 - exp(-r^2 / (2 sigma^2)) on linspace(-H/2, H/2, H) x linspace(-W/2, W/2, W)
// (torch_engine.py:123-136), evaluated in fp64.
__global__ void hp_filter_kernel(float* __restrict__ out, int H, int W, double sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= H * W) return;
  const int r = i / W, c = i - r * W;
  const double y = H > 1 ? -0.5 * H + r * (static_cast<double>(H) / (H - 1)) : -0.5 * H;
  const double x = W > 1 ? -0.5 * W + c * (static_cast<double>(W) / (W - 1)) : -0.5 * W;
  out[i] = static_cast<float>(1.0 - exp(-(x * x + y * y) / (2.0 * sigma * sigma)));
}

__global__ void linspace_kernel(float* out, float start, float end, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = linspace_f32(start, end, n, i);
}

static int stencil_from(int dtype, const void* data, const float* scales, int64_t D, int64_t H, int64_t W,
                        Stencil* s) {
  if (!data || D < 1 || H < 1 || W < 1 || D > 8192 || H > 8192 || W > 8192) return FVR_ERR_ARG;
  if (dtype != FVR_F32 && dtype != FVR_BF16 && dtype != FVR_F16) return FVR_ERR_DTYPE;
  if (dtype == FVR_F16 && !scales) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(data) & 15) != 0) return FVR_ERR_ARG;
  *s = Stencil{data, scales, static_cast<int>(D), static_cast<int>(H), static_cast<int>(W), dtype};
  return FVR_OK;
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int64_t fvr_stencil_bytes(int64_t D, int64_t H, int64_t W, int dtype) {
  const int64_t n = (D + 1) * (H + 1) * (W + 1);
  if (dtype == FVR_F32) return n * 64;
  if (dtype == FVR_BF16 || dtype == FVR_F16) return n * 32;
  return -1;
}

int64_t fvr_stencil_scale_count(int64_t D, int64_t H, int64_t W) {
  return fvr::cdiv64(D + 1, kBrick) * fvr::cdiv64(H + 1, kBrick) * fvr::cdiv64(W + 1, kBrick);
}

int fvr_stencil_build(const void* master, int master_dtype, int master_planar, int64_t D, int64_t H, int64_t W,
                      int out_dtype, void* out, float* scales, unsigned int* scratch_max, void* stream) {
  if (!master || !out || D < 1 || H < 1 || W < 1 || D > 8192 || H > 8192 || W > 8192) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(out) & 15) != 0) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n = (D + 1) * (H + 1) * (W + 1);
  const int64_t nblk = cdiv64(n, 256);
  const unsigned grid = static_cast<unsigned>(nblk < 148 * 64 ? nblk : 148 * 64);
  const int d = (int)D, h = (int)H, w = (int)W;
  const int64_t plane = master_planar ? D * H * W : 0;
  if (out_dtype == FVR_F16) {
    if (!scales || !scratch_max) return FVR_ERR_ARG;
    const int64_t nb = fvr_stencil_scale_count(D, H, W);
    if (cudaMemsetAsync(scratch_max, 0, nb * sizeof(unsigned int), s) != cudaSuccess) return FVR_ERR_CUDA;
    if (master_dtype == FVR_F32)
      stencil_brick_max_kernel<float>
          <<<grid, 256, 0, s>>>(static_cast<const float*>(master), plane, d, h, w, scratch_max);
    else if (master_dtype == FVR_BF16)
      stencil_brick_max_kernel<__nv_bfloat16>
          <<<grid, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(master), plane, d, h, w, scratch_max);
    else
      return FVR_ERR_DTYPE;
    stencil_scale_kernel<<<static_cast<unsigned>(cdiv64(nb, 256)), 256, 0, s>>>(scratch_max, scales, nb);
  }
#define FVR_BUILD(MT, DT)                                                                                  \
  stencil_build_kernel<MT, DT><<<grid, 256, 0, s>>>(static_cast<const MT*>(master), plane, d, h, w, out, scales); \
  break;
  if (master_dtype == FVR_F32) {
    switch (out_dtype) {
      case FVR_F32: FVR_BUILD(float, FVR_F32)
      case FVR_BF16: FVR_BUILD(float, FVR_BF16)
      case FVR_F16: FVR_BUILD(float, FVR_F16)
      default: return FVR_ERR_DTYPE;
    }
  } else if (master_dtype == FVR_BF16) {
    switch (out_dtype) {
      case FVR_F32: FVR_BUILD(__nv_bfloat16, FVR_F32)
      case FVR_BF16: FVR_BUILD(__nv_bfloat16, FVR_BF16)
      case FVR_F16: FVR_BUILD(__nv_bfloat16, FVR_F16)
      default: return FVR_ERR_DTYPE;
    }
  } else {
    return FVR_ERR_DTYPE;
  }
#undef FVR_BUILD
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_slice3d_fwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const float* u,
                    const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx, float cy,
                    float cz, void* out, void* stream) {
  if (!vol || !u || !v || !fx || !fy || !out) return FVR_ERR_ARG;
  if (B < 1 || N < 1 || K < 1 || D < 1 || H < 1 || W < 1) return FVR_ERR_ARG;
  if (B * N > 65535 || K > (int64_t)1 << 30) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dim3 grid(static_cast<unsigned>(cdiv64(K, 256)), static_cast<unsigned>(B * N));
  switch (dtype) {
    case FVR_F32:
      slice3d_fwd_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float*>(vol), (int)D, (int)H, (int)W, u, v,
                                                     (int)N, fx, fy, (int)K, cx, cy, cz, static_cast<float*>(out));
      break;
    case FVR_BF16:
      slice3d_fwd_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(vol), (int)D, (int)H,
                                                             (int)W, u, v, (int)N, fx, fy, (int)K, cx, cy, cz,
                                                             static_cast<__nv_bfloat16*>(out));
      break;
    case FVR_F16:
      slice3d_fwd_kernel<__half><<<grid, 256, 0, s>>>(static_cast<const __half*>(vol), (int)D, (int)H, (int)W, u, v,
                                                      (int)N, fx, fy, (int)K, cx, cy, cz, static_cast<__half*>(out));
      break;
    default:
      return FVR_ERR_DTYPE;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_slice3d_bwd_workspace(int64_t N, int64_t K) { return N * cdiv64(K, 256) * 6 * (int64_t)sizeof(double); }

int fvr_slice3d_bwd(const void* vol, int dtype, int64_t B, int64_t D, int64_t H, int64_t W, const void* grad_out,
                    const float* u, const float* v, int64_t N, const float* fx, const float* fy, int64_t K, float cx,
                    float cy, float cz, float* gu, float* gv, void* workspace, int64_t ws_bytes, void* stream) {
  if (!vol || !grad_out || !u || !v || !fx || !fy || !gu || !gv || !workspace) return FVR_ERR_ARG;
  if (B < 1 || N < 1 || K < 1 || D < 1 || H < 1 || W < 1 || N > 65535) return FVR_ERR_ARG;
  if (ws_bytes < fvr_slice3d_bwd_workspace(N, K)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tiles = static_cast<int>(cdiv64(K, 256));
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(N));
  double* part = static_cast<double*>(workspace);
  switch (dtype) {
    case FVR_F32:
      slice3d_bwd_kernel<float, float><<<grid, 256, 0, s>>>(static_cast<const float*>(vol), (int)B, (int)D, (int)H,
                                                            (int)W, static_cast<const float*>(grad_out), u, v, (int)N,
                                                            fx, fy, (int)K, cx, cy, cz, part);
      break;
    case FVR_BF16:
      slice3d_bwd_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, 256, 0, s>>>(
          static_cast<const __nv_bfloat16*>(vol), (int)B, (int)D, (int)H, (int)W,
          static_cast<const __nv_bfloat16*>(grad_out), u, v, (int)N, fx, fy, (int)K, cx, cy, cz, part);
      break;
    case FVR_F16:
      slice3d_bwd_kernel<__half, __half><<<grid, 256, 0, s>>>(static_cast<const __half*>(vol), (int)B, (int)D,
                                                              (int)H, (int)W, static_cast<const __half*>(grad_out), u,
                                                              v, (int)N, fx, fy, (int)K, cx, cy, cz, part);
      break;
    default:
      return FVR_ERR_DTYPE;
  }
  FVR_LAUNCH_CHECK();
  slice3d_bwd_finalize_kernel<<<static_cast<unsigned>(cdiv64(N * 6, 256)), 256, 0, s>>>(part, (int)N, tiles, gu, gv);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_axes(const float* poses, int64_t C, int view, int64_t D, int64_t H, int64_t W, float* axes,
                void* stream) {
  if (!poses || !axes || C < 1 || (view != 0 && view != 1)) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double sx = 0.5 * static_cast<double>(W > 1 ? W - 1 : 1);
  const double sy = 0.5 * static_cast<double>(H > 1 ? H - 1 : 1);
  const double sz = 0.5 * static_cast<double>(D > 1 ? D - 1 : 1);
  tc_axes_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, s>>>(poses, (int)C, view, sx, sy, sz, axes);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_tc_sncc_workspace(int64_t C, int64_t R) {
  return C * cdiv64(R * R, kSnccTile) * M_NGRAD * (int64_t)sizeof(double);
}

int fvr_tc_sncc_moments(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                        const float* axes, int64_t C, const void* ftarg, const float* hp, const float* lin,
                        int64_t R, double kappa, int with_grad, void* workspace, int64_t ws_bytes, void* stream) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!axes || !ftarg || !lin || !workspace || C < 1 || R < 1 || C > 65535) return FVR_ERR_ARG;
  if (R * R > (int64_t)1 << 30) return FVR_ERR_ARG;
  if (ws_bytes < fvr_tc_sncc_workspace(C, R)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tiles = static_cast<int>(cdiv64(R * R, kSnccTile));
  SnccArgs a{st,
             axes,
             static_cast<const float2*>(ftarg),
             hp,
             lin,
             (int)R,
             static_cast<float>(kappa / 3.14159265358979323846),
             static_cast<float>(0.5 * (W > 1 ? W - 1 : 1)),
             static_cast<float>(0.5 * (H > 1 ? H - 1 : 1)),
             static_cast<float>(0.5 * (D > 1 ? D - 1 : 1)),
             static_cast<double*>(workspace)};
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(C));
#define FVR_SNCC(DT)                                                    \
  if (with_grad)                                                        \
    tc_sncc_moments_kernel<DT, true><<<grid, kSnccThreads, 0, s>>>(a);  \
  else                                                                  \
    tc_sncc_moments_kernel<DT, false><<<grid, kSnccThreads, 0, s>>>(a); \
  break;
  switch (dtype) {
    case FVR_F32: FVR_SNCC(FVR_F32)
    case FVR_BF16: FVR_SNCC(FVR_BF16)
    case FVR_F16: FVR_SNCC(FVR_F16)
  }
#undef FVR_SNCC
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_finalize(const void* workspace, int64_t C, int64_t R, int with_grad, double* mom, float* loss,
                         float* ncc_out, void* stream) {
  if (!workspace || !mom || !loss || C < 1 || R < 1) return FVR_ERR_ARG;
  const int tiles = static_cast<int>(cdiv64(R * R, kSnccTile));
  tc_sncc_finalize_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const double*>(workspace), (int)C, tiles, with_grad ? M_NGRAD : 3, mom, loss, ncc_out);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_backward(const double* mom, const float* g, const float* poses, int64_t C, int view, int64_t D,
                         int64_t H, int64_t W, double kappa, float* grad_poses, int accumulate, void* stream) {
  if (!mom || !g || !poses || !grad_poses || C < 1 || (view != 0 && view != 1)) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  tc_pose_grad_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, s>>>(
      0, mom, 1, g, poses, (int)C, view, 0.5 * (W > 1 ? W - 1 : 1), 0.5 * (H > 1 ? H - 1 : 1),
      0.5 * (D > 1 ? D - 1 : 1), kappa, grad_poses, accumulate);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_slice(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                 const float* axes, int64_t C, const float* lin, int64_t R, double kappa, int shift, void* out,
                 void* stream) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!axes || !lin || !out || C < 1 || R < 1 || C > 65535 || R * R > (int64_t)1 << 30) return FVR_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SliceArgs a{st,
              axes,
              lin,
              (int)R,
              static_cast<float>(kappa / 3.14159265358979323846),
              static_cast<float>(0.5 * (W > 1 ? W - 1 : 1)),
              static_cast<float>(0.5 * (H > 1 ? H - 1 : 1)),
              static_cast<float>(0.5 * (D > 1 ? D - 1 : 1)),
              shift ? 1 : 0};
  dim3 grid(static_cast<unsigned>(cdiv64(R * R, 256)), static_cast<unsigned>(C));
  float2* o = static_cast<float2*>(out);
  switch (dtype) {
    case FVR_F32: tc_slice_kernel<FVR_F32><<<grid, 256, 0, s>>>(a, o); break;
    case FVR_BF16: tc_slice_kernel<FVR_BF16><<<grid, 256, 0, s>>>(a, o); break;
    case FVR_F16: tc_slice_kernel<FVR_F16><<<grid, 256, 0, s>>>(a, o); break;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_tc_slice_adjoint_workspace(int64_t C, int64_t R) {
  return C * cdiv64(R * R, 256) * 8 * (int64_t)sizeof(double);
}

int fvr_tc_slice_adjoint(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                         const float* axes, const float* poses, int64_t C, int view, const float* lin, int64_t R,
                         double kappa, int shift, const void* G, void* workspace, int64_t ws_bytes,
                         float* grad_poses, int accumulate, void* stream) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!axes || !poses || !lin || !G || !workspace || !grad_poses || C < 1 || R < 1 || C > 65535) return FVR_ERR_ARG;
  if (view != 0 && view != 1) return FVR_ERR_ARG;
  if (ws_bytes < fvr_tc_slice_adjoint_workspace(C, R)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SliceArgs a{st,
              axes,
              lin,
              (int)R,
              static_cast<float>(kappa / 3.14159265358979323846),
              static_cast<float>(0.5 * (W > 1 ? W - 1 : 1)),
              static_cast<float>(0.5 * (H > 1 ? H - 1 : 1)),
              static_cast<float>(0.5 * (D > 1 ? D - 1 : 1)),
              shift ? 1 : 0};
  const int tiles = static_cast<int>(cdiv64(R * R, 256));
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(C));
  double* part = static_cast<double*>(workspace);
  const float2* g = static_cast<const float2*>(G);
  switch (dtype) {
    case FVR_F32: tc_slice_adjoint_kernel<FVR_F32><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_BF16: tc_slice_adjoint_kernel<FVR_BF16><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_F16: tc_slice_adjoint_kernel<FVR_F16><<<grid, 256, 0, s>>>(a, g, part); break;
  }
  FVR_LAUNCH_CHECK();
  tc_pose_grad_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, s>>>(
      1, part, tiles, nullptr, poses, (int)C, view, 0.5 * (W > 1 ? W - 1 : 1), 0.5 * (H > 1 ? H - 1 : 1),
      0.5 * (D > 1 ? D - 1 : 1), kappa, grad_poses, accumulate);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_relu_mask(const float* img, const float* g, float* out, int64_t n, void* stream) {
  if (!img || !g || !out || n < 1) return FVR_ERR_ARG;
  relu_mask_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(img, g,
                                                                                                          out, n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_cmul_table(void* x, const float* table, int64_t per, int64_t n, void* stream) {
  if (!x || !table || per < 1 || n < 1) return FVR_ERR_ARG;
  cmul_table_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<float2*>(x), table, per, n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_hp_filter(float* out, int64_t H, int64_t W, double sigma, void* stream) {
  if (!out || H < 1 || W < 1 || H * W > (int64_t)1 << 30) return FVR_ERR_ARG;
  hp_filter_kernel<<<static_cast<unsigned>(cdiv64(H * W, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      out, (int)H, (int)W, sigma);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_linspace(float* out, float start, float end, int64_t n, void* stream) {
  if (!out || n < 1 || n > (int64_t)1 << 30) return FVR_ERR_ARG;
  linspace_kernel<<<static_cast<unsigned>(cdiv64(n, 256)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      out, start, end, (int)n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
