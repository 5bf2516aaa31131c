// Parallel-beam (torch-engine convention) kernels, sm_100a.
//
//  * fused zero-IFFT spectral NCC (src/fvr/torch_engine.py:176-234, 269-307):
//    one pass per (candidate, view) that forms the slice axes from the pose in
//    FP64, gathers the slice from the stencil spectrum at positions built
//    from FP64 per-row / per-column tables, applies the phase ramp (table
//    factors) and the high-pass filter, and reduces the NCC
//    moments together with the 14 moments the pose gradient needs, so the
//    adjoint is a per-candidate FP64 epilogue (no slice is stored and none is
//    recomputed).  Several views share one launch.
//  * image path (torch_engine.py:236-241): modulated slice written in
//    ifftshift order for the 2D IFFT, and the per-sample slice adjoint.
//  * FP64 pose maps: Euler (yaw Z, pitch Y, roll X) -> slice axes and the
//    Euler vector-Jacobian product (torch_engine.py:139-211).
#include <mutex>

#include "fvr_pose.cuh"
#include "fvr_stencil.cuh"

namespace fvr {

// ----------------------------------------------------------------------------
// slice axes
// ----------------------------------------------------------------------------

// u = R[0,:] * scale, v = R[1,:] * scale with R the (lateral-composed) rotation.
__device__ __forceinline__ void slice_axes(const float* p, int lateral, double sx, double sy, double sz,
                                           double* ax) {
  Mat3 R = euler_R(p[0], p[1], p[2]);
  if (lateral) R = mat_mul(R, lateral_rot());
  ax[0] = R.m[0][0] * sx;
  ax[1] = R.m[0][1] * sy;
  ax[2] = R.m[0][2] * sz;
  ax[3] = R.m[1][0] * sx;
  ax[4] = R.m[1][1] * sy;
  ax[5] = R.m[1][2] * sz;
  ax[6] = p[3];
  ax[7] = p[4];
}

// Slice axes (as slice_axes) and their Jacobian with respect to the pose
// angles: jac[k][r][i] = d(R_total[r][i]) / d(angle k) per degree, k = yaw,
// pitch, roll, rows r = 0 (u) and 1 (v), R_total = R (. Rz(90) for lateral).
__device__ __forceinline__ void slice_axes_jac(const float* p, int lateral, double sx, double sy, double sz,
                                               double* ax, double* jac) {
  Mat3 R, dR[3];
  euler_R_jac(p[0], p[1], p[2], &R, dR);
  if (lateral) {
    R = mat_mul(R, lateral_rot());
#pragma unroll
    for (int k = 0; k < 3; ++k) dR[k] = mat_mul(dR[k], lateral_rot());
  }
  ax[0] = R.m[0][0] * sx;
  ax[1] = R.m[0][1] * sy;
  ax[2] = R.m[0][2] * sz;
  ax[3] = R.m[1][0] * sx;
  ax[4] = R.m[1][1] * sy;
  ax[5] = R.m[1][2] * sz;
  ax[6] = p[3];
  ax[7] = p[4];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int i = 0; i < 3; ++i) jac[(k * 2 + r) * 3 + i] = dR[k].m[r][i] * kDeg;
}

__global__ void tc_axes_kernel(const float* __restrict__ poses, int C, int lateral, double sx, double sy, double sz,
                               double* __restrict__ axes) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  slice_axes(poses + 6 * c, lateral, sx, sy, sz, axes + 8 * c);
}

// dL/d(yaw, pitch, roll) from dL/du, dL/dv (slice axes) for one view.
__device__ __forceinline__ void axes_vjp(const float* p, int lateral, double sx, double sy, double sz,
                                         const double du[3], const double dv[3], double out[3]) {
  Mat3 G{{{du[0] * sx, du[1] * sy, du[2] * sz}, {dv[0] * sx, dv[1] * sy, dv[2] * sz}, {0.0, 0.0, 0.0}}};
  if (lateral) G = mat_mul_bt(G, lateral_rot());  // R_total = R_pose . L -> dR_pose = dR_total . L^T
  euler_vjp(p[0], p[1], p[2], G, out);
}

// Compensated phase / pi: the products of the float32 grid values and
// translations are exact in FP64; one rounding to float before sincospif.
__device__ __forceinline__ void phase_sincos(double kpi, float ku, float kv, float tx, float ty, float* sn,
                                             float* cs) {
  const double arg =
      kpi * fma(static_cast<double>(ku), static_cast<double>(tx), static_cast<double>(kv) * static_cast<double>(ty));
  sincospif(static_cast<float>(arg), sn, cs);
}

// ----------------------------------------------------------------------------
// fused zero-IFFT spectral NCC
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
constexpr int kMomStride = 18;  // mom[v][c][18]: 17 moments + ncc
constexpr int kMaxViews = 4;
constexpr int kSnccThreads = 256;

// Launch variants of the moments kernel (chosen per shape by the caller's
// autotuner): samples whose loads are in flight per thread, and the resident
// CTAs per SM the register budget is sized for.
struct SnccVariant {
  int group, min_blocks;
};
constexpr int kSnccVariants = 6;
__host__ __device__ constexpr SnccVariant sncc_variant(int v) {
  return v == 1 ? SnccVariant{2, 4} : v == 2 ? SnccVariant{4, 3} : v == 3 ? SnccVariant{8, 1}
                : v == 4 ? SnccVariant{2, 3} : v == 5 ? SnccVariant{3, 3} : SnccVariant{4, 2};
}

struct SnccArgs {
  Stencil st;
  const float* poses;  // [C][6]
  const float2* ftarg[kMaxViews];
  int lateral[kMaxViews];
  const float* hp;   // [R*R] or null
  const float* lin;  // [R]
  int R, C, tile;    // tile = samples per CTA
  int tab_rows;      // row-table entries per CTA (>= rows a tile touches)
  double kpi;        // kappa / pi
  double sx, sy, sz;
  double* partial;  // [nv][C][tiles][NM]
  // fused epilogue (value_and_grad launch) only
  unsigned* counters;  // [C + 1], zero on entry, left zero on exit
  double* mom;         // [nv][C][kMomStride]
  double* jac;         // [nv][C][18]: slice-axes Jacobian per (view, candidate)
  float* loss;         // [nv + 1]
  float* ncc_out;      // [nv][C] or null
  float* grad;         // [C][6]
  const float* g;      // dL/dloss_v at g[v * g_stride]; null = all ones
  int g_stride, accumulate;
  double kappa;
};

// dL/dpose of one candidate from its per-view moment records (record of view v
// at mom + v * view_stride): per axis dL/dp = gc (a A + 2 b B) with
// a = 1/(s + eps), b = -cross Et / (2 s (s + eps)^2), s = sqrt(Ep Et),
// gc = -g_v / C; rotations through the Euler vector-Jacobian product, the
// in-plane translations from the phase moments.
__device__ __forceinline__ void sncc_pose_grad(const double* mom, int64_t view_stride, const float* p, int nv,
                                               int lat_bits, const float* g, int g_stride, int C, double sx,
                                               double sy, double sz, double kappa, float r[6]) {
  double gang[3] = {0.0, 0.0, 0.0}, gtx = 0.0, gty = 0.0;
  for (int v = 0; v < nv; ++v) {
    const double* m = mom + v * view_stride;
    const double s = sqrt(m[M_EP] * m[M_ET]);
    const double aa = 1.0 / (s + 1e-8);
    const double bb = s > 0.0 ? -m[M_CROSS] * m[M_ET] / (2.0 * s * (s + 1e-8) * (s + 1e-8)) : 0.0;
    const double gc = -(g ? static_cast<double>(g[v * g_stride]) : 1.0) / C;
    double du[3], dv[3], ga[3];
    for (int k = 0; k < 3; ++k) {
      du[k] = gc * (aa * m[M_AU + k] + 2.0 * bb * m[M_BU + k]);
      dv[k] = gc * (aa * m[M_AV + k] + 2.0 * bb * m[M_BV + k]);
    }
    axes_vjp(p, (lat_bits >> v) & 1, sx, sy, sz, du, dv, ga);
    for (int k = 0; k < 3; ++k) gang[k] += ga[k];
    gtx += gc * aa * kappa * m[M_PHU];
    gty += gc * aa * kappa * m[M_PHV];
  }
  r[0] = static_cast<float>(gang[0]);
  r[1] = static_cast<float>(gang[1]);
  r[2] = static_cast<float>(gang[2]);
  r[3] = static_cast<float>(gtx);
  r[4] = static_cast<float>(gty);
  r[5] = 0.f;
}

// bit v = lateral flag of view v (constant indices only: no dynamic indexing
// of the kernel parameter space)
__device__ __forceinline__ int lateral_bits(const int (&lat)[kMaxViews]) {
  return (lat[0] & 1) | ((lat[1] & 1) << 1) | ((lat[2] & 1) << 2) | ((lat[3] & 1) << 3);
}

__device__ __forceinline__ double sncc_ncc(const double* m) {
  return m[M_CROSS] / (sqrt(m[M_EP] * m[M_ET]) + 1e-8);
}

// CTA sum of per-thread partials; cross-lane in T, cross-warp in fp64 (the
// pose-gradient moments are small residuals of large cancelling sums: each
// lane holds a short run of samples, the long sums are fp64).
template <int NV, typename T>
__device__ __forceinline__ void block_reduce_d(T (&acc)[NV], double* red, double* out_m) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    T t = acc[m];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[m * nw + wid] = static_cast<double>(t);
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    *out_m = s;
  }
}

__device__ __forceinline__ void build_axis_tables(const AxisTables& t, int R, int row0, int n_row,
                                                  const float* __restrict__ lin, const double* ax, double sx,
                                                  double sy, double sz, double kpi) {
  for (int n = threadIdx.x; n < R + n_row; n += blockDim.x) {
    const bool col = n < R;
    const float kf = __ldg(lin + (col ? n : row0 + n - R));
    const double k = kf;
    const double px = col ? k * ax[3] : fma(k, ax[0], sx);
    const double py = col ? k * ax[4] : fma(k, ax[1], sy);
    const double pz = col ? k * ax[5] : fma(k, ax[2], sz);
    const double fx = floor(px), fy = floor(py), fz = floor(pz);
    t.idx[n] = make_int4(static_cast<int>(fx), static_cast<int>(fy), static_cast<int>(fz), 0);
    t.frac[n] = make_float4(static_cast<float>(px - fx), static_cast<float>(py - fy), static_cast<float>(pz - fz), kf);
    double sn, cs;
    sincospi(kpi * k * (col ? ax[7] : ax[6]), &sn, &cs);
    t.ph[n] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
  }
}


// Ticket protocol (as a grid barrier does it): the CTA barrier orders every
// thread's stores before thread 0, whose fence publishes them at device scope
// before it takes a ticket; the thread that takes a last ticket fences again
// before its CTA reads the other CTAs' records (through L2).  The candidate
// epilogue needs one round of loads (tile sums and the stored axes
// Jacobians) and fp64 arithmetic in one thread; the losses one more round.
__device__ __forceinline__ void sncc_fused_epilogue(const SnccArgs& a, int c) {
  __shared__ int s_last;
  __shared__ double s_mom[kMaxViews][kMomStride];
  __shared__ double s_jac[kMaxViews][18];
  const int tiles = gridDim.x, nv = gridDim.z, C = a.C;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const bool last = atomicAdd(a.counters + c, 1u) == static_cast<unsigned>(tiles * nv - 1);
    if (last) __threadfence();
    s_last = last;
  }
  __syncthreads();
  if (!s_last) return;
  // candidate c is complete: tile sums (fixed order) and Jacobians in one round
  for (int t = threadIdx.x; t < nv * (M_NGRAD + 18); t += blockDim.x) {
    if (t < nv * M_NGRAD) {
      const int v = t / M_NGRAD, m = t - v * M_NGRAD;
      const double* src = a.partial + (static_cast<int64_t>(v) * C + c) * tiles * M_NGRAD + m;
      double sum = 0.0;
      for (int k0 = 0; k0 < tiles; k0 += 4) {  // four independent loads in flight
        double x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = k0 + u < tiles ? __ldcg(src + (k0 + u) * M_NGRAD) : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) sum += x[u];
      }
      s_mom[v][m] = sum;
    } else {
      const int k = t - nv * M_NGRAD, v = k / 18;
      s_jac[v][k - v * 18] = __ldcg(a.jac + (static_cast<int64_t>(v) * C + c) * 18 + (k - v * 18));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // ncc per view and dL/dpose: per axis gc (a A + 2 b B) through the Jacobian
    double ga[3] = {0.0, 0.0, 0.0}, gtx = 0.0, gty = 0.0;
    const double s3[3] = {a.sx, a.sy, a.sz};
    for (int v = 0; v < nv; ++v) {
      double* m = s_mom[v];
      const double sq = sqrt(m[M_EP] * m[M_ET]);
      const double inv = 1.0 / (sq + 1e-8);
      m[17] = m[M_CROSS] * inv;
      const double bb = sq > 0.0 ? -0.5 * m[M_CROSS] * m[M_ET] * inv * inv / sq : 0.0;
      const double gc = -(a.g ? static_cast<double>(a.g[v * a.g_stride]) : 1.0) / C;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double du = gc * (inv * m[M_AU + i] + 2.0 * bb * m[M_BU + i]) * s3[i];
        const double dv = gc * (inv * m[M_AV + i] + 2.0 * bb * m[M_BV + i]) * s3[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) ga[k] += du * s_jac[v][(k * 2 + 0) * 3 + i] + dv * s_jac[v][(k * 2 + 1) * 3 + i];
      }
      gtx += gc * inv * a.kappa * m[M_PHU];
      gty += gc * inv * a.kappa * m[M_PHV];
      if (a.ncc_out) a.ncc_out[v * C + c] = static_cast<float>(m[17]);
      double* out = a.mom + (static_cast<int64_t>(v) * C + c) * kMomStride;
      for (int k = 0; k < kMomStride; ++k) out[k] = m[k];
    }
    float* o = a.grad + 6 * c;
    const float r[6] = {static_cast<float>(ga[0]), static_cast<float>(ga[1]), static_cast<float>(ga[2]),
                        static_cast<float>(gtx), static_cast<float>(gty), 0.f};
    for (int k = 0; k < 6; ++k) o[k] = a.accumulate ? o[k] + r[k] : r[k];
    a.counters[c] = 0u;  // every ticket of candidate c has been taken
    // global ticket: the CTA that completes the last candidate forms the losses
    __threadfence();
    const bool last = atomicAdd(a.counters + C, 1u) == static_cast<unsigned>(C - 1);
    if (last) __threadfence();
    s_last = last;
  }
  __syncthreads();
  if (!s_last || threadIdx.x >= 32) return;
  // one warp: loss[v] = 1 - mean_c ncc (fixed lane order), loss[nv] = their sum;
  // every view's loads are issued before any sum
  double part[kMaxViews] = {0.0, 0.0, 0.0, 0.0};
  for (int k = threadIdx.x; k < C; k += 32) {
#pragma unroll
    for (int v = 0; v < kMaxViews; ++v)
      if (v < nv) part[v] += __ldcg(a.mom + (static_cast<int64_t>(v) * C + k) * kMomStride + 17);
  }
  double total = 0.0;
#pragma unroll
  for (int v = 0; v < kMaxViews; ++v) {
    if (v < nv) {
      const double l = 1.0 - warp_sum(part[v]) / C;
      if (threadIdx.x == 0) a.loss[v] = static_cast<float>(l);
      total += l;
    }
  }
  if (threadIdx.x == 0) {
    a.loss[nv] = static_cast<float>(total);
    a.counters[C] = 0u;
  }
}

// FUSE: the last CTA to finish a candidate (ticket per candidate) sums its
// tiles, writes its moments, ncc and pose gradient; the last candidate to
// finish (global ticket) forms the view losses.  Tickets reset themselves, so
// the counters stay zero between launches.  No CTA ever waits on another.
template <int DT, bool GRAD, int GROUP, int MINB, bool FUSE>
__global__ void __launch_bounds__(kSnccThreads, MINB) tc_sncc_moments_kernel(SnccArgs a) {
  constexpr int NM = GRAD ? M_NGRAD : 3;
  __shared__ double red[NM * (kSnccThreads / 32)];
  __shared__ double ax_s[8];
  extern __shared__ __align__(16) unsigned char tab_smem[];
  const int tile = blockIdx.x, c = blockIdx.y, v = blockIdx.z;
  // select the view's parameters without dynamic indexing of the parameter space
  const int lateral = v == 0 ? a.lateral[0] : v == 1 ? a.lateral[1] : v == 2 ? a.lateral[2] : a.lateral[3];
  const float2* __restrict__ ft = v == 0 ? a.ftarg[0] : v == 1 ? a.ftarg[1] : v == 2 ? a.ftarg[2] : a.ftarg[3];
  const int R = a.R, K = R * R;
  const int q_begin = tile * a.tile;
  const int q_end = min(q_begin + a.tile, K);
  const int row0 = q_begin / R;
  const AxisTables tab = axis_tables(tab_smem, R + a.tab_rows);
  if (threadIdx.x == 0) {
    if (FUSE && GRAD) {
      double jac[18];
      slice_axes_jac(a.poses + 6 * c, lateral, a.sx, a.sy, a.sz, ax_s, jac);
      if (tile == 0)  // one CTA per (view, candidate) stores the axes Jacobian for the epilogue
        for (int k = 0; k < 18; ++k) a.jac[(static_cast<int64_t>(v) * a.C + c) * 18 + k] = jac[k];
    } else {
      slice_axes(a.poses + 6 * c, lateral, a.sx, a.sy, a.sz, ax_s);
    }
  }
  __syncthreads();
  build_axis_tables(tab, R, row0, (q_end - 1) / R - row0 + 1, a.lin, ax_s, a.sx, a.sy, a.sz, a.kpi);
  __syncthreads();
  float acc[NM];  // per-thread partial over ~K*C*nv/(2*SMs*256) samples
#pragma unroll
  for (int m = 0; m < NM; ++m) acc[m] = 0.f;

  // this thread's samples: q = q_begin + threadIdx.x + 256 m, (i, j) = divmod(q, R)
  const int di = kSnccThreads / R, dj = kSnccThreads - di * R;
  int q = q_begin + threadIdx.x;
  int i = q / R, j = q - i * R;
  while (q < q_end) {
    Raw<DT> raw[GROUP];
    int rc[GROUP];  // row entry << 16 | column entry
    float hs[GROUP];
    float2 Ts[GROUP];
    // issue every load of the group before using any of them; only the loads
    // and the table entries stay live, positions and phases are re-derived
#pragma unroll
    for (int g = 0; g < GROUP; ++g) {
      const bool ok = q < q_end;
      const int rn = ok ? R + i - row0 : 0, cn = ok ? j : 0;
      rc[g] = (rn << 16) | cn;
      TabCell cell = tab_cell(a.st, tab.idx[rn], tab.frac[rn], tab.idx[cn], tab.frac[cn]);
      if (!ok) cell.e = -1;
      tab_load<DT>(a.st, cell, raw[g]);
      Ts[g] = ok ? __ldg(ft + q) : make_float2(0.f, 0.f);
      hs[g] = ok ? (a.hp ? __ldg(a.hp + q) : 1.f) : 0.f;
      q += kSnccThreads;
      i += di;
      j += dj;
      if (j >= R) {
        j -= R;
        ++i;
      }
    }
#pragma unroll
    for (int g = 0; g < GROUP; ++g) {
      const int rn = rc[g] >> 16, cn = rc[g] & 0xffff;
      const float4 fa = tab.frac[rn], fb = tab.frac[cn];
      const float2 pa = tab.ph[rn], pb = tab.ph[cn];
      float tx = fa.x + fb.x, ty = fa.y + fb.y, tz = fa.z + fb.z;
      if (tx >= 1.f) tx -= 1.f;
      if (ty >= 1.f) ty -= 1.f;
      if (tz >= 1.f) tz -= 1.f;
      Sample8 sm;
      tab_decode<DT>(raw[g], sm);
      Interp o;
      trilerp<GRAD>(sm, tx, ty, tz, o);
      // f16: the brick scale rides on the high-pass weight (every moment is
      // linear in h S or quadratic in it) instead of rescaling 8 values
      const float ku = fa.w, kv = fb.w, h = DT == FVR_F16 ? hs[g] * raw_scale(raw[g]) : hs[g];
      const float cs = pa.x * pb.x - pa.y * pb.y, sn = pa.y * pb.x + pa.x * pb.y;
      const float2 T = Ts[g];
      const float shr = h * (o.sr * cs - o.si * sn);
      const float shi = h * (o.sr * sn + o.si * cs);
      acc[M_CROSS] = fmaf(shr, T.x, fmaf(shi, T.y, acc[M_CROSS]));
      acc[M_EP] = fmaf(shr, shr, fmaf(shi, shi, acc[M_EP]));
      acc[M_ET] = fmaf(T.x, T.x, fmaf(T.y, T.y, acc[M_ET]));
      if constexpr (GRAD) {
        // dL/dphi direction: Re(conj(T) i S_hat) = T.y*shr - T.x*shi
        const float ph = T.y * shr - T.x * shi;
        acc[M_PHU] += ku * ph;
        acc[M_PHV] += kv * ph;
        // M_T = h e^{-i phi} T ;  A_k = <M_T, dS/dp_k> ;  B_k = h^2 <S, dS/dp_k>
        const float mtr = h * (cs * T.x + sn * T.y);
        const float mti = h * (cs * T.y - sn * T.x);
        const float h2 = h * h;
        const float a0 = mtr * o.dxr + mti * o.dxi, a1 = mtr * o.dyr + mti * o.dyi, a2 = mtr * o.dzr + mti * o.dzi;
        const float b0 = h2 * (o.sr * o.dxr + o.si * o.dxi), b1 = h2 * (o.sr * o.dyr + o.si * o.dyi),
                    b2 = h2 * (o.sr * o.dzr + o.si * o.dzi);
        acc[M_AU + 0] += ku * a0;
        acc[M_AU + 1] += ku * a1;
        acc[M_AU + 2] += ku * a2;
        acc[M_AV + 0] += kv * a0;
        acc[M_AV + 1] += kv * a1;
        acc[M_AV + 2] += kv * a2;
        acc[M_BU + 0] += ku * b0;
        acc[M_BU + 1] += ku * b1;
        acc[M_BU + 2] += ku * b2;
        acc[M_BV + 0] += kv * b0;
        acc[M_BV + 1] += kv * b1;
        acc[M_BV + 2] += kv * b2;
      }
    }
  }
  double tot;
  block_reduce_d<NM, float>(acc, red, &tot);
  if (threadIdx.x < NM)
    a.partial[((static_cast<int64_t>(v) * a.C + c) * gridDim.x + tile) * NM + threadIdx.x] = tot;
  if constexpr (FUSE && GRAD) sncc_fused_epilogue(a, c);
}

// Tile sums (fp64, fixed order) -> mom[v][c][0..NM), ncc in mom[v][c][17];
// loss[v] = 1 - mean_c ncc, loss[nv] = sum_v loss[v].  One CTA, warp per (v, c).
__global__ void __launch_bounds__(1024) tc_sncc_finalize_kernel(const double* __restrict__ partial, int C, int nv,
                                                                int tiles, int NM, double* __restrict__ mom,
                                                                float* __restrict__ loss,
                                                                float* __restrict__ ncc_out) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int item = w; item < nv * C; item += nw) {
    double s = 0.0;
    if (lane < NM) {
      for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(item) * tiles + t) * NM + lane];
      mom[static_cast<int64_t>(item) * kMomStride + lane] = s;
    }
    const double cross = __shfl_sync(0xffffffffu, s, 0), ep = __shfl_sync(0xffffffffu, s, 1),
                 et = __shfl_sync(0xffffffffu, s, 2);
    if (lane == 0) {
      const double n = cross / (sqrt(ep * et) + 1e-8);
      mom[static_cast<int64_t>(item) * kMomStride + 17] = n;
      if (ncc_out) ncc_out[item] = static_cast<float>(n);
    }
  }
  __syncthreads();
  double total = 0.0;
  for (int v = 0; v < nv; ++v) {
    double s = 0.0;
    for (int c = threadIdx.x; c < C; c += blockDim.x) s += mom[(static_cast<int64_t>(v) * C + c) * kMomStride + 17];
    s = warp_sum(s);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < nw; ++k) t += red[k];
      const double l = 1.0 - t / C;
      loss[v] = static_cast<float>(l);
      total += l;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[nv] = static_cast<float>(total);
}

struct SnccGradArgs {
  const double* mom;  // [nv][C][18]
  const float* g;     // dL/dloss_v at g[v * g_stride]
  int g_stride;
  const float* poses;
  int C, nv;
  int lateral[kMaxViews];
  double sx, sy, sz, kappa;
  float* grad;  // [C][6]
  int accumulate;
};

__global__ void tc_sncc_grad_kernel(SnccGradArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.C) return;
  float r[6];
  sncc_pose_grad(a.mom + static_cast<int64_t>(c) * kMomStride, static_cast<int64_t>(a.C) * kMomStride,
                 a.poses + 6 * c, a.nv, lateral_bits(a.lateral), a.g, a.g_stride, a.C, a.sx, a.sy, a.sz, a.kappa, r);
  float* o = a.grad + 6 * c;
  for (int k = 0; k < 6; ++k) o[k] = a.accumulate ? o[k] + r[k] : r[k];
}

// ----------------------------------------------------------------------------
// image path: modulated slice and its adjoint  (torch_engine.py:176-241)
// ----------------------------------------------------------------------------

struct SliceArgs {
  Stencil st;
  const double* axes;  // [C][8]
  const float* lin;
  int R;
  double kpi;
  double sx, sy, sz;
  int shift;  // 1: position ifftshift(q) (image path), 0: natural order
};

__device__ __forceinline__ int shifted_pos(int i, int j, int R, int shift) {
  if (shift) {  // ifftshift: element (i, j) lands at ((i - R/2) mod R, (j - R/2) mod R)
    const int h = R / 2;
    i -= h;
    if (i < 0) i += R;
    j -= h;
    if (j < 0) j += R;
  }
  return i * R + j;
}

template <int DT, bool DERIV>
__device__ __forceinline__ void slice_sample(const SliceArgs& a, const double* ax, float ku, float kv, Interp& o,
                                             float& sn, float& cs) {
  const double dku = ku, dkv = kv;
  stencil_sample_d<DT, DERIV, false>(a.st, fma(dkv, ax[3], fma(dku, ax[0], a.sx)),
                                     fma(dkv, ax[4], fma(dku, ax[1], a.sy)), fma(dkv, ax[5], fma(dku, ax[2], a.sz)),
                                     o);
  phase_sincos(a.kpi, ku, kv, static_cast<float>(ax[6]), static_cast<float>(ax[7]), &sn, &cs);
}

template <int DT>
__global__ void __launch_bounds__(256) tc_slice_kernel(SliceArgs a, float2* __restrict__ out) {
  const int c = blockIdx.y, R = a.R;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= R * R) return;
  const int i = q / R, j = q - (q / R) * R;
  Interp o;
  float sn, cs;
  slice_sample<DT, false>(a, a.axes + 8 * c, __ldg(a.lin + i), __ldg(a.lin + j), o, sn, cs);
  out[static_cast<int64_t>(c) * R * R + shifted_pos(i, j, R, a.shift)] =
      make_float2(o.sr * cs - o.si * sn, o.sr * sn + o.si * cs);
}

// Given G = dL/dS_hat per sample: partials (dU[3], dV[3], PHU, PHV) per
// (candidate, tile) with dL/dS = e^{-i phi} G and dL/dphi = Re(conj(G) i S_hat).
template <int DT>
__global__ void __launch_bounds__(256) tc_slice_adjoint_kernel(SliceArgs a, const float2* __restrict__ G,
                                                               double* __restrict__ partial) {
  __shared__ double red[8 * 8];
  const int c = blockIdx.y, R = a.R;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (q < R * R) {
    const int i = q / R, j = q - (q / R) * R;
    const float ku = __ldg(a.lin + i), kv = __ldg(a.lin + j);
    Interp o;
    float sn, cs;
    slice_sample<DT, true>(a, a.axes + 8 * c, ku, kv, o, sn, cs);
    const float2 g = __ldg(G + static_cast<int64_t>(c) * R * R + shifted_pos(i, j, R, a.shift));
    const float shr = o.sr * cs - o.si * sn, shi = o.sr * sn + o.si * cs;
    const float ph = g.y * shr - g.x * shi;
    const float dr = cs * g.x + sn * g.y, di = cs * g.y - sn * g.x;  // e^{-i phi} G
    const float e0 = dr * o.dxr + di * o.dxi, e1 = dr * o.dyr + di * o.dyi, e2 = dr * o.dzr + di * o.dzi;
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
  block_reduce_d<8, double>(acc, red, &tot);
  if (threadIdx.x < 8) partial[(static_cast<int64_t>(c) * gridDim.x + blockIdx.x) * 8 + threadIdx.x] = tot;
}

__global__ void tc_adjoint_grad_kernel(const double* __restrict__ part, int tiles, const float* __restrict__ poses,
                                       int C, int lateral, double sx, double sy, double sz, double kappa,
                                       float* __restrict__ grad, int accumulate) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < tiles; ++i)
    for (int m = 0; m < 8; ++m) t[m] += part[(static_cast<int64_t>(c) * tiles + i) * 8 + m];
  const double du[3] = {t[0], t[1], t[2]}, dv[3] = {t[3], t[4], t[5]};
  double ga[3];
  axes_vjp(poses + 6 * c, lateral, sx, sy, sz, du, dv, ga);
  float* o = grad + 6 * c;
  const float r[6] = {static_cast<float>(ga[0]), static_cast<float>(ga[1]), static_cast<float>(ga[2]),
                      static_cast<float>(kappa * t[6]), static_cast<float>(kappa * t[7]), 0.f};
  for (int k = 0; k < 6; ++k) o[k] = accumulate ? o[k] + r[k] : r[k];
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

static double half_extent(int64_t n) { return 0.5 * static_cast<double>(n > 1 ? n - 1 : 1); }

// Samples per CTA: one wave of min_blocks resident CTAs per SM (never more
// CTAs than slots), at least 256 samples (one per thread) per CTA.
static int sncc_tile(int64_t C, int64_t K, int nv, int variant) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const SnccVariant v = sncc_variant(variant);
  const int64_t items = C * nv;
  int64_t tiles = (static_cast<int64_t>(v.min_blocks) * sms) / items;
  const int64_t max_tiles = cdiv64(K, kSnccThreads);
  if (tiles > max_tiles) tiles = max_tiles;
  if (tiles < 1) tiles = 1;
  return static_cast<int>(cdiv64(K, tiles));
}

// Row-table entries and dynamic shared memory of one moments CTA.
static int sncc_tab_rows(int64_t R, int tile) { return static_cast<int>(tile / R + 2); }
static int64_t sncc_smem(int64_t R, int tile) { return (R + sncc_tab_rows(R, tile)) * 40; }
constexpr int64_t kSnccMaxSmem = 200 * 1024;

template <int DT, bool GRAD, int GROUP, int MINB, bool FUSE>
static void launch_sncc_v(dim3 grid, int smem, cudaStream_t s, const SnccArgs& a) {
  auto k = tc_sncc_moments_kernel<DT, GRAD, GROUP, MINB, FUSE>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k<<<grid, kSnccThreads, smem, s>>>(a);
}

template <int DT, bool GRAD, bool FUSE = false>
static void launch_sncc(int variant, dim3 grid, int smem, cudaStream_t s, const SnccArgs& a) {
  switch (variant) {
    case 1: launch_sncc_v<DT, GRAD, 2, 4, FUSE>(grid, smem, s, a); break;
    case 2: launch_sncc_v<DT, GRAD, 4, 3, FUSE>(grid, smem, s, a); break;
    case 3: launch_sncc_v<DT, GRAD, 8, 1, FUSE>(grid, smem, s, a); break;
    case 4: launch_sncc_v<DT, GRAD, 2, 3, FUSE>(grid, smem, s, a); break;
    case 5: launch_sncc_v<DT, GRAD, 3, 3, FUSE>(grid, smem, s, a); break;
    default: launch_sncc_v<DT, GRAD, 4, 2, FUSE>(grid, smem, s, a); break;
  }
}

// Shared argument set-up of the moments launches.
static int sncc_setup(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                      const float* poses, int64_t C, int nviews, const int* views, const void* const* ftargs,
                      const float* hp, const float* lin, int64_t R, double kappa, int variant, SnccArgs* a,
                      dim3* grid, int64_t* smem) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!poses || !views || !ftargs || !lin || C < 1 || R < 1 || C > 65535) return FVR_ERR_ARG;
  if (nviews < 1 || nviews > kMaxViews || R * R > (int64_t)1 << 30) return FVR_ERR_ARG;
  if (variant < 0 || variant >= kSnccVariants) return FVR_ERR_ARG;
  if ((D + 1) * (H + 1) * (W + 1) > INT32_MAX) return FVR_ERR_UNSUPPORTED;  // 32-bit entry index
  const int64_t K = R * R;
  const int tile = sncc_tile(C, K, nviews, variant);
  *a = SnccArgs{};
  a->st = st;
  a->poses = poses;
  for (int v = 0; v < nviews; ++v) {
    if (!ftargs[v] || (views[v] != 0 && views[v] != 1)) return FVR_ERR_ARG;
    a->ftarg[v] = static_cast<const float2*>(ftargs[v]);
    a->lateral[v] = views[v];
  }
  a->hp = hp;
  a->lin = lin;
  a->R = (int)R;
  a->C = (int)C;
  a->tile = tile;
  a->tab_rows = sncc_tab_rows(R, tile);
  *smem = sncc_smem(R, tile);
  if (*smem > kSnccMaxSmem) return FVR_ERR_UNSUPPORTED;
  a->kpi = kappa / 3.14159265358979323846;
  a->kappa = kappa;
  a->sx = half_extent(W);
  a->sy = half_extent(H);
  a->sz = half_extent(D);
  *grid = dim3(static_cast<unsigned>(cdiv64(K, tile)), static_cast<unsigned>(C), static_cast<unsigned>(nviews));
  return FVR_OK;
}

// ----------------------------------------------------------------------------
// Scratch of the allocation-free value-and-gradient entry point.
//
// fvr_tc_sncc_value_and_grad_static computes exactly what
// fvr_tc_sncc_value_and_grad computes, with its workspace in this fixed
// file-scope device array instead of caller memory.  It serves callers that
// cannot allocate device memory where they call: a host program that links
// only this C ABI and owns no device allocator, or a loop that must not enter
// an allocator between steps (cudaMalloc / cudaFree may synchronise the
// device).
//
// Size (about 428 KB per device): kStaticRecords partial-moment records of
// 17 doubles, kStaticItems (candidate, view) moment records and axes
// Jacobians of 18 doubles each, and kStaticItems + 1 ticket counters.  Calls
// needing more -- more than 512 (candidate, view) pairs, or more than 2048
// (candidate, view, tile) partial records for the launch variant -- are
// refused with FVR_ERR_WORKSPACE before anything is launched.
//
// Start state: the ticket counters must be zero before a launch; the static
// initialiser zeroes them and every completed launch leaves them zero.  The
// partial, moment and Jacobian records are written by every launch before
// they are read, so nothing else needs to start at zero.
//
// Set-up: the first call on each device, made with that device current,
// resolves the array's device address with cudaGetSymbolAddress and caches
// it; make that first call before any stream capture begins.
//
// Races: one array per device is shared by every caller in the process.
// Calls on the same device must be ordered (one stream, or explicit
// synchronisation); two calls that overlap in time corrupt each other's
// scratch and tickets.
// ----------------------------------------------------------------------------
constexpr int64_t kStaticItems = 512;
constexpr int64_t kStaticRecords = 2048;
constexpr int64_t kStaticPartialDoubles = kStaticRecords * M_NGRAD;
constexpr int64_t kStaticMomDoubles = kStaticItems * kMomStride;
constexpr int64_t kStaticJacDoubles = kStaticItems * 18;
constexpr int64_t kStaticTicketDoubles = (kStaticItems + 1 + 1) / 2;  // unsigned counters, two per double
constexpr int64_t kStaticDoubles = kStaticPartialDoubles + kStaticMomDoubles + kStaticJacDoubles +
                                   kStaticTicketDoubles;
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) double g_sncc_static_scratch[kStaticDoubles];

static std::mutex g_static_mu;
static double* g_static_ptr[kStaticMaxDevices] = {};

// Device address of this device's scratch array (resolved once per device).
static int static_scratch(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return FVR_ERR_CUDA;
  if (dev < 0 || dev >= kStaticMaxDevices) return FVR_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_sncc_static_scratch);
    if (rc != cudaSuccess || !p) return FVR_ERR_CUDA;
    g_static_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_static_ptr[dev];
  return FVR_OK;
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_tc_axes(const float* poses, int64_t C, int view, int64_t D, int64_t H, int64_t W, double* axes,
                void* stream) {
  if (!poses || !axes || C < 1 || (view != 0 && view != 1)) return FVR_ERR_ARG;
  tc_axes_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      poses, (int)C, view, half_extent(W), half_extent(H), half_extent(D), axes);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int64_t fvr_tc_sncc_workspace(int64_t C, int64_t R, int64_t nviews) {
  return nviews * C * cdiv64(R * R, kSnccThreads) * M_NGRAD * (int64_t)sizeof(double);
}

int64_t fvr_tc_sncc_mom_stride(void) { return kMomStride; }

int fvr_tc_sncc_variants(void) { return kSnccVariants; }

int fvr_tc_sncc_moments(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                        const float* poses, int64_t C, int nviews, const int* views, const void* const* ftargs,
                        const float* hp, const float* lin, int64_t R, double kappa, int with_grad, int variant,
                        void* workspace, int64_t ws_bytes, void* stream) {
  SnccArgs a;
  dim3 grid;
  int64_t smem = 0;
  int rc = sncc_setup(dtype, stencil, scales, D, H, W, poses, C, nviews, views, ftargs, hp, lin, R, kappa, variant,
                      &a, &grid, &smem);
  if (rc) return rc;
  if (!workspace) return FVR_ERR_ARG;
  if (ws_bytes < fvr_tc_sncc_workspace(C, R, nviews)) return FVR_ERR_WORKSPACE;
  a.partial = static_cast<double*>(workspace);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define FVR_SNCC(DT)                                         \
  if (with_grad)                                             \
    launch_sncc<DT, true>(variant, grid, (int)smem, s, a);   \
  else                                                       \
    launch_sncc<DT, false>(variant, grid, (int)smem, s, a);  \
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

// Fused workspace: partial records | moments [nv][C][18] | axes Jacobians
// [nv][C][18] | tickets [C + 1] (the last region must start zeroed).
int64_t fvr_tc_sncc_fused_workspace(int64_t C, int64_t R, int64_t nviews) {
  if (C < 1 || R < 1 || nviews < 1) return 0;
  return fvr_tc_sncc_workspace(C, R, nviews) + 2 * nviews * C * kMomStride * (int64_t)sizeof(double) +
         cdiv64((C + 1) * (int64_t)sizeof(unsigned), 256) * 256;
}

int fvr_tc_sncc_value_and_grad(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                               const float* poses, int64_t C, int nviews, const int* views,
                               const void* const* ftargs, const float* hp, const float* lin, int64_t R,
                               double kappa, int variant, const float* g, int64_t g_stride, void* workspace,
                               int64_t ws_bytes, float* loss, float* ncc_out, float* grad_poses, int accumulate,
                               void* stream) {
  SnccArgs a;
  dim3 grid;
  int64_t smem = 0;
  int rc = sncc_setup(dtype, stencil, scales, D, H, W, poses, C, nviews, views, ftargs, hp, lin, R, kappa, variant,
                      &a, &grid, &smem);
  if (rc) return rc;
  if (!workspace || !loss || !grad_poses) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return FVR_ERR_ARG;
  if (ws_bytes < fvr_tc_sncc_fused_workspace(C, R, nviews)) return FVR_ERR_WORKSPACE;
  char* ws = static_cast<char*>(workspace);
  a.partial = reinterpret_cast<double*>(ws);
  const int64_t mom_bytes = nviews * C * kMomStride * (int64_t)sizeof(double);
  a.mom = reinterpret_cast<double*>(ws + fvr_tc_sncc_workspace(C, R, nviews));
  a.jac = reinterpret_cast<double*>(ws + fvr_tc_sncc_workspace(C, R, nviews) + mom_bytes);
  a.counters = reinterpret_cast<unsigned*>(ws + fvr_tc_sncc_workspace(C, R, nviews) + 2 * mom_bytes);
  a.loss = loss;
  a.ncc_out = ncc_out;
  a.grad = grad_poses;
  a.g = g;
  a.g_stride = (int)g_stride;
  a.accumulate = accumulate;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FVR_F32: launch_sncc<FVR_F32, true, true>(variant, grid, (int)smem, s, a); break;
    case FVR_BF16: launch_sncc<FVR_BF16, true, true>(variant, grid, (int)smem, s, a); break;
    case FVR_F16: launch_sncc<FVR_F16, true, true>(variant, grid, (int)smem, s, a); break;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_finalize(const void* workspace, int64_t C, int64_t R, int nviews, int with_grad, int variant,
                         double* mom, float* loss, float* ncc_out, void* stream) {
  if (!workspace || !mom || !loss || C < 1 || R < 1 || nviews < 1 || nviews > kMaxViews) return FVR_ERR_ARG;
  if (variant < 0 || variant >= kSnccVariants) return FVR_ERR_ARG;
  const int64_t K = R * R;
  const int tiles = static_cast<int>(cdiv64(K, sncc_tile(C, K, nviews, variant)));
  tc_sncc_finalize_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const double*>(workspace), (int)C, nviews, tiles, with_grad ? M_NGRAD : 3, mom, loss, ncc_out);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_backward(const double* mom, int nviews, const int* views, const float* g, int64_t g_stride,
                         const float* poses, int64_t C, int64_t D, int64_t H, int64_t W, double kappa,
                         float* grad_poses, int accumulate, void* stream) {
  if (!mom || !views || !g || !poses || !grad_poses || C < 1 || nviews < 1 || nviews > kMaxViews)
    return FVR_ERR_ARG;
  SnccGradArgs a{};
  a.mom = mom;
  a.g = g;
  a.g_stride = (int)g_stride;
  a.poses = poses;
  a.C = (int)C;
  a.nv = nviews;
  for (int v = 0; v < nviews; ++v) {
    if (views[v] != 0 && views[v] != 1) return FVR_ERR_ARG;
    a.lateral[v] = views[v];
  }
  a.sx = half_extent(W);
  a.sy = half_extent(H);
  a.sz = half_extent(D);
  a.kappa = kappa;
  a.grad = grad_poses;
  a.accumulate = accumulate;
  tc_sncc_grad_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, static_cast<cudaStream_t>(stream)>>>(a);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_slice(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                 const double* axes, int64_t C, const float* lin, int64_t R, double kappa, int shift, void* out,
                 void* stream) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!axes || !lin || !out || C < 1 || R < 1 || C > 65535 || R * R > (int64_t)1 << 30) return FVR_ERR_ARG;
  SliceArgs a{st, axes, lin, (int)R, kappa / 3.14159265358979323846, half_extent(W), half_extent(H),
              half_extent(D), shift ? 1 : 0};
  dim3 grid(static_cast<unsigned>(cdiv64(R * R, 256)), static_cast<unsigned>(C));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
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
                         const double* axes, const float* poses, int64_t C, int view, const float* lin, int64_t R,
                         double kappa, int shift, const void* G, void* workspace, int64_t ws_bytes,
                         float* grad_poses, int accumulate, void* stream) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st);
  if (rc) return rc;
  if (!axes || !poses || !lin || !G || !workspace || !grad_poses || C < 1 || R < 1 || C > 65535)
    return FVR_ERR_ARG;
  if (view != 0 && view != 1) return FVR_ERR_ARG;
  if (ws_bytes < fvr_tc_slice_adjoint_workspace(C, R)) return FVR_ERR_WORKSPACE;
  SliceArgs a{st, axes, lin, (int)R, kappa / 3.14159265358979323846, half_extent(W), half_extent(H),
              half_extent(D), shift ? 1 : 0};
  const int tiles = static_cast<int>(cdiv64(R * R, 256));
  dim3 grid(static_cast<unsigned>(tiles), static_cast<unsigned>(C));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  const float2* g = static_cast<const float2*>(G);
  switch (dtype) {
    case FVR_F32: tc_slice_adjoint_kernel<FVR_F32><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_BF16: tc_slice_adjoint_kernel<FVR_BF16><<<grid, 256, 0, s>>>(a, g, part); break;
    case FVR_F16: tc_slice_adjoint_kernel<FVR_F16><<<grid, 256, 0, s>>>(a, g, part); break;
  }
  FVR_LAUNCH_CHECK();
  tc_adjoint_grad_kernel<<<static_cast<unsigned>(cdiv64(C, 128)), 128, 0, s>>>(
      part, tiles, poses, (int)C, view, half_extent(W), half_extent(H), half_extent(D), kappa, grad_poses,
      accumulate);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_value_and_grad_static(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H,
                                      int64_t W, const float* poses, int64_t C, int nviews, const int* views,
                                      const void* const* ftargs, const float* hp, const float* lin, int64_t R,
                                      double kappa, int variant, const float* g, int64_t g_stride, float* loss,
                                      float* ncc_out, float* grad_poses, int accumulate, void* stream) {
  SnccArgs a;
  dim3 grid;
  int64_t smem = 0;
  int rc = sncc_setup(dtype, stencil, scales, D, H, W, poses, C, nviews, views, ftargs, hp, lin, R, kappa, variant,
                      &a, &grid, &smem);
  if (rc) return rc;
  if (!loss || !grad_poses) return FVR_ERR_ARG;
  const int64_t items = C * nviews;
  if (items > kStaticItems || items * static_cast<int64_t>(grid.x) > kStaticRecords) return FVR_ERR_WORKSPACE;
  double* scratch = nullptr;
  rc = static_scratch(&scratch);
  if (rc) return rc;
  a.partial = scratch;
  a.mom = scratch + kStaticPartialDoubles;
  a.jac = scratch + kStaticPartialDoubles + kStaticMomDoubles;
  a.counters = reinterpret_cast<unsigned*>(scratch + kStaticPartialDoubles + kStaticMomDoubles + kStaticJacDoubles);
  a.loss = loss;
  a.ncc_out = ncc_out;
  a.grad = grad_poses;
  a.g = g;
  a.g_stride = (int)g_stride;
  a.accumulate = accumulate;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FVR_F32: launch_sncc<FVR_F32, true, true>(variant, grid, (int)smem, s, a); break;
    case FVR_BF16: launch_sncc<FVR_BF16, true, true>(variant, grid, (int)smem, s, a); break;
    case FVR_F16: launch_sncc<FVR_F16, true, true>(variant, grid, (int)smem, s, a); break;
  }
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
