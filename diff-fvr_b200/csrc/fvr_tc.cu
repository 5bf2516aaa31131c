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
#include <algorithm>
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
// autotuner): rows per thread whose loads are in flight together (a group),
// and the resident CTAs per SM the register budget is sized for.
struct SnccVariant {
  int group, min_blocks;
};
constexpr SnccVariant kSnccVariantTable[] = {{4, 2}, {2, 4}, {4, 3}, {8, 1}, {2, 3}, {3, 3}, {6, 1}, {3, 2}};
constexpr int kSnccVariants = sizeof(kSnccVariantTable) / sizeof(kSnccVariantTable[0]);
constexpr SnccVariant sncc_variant(int v) { return kSnccVariantTable[v]; }

struct SnccArgs {
  Stencil st;
  const float* poses;  // [C][6]
  const float2* ftarg[kMaxViews];
  int lateral[kMaxViews];
  const float* hp;   // [R*R] or null
  const float* lin;  // [R]
  int R, C, nv;
  int tile_rows;     // slice rows per CTA (= row-table entries)
  int tiles;         // CTAs per (candidate, view): record (v * C + c) * tiles + tile
  double kpi;        // kappa / pi
  double sx, sy, sz;
  double* partial;  // partial-moment records of NM doubles
  // value-and-gradient epilogue only
  double* mom;         // [nv][C][kMomStride]
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

// Per-(candidate, view) sample tables of the moments kernels (see
// AxisTables): integer cell, fraction, and (k, k, cos, sin) with the grid
// value k kept as a pair for the packed moment products.  48 B per entry.
// Column entries' integer parts include the stencil's +1 entry offset.
struct SnccTab {
  int4* idx;    // (floor x, floor y, floor z, -), columns + 1
  float4* frac; // (frac x, frac y, frac z, k)
  float4* kph;  // (k, k, cos, sin)
};
constexpr int kSnccTabEntryBytes = 48;

__device__ __forceinline__ SnccTab sncc_tab(unsigned char* smem, int n_tab) {
  SnccTab t;
  t.idx = reinterpret_cast<int4*>(smem);
  t.frac = reinterpret_cast<float4*>(smem + 16 * n_tab);
  t.kph = reinterpret_cast<float4*>(smem + 32 * n_tab);
  return t;
}

__device__ __forceinline__ void build_sncc_tables(const SnccTab& t, int R, int row0, int n_row,
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
    const int one = col ? 1 : 0;  // entry = voxel + 1, carried by the column part
    t.idx[n] = make_int4(static_cast<int>(fx) + one, static_cast<int>(fy) + one, static_cast<int>(fz) + one, 0);
    t.frac[n] = make_float4(static_cast<float>(px - fx), static_cast<float>(py - fy), static_cast<float>(pz - fz), kf);
    double sn, cs;
    sincospi(kpi * k * (col ? ax[7] : ax[6]), &sn, &cs);
    t.kph[n] = make_float4(kf, kf, static_cast<float>(cs), static_cast<float>(sn));
  }
}

// view v's parameters without dynamic indexing of the kernel parameter space
__device__ __forceinline__ int view_lateral(const SnccArgs& a, int v) {
  return v == 0 ? a.lateral[0] : v == 1 ? a.lateral[1] : v == 2 ? a.lateral[2] : a.lateral[3];
}
__device__ __forceinline__ const float2* view_target(const SnccArgs& a, int v) {
  return v == 0 ? a.ftarg[0] : v == 1 ? a.ftarg[1] : v == 2 ? a.ftarg[2] : a.ftarg[3];
}

// Slice axes of (candidate c, view v) into ax[8].
__device__ __forceinline__ void sncc_item_axes(const SnccArgs& a, int v, int c, double* ax) {
  slice_axes(a.poses + 6 * c, view_lateral(a, v), a.sx, a.sy, a.sz, ax);
}

// Programmatic dependent launch (sm_90+): a kernel launched after this one
// with programmatic stream serialisation may start once every CTA of this
// grid has signalled; griddepcontrol.wait in that kernel still returns only
// when this grid has completed and its memory is visible.  Both are no-ops
// without such a launch.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Cell of the sample at (row entry a, column entry b) for the moments
// kernels: the column table's integer part already carries the +1 entry
// offset of the stencil (entry = voxel + 1); e = -1 when no corner of the
// cell is inside (zero-padding partial: -1 <= p < n on every axis).
struct SCell {
  int e;
  float tx, ty, tz;
  int ex, ey, ez;
};

template <int DT>
__device__ __forceinline__ SCell sncc_cell(const Stencil& s, int4 ia, float4 fa, int4 ib1, float4 fb) {
  SCell c;
  c.tx = fa.x + fb.x;
  c.ty = fa.y + fb.y;
  c.tz = fa.z + fb.z;
  c.ex = ia.x + ib1.x;
  c.ey = ia.y + ib1.y;
  c.ez = ia.z + ib1.z;
  if (c.tx >= 1.f) { c.tx -= 1.f; ++c.ex; }
  if (c.ty >= 1.f) { c.ty -= 1.f; ++c.ey; }
  if (c.tz >= 1.f) { c.tz -= 1.f; ++c.ez; }
  const bool ok = static_cast<unsigned>(c.ex) <= static_cast<unsigned>(s.W) &&
                  static_cast<unsigned>(c.ey) <= static_cast<unsigned>(s.H) &&
                  static_cast<unsigned>(c.ez) <= static_cast<unsigned>(s.D);
  // x-pair storage: W + 2 entries per x row, the cell's two at e and e + 1
  c.e = ok ? (c.ez * (s.H + 1) + c.ey) * (s.W + (is_pair(DT) ? 2 : 1)) + c.ex : -1;
  return c;
}

// Entry load of cell c (zeros when e < 0); f16: the brick scale, unapplied.
template <int DT>
__device__ __forceinline__ void sncc_load(const Stencil& s, const SCell& c, Raw<DT>& r) {
  if constexpr (is_pair(DT)) {
    pair_load<DT>(s, c.e, c.ez, c.ey, r);
  } else if constexpr (DT == FVR_F32) {
    if (c.e < 0 || !fvr_checked(c.e, stencil_entries(s), kSiteStencilEntry)) {
#pragma unroll
      for (int i = 0; i < 4; ++i) r.q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      return;
    }
    const float4* p = static_cast<const float4*>(s.data) + static_cast<int64_t>(c.e) * 4;
    ldg256(p, r.q[0], r.q[1]);
    ldg256(p + 2, r.q[2], r.q[3]);
  } else {
    if (c.e < 0 || !fvr_checked(c.e, stencil_entries(s), kSiteStencilEntry)) {
      r.q[0] = r.q[1] = make_uint4(0u, 0u, 0u, 0u);
      if constexpr (DT == FVR_F16) r.sc = 0.f;
      return;
    }
    ldg256(static_cast<const uint4*>(s.data) + static_cast<int64_t>(c.e) * 2, r.q[0], r.q[1]);
    if constexpr (DT == FVR_F16) {
      const unsigned bx = static_cast<unsigned>(s.W + kBrick) / kBrick, by = static_cast<unsigned>(s.H + kBrick) / kBrick;
      const unsigned ex = static_cast<unsigned>(c.ex) / kBrick, ey = static_cast<unsigned>(c.ey) / kBrick,
                     ez = static_cast<unsigned>(c.ez) / kBrick;
      const unsigned si = (ez * by + ey) * bx + ex;
      r.sc = fvr_checked(si, stencil_scales(s), kSiteStencilScale) ? __ldg(s.scales + si) : 0.f;
    }
  }
}

// The per-sample reduction.  With S the interpolated sample, D_k its
// derivative along axis k, P = e^{i phi} the phase factor, T the target and h
// the high-pass weight (f16: times the brick scale), and M = h conj(P) T:
//   cross = S.M    Ep = h^2 S.S    Et = T.T    ph = S x M = Im(conj(S) M)
//   A_k = M.D_k    B_k = h^2 S.D_k,    (PHU, AU, BU) weighted by ku, (PHV, AV, BV) by kv,
// where x.y = Re(x conj y).  Pair accumulators hold the two component
// products in packed (re, im) form; acc.x + acc.y is the moment (acc.y -
// acc.x for the ph pair, which multiplies (si, sr) by M).
template <int DT, bool GRAD, int NM>
__device__ __forceinline__ void sncc_accumulate(const Raw<DT>& raw, float tx, float ty, float tz, float4 ka,
                                                float4 kb, float2 T, float h, float2 (&acc)[NM]) {
  Sample8c sm;
  tab_decode2<DT>(raw, sm);
  Interp2 o;
  trilerp2<GRAD>(sm, tx, ty, tz, o);
  const float cs = ka.z * kb.z - ka.w * kb.w, sn = ka.w * kb.z + ka.z * kb.w;
  const float htx = h * T.x, hty = h * T.y;
  const float2 M = make_float2(cs * htx + sn * hty, cs * hty - sn * htx);
  const float2 hS = mul2(f2(h * h), o.s);
  acc[M_CROSS] = fma2(o.s, M, acc[M_CROSS]);
  acc[M_EP] = fma2(hS, o.s, acc[M_EP]);
  acc[M_ET] = fma2(T, T, acc[M_ET]);
  if constexpr (GRAD) {
    const float2 kU = make_float2(ka.x, ka.y), kV = make_float2(kb.x, kb.y);
    const float2 uM = mul2(kU, M), vM = mul2(kV, M), uH = mul2(kU, hS), vH = mul2(kV, hS);
    const float2 sw = make_float2(o.s.y, o.s.x);
    acc[M_PHU] = fma2(sw, uM, acc[M_PHU]);
    acc[M_PHV] = fma2(sw, vM, acc[M_PHV]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      acc[M_AU + k] = fma2(uM, o.d[k], acc[M_AU + k]);
      acc[M_AV + k] = fma2(vM, o.d[k], acc[M_AV + k]);
      acc[M_BU + k] = fma2(uH, o.d[k], acc[M_BU + k]);
      acc[M_BV + k] = fma2(vH, o.d[k], acc[M_BV + k]);
    }
  }
}

// Rows [row_begin, row_end) of one (candidate, view), column-stationary: the
// CTA's 256 threads cover min(R, 256) columns x 256 / min(R, 256) rows per
// pass, so a thread keeps its column's table entry in registers for the
// whole range and every lane of a warp reads the same row entry (a
// broadcast).  GROUP rows' loads are in flight before any of them is used.
// Threads past the last whole column set (R < 256 not dividing 256) idle.
template <int DT, bool GRAD, int GROUP, int NM>
__device__ __forceinline__ void sncc_run(const SnccArgs& a, const SnccTab& tab, const float2* __restrict__ ft,
                                         int row_begin, int row_end, float2 (&acc)[NM]) {
  const int R = a.R, t = threadIdx.x;
  const int cpp = min(R, kSnccThreads), rpp = kSnccThreads / cpp;
  const int r_off = t / cpp;
  if (r_off >= rpp) return;
  for (int j = t - r_off * cpp; j < R; j += cpp) {
    const int4 ib = tab.idx[j];
    const float4 fb = tab.frac[j], kb = tab.kph[j];
    for (int i = row_begin + r_off; i < row_end; i += rpp * GROUP) {
      Raw<DT> raw[GROUP];
      float hs[GROUP];
      float2 Ts[GROUP];
      // issue every load of the group before using any of them
#pragma unroll
      for (int g = 0; g < GROUP; ++g) {
        const int ig = i + g * rpp;
        const bool ok = ig < row_end;
        const int rn = R + (ok ? ig : row_begin) - row_begin;
        SCell cell = sncc_cell<DT>(a.st, tab.idx[rn], tab.frac[rn], ib, fb);
        if (!ok) cell.e = -1;
        sncc_load<DT>(a.st, cell, raw[g]);
        const int q = ig * R + j;
        const bool inq = ok && fvr_checked(q, static_cast<long long>(R) * R, kSiteSnccTarget);
        Ts[g] = inq ? __ldg(ft + q) : make_float2(0.f, 0.f);
        hs[g] = inq ? (a.hp ? __ldg(a.hp + q) : 1.f) : 0.f;
      }
#pragma unroll
      for (int g = 0; g < GROUP; ++g) {
        const int ig = i + g * rpp;
        const int rn = R + (ig < row_end ? ig : row_begin) - row_begin;
        const float4 fa = tab.frac[rn];
        float tx = fa.x + fb.x, ty = fa.y + fb.y, tz = fa.z + fb.z;
        if (tx >= 1.f) tx -= 1.f;
        if (ty >= 1.f) ty -= 1.f;
        if (tz >= 1.f) tz -= 1.f;
        // f16: the brick scale rides on the high-pass weight (every moment is
        // linear in h S or quadratic in it) instead of rescaling 8 values
        const float h = (DT == FVR_F16 || DT == FVR_F16_PAIR) ? hs[g] * raw_scale(raw[g]) : hs[g];
        sncc_accumulate<DT, GRAD, NM>(raw[g], tx, ty, tz, tab.kph[rn], kb, Ts[g], h, acc);
      }
    }
  }
}

// Pair accumulators -> CTA moment sums (fp64 across warps), written to record rec.
template <int NM>
__device__ __forceinline__ void sncc_store_record(const float2 (&acc)[NM], double* red, double* partial,
                                                  int64_t rec) {
  float m[NM];
#pragma unroll
  for (int k = 0; k < NM; ++k) m[k] = (k == M_PHU || k == M_PHV) ? acc[k].y - acc[k].x : acc[k].x + acc[k].y;
  double tot;
  block_reduce_d<NM, float>(m, red, &tot);
  if (threadIdx.x < NM) partial[rec * NM + threadIdx.x] = tot;
}

// Tile grid: CTA (tile, c, v) reduces rows [tile * a.tile_rows, ...) of
// (candidate c, view v) into one partial record.
template <int DT, bool GRAD, int GROUP, int MINB>
__global__ void __launch_bounds__(kSnccThreads, MINB) tc_sncc_moments_kernel(SnccArgs a) {
  constexpr int NM = GRAD ? M_NGRAD : 3;
  __shared__ double red[NM * (kSnccThreads / 32)];
  __shared__ double ax_s[8];
  extern __shared__ __align__(16) unsigned char tab_smem[];
  const int tile = blockIdx.x, c = blockIdx.y, v = blockIdx.z;
  const int R = a.R;
  const int row_begin = tile * a.tile_rows;
  const int row_end = min(row_begin + a.tile_rows, R);
  const SnccTab tab = sncc_tab(tab_smem, R + a.tile_rows);
  pdl_launch_dependents();
  pdl_wait();  // launched as a programmatic dependent: the kernel before it has completed (else a no-op)
  if (threadIdx.x == 0) sncc_item_axes(a, v, c, ax_s);
  __syncthreads();
  build_sncc_tables(tab, R, row_begin, row_end - row_begin, a.lin, ax_s, a.sx, a.sy, a.sz, a.kpi);
  __syncthreads();
  float2 acc[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m) acc[m] = make_float2(0.f, 0.f);
  sncc_run<DT, GRAD, GROUP, NM>(a, tab, view_target(a, v), row_begin, row_end, acc);
  sncc_store_record<NM>(acc, red, a.partial, (static_cast<int64_t>(v) * a.C + c) * gridDim.x + tile);
}

// Value-and-gradient epilogue, launched right after the moments kernel as its
// programmatic dependent (one CTA of 512 threads).  The work goes in chunks
// of candidates whose (view, candidate) items fit in shared memory:
//  0. the slice-axes Jacobians of the first chunk's items, formed while the
//     moments kernel still runs (later chunks: before their record sums);
//  1. after griddepcontrol.wait, one thread per (item, moment): the item's
//     records summed in record order, every load of a thread issued in one
//     round, kept in shared memory;
//  2. one thread per item: its ncc and its per-view part of the pose gradient
//     (per axis gc (a A + 2 b B) through the Jacobian, translations from the
//     phase moments);
//  3. one thread per candidate: the views summed in order; the ncc sums for
//     the losses accumulate per thread across chunks and are reduced in a
//     fixed order at the end.
constexpr int kFinalThreads = 512;
constexpr int kFinalChunkItems = 128;  // 128 items x 44 doubles = 44 KB of shared memory
constexpr int kFinalPairs = (kFinalChunkItems * M_NGRAD + kFinalThreads - 1) / kFinalThreads;  // per thread
constexpr int kFinalRecords = 4;  // records per (item, moment) per load round

__global__ void __launch_bounds__(kFinalThreads) tc_sncc_final_kernel(SnccArgs a) {
  __shared__ double s_mom[kFinalChunkItems][M_NGRAD];
  __shared__ double s_jac[kFinalChunkItems][18];
  __shared__ double s_part[kFinalChunkItems][6];  // ga[3], gtx, gty, ncc
  __shared__ double red[kMaxViews][kFinalThreads / 32];
  const int t = threadIdx.x, nv = a.nv, C = a.C, tiles = a.tiles;
  const double s3[3] = {a.sx, a.sy, a.sz};
  double lsum[kMaxViews] = {0.0, 0.0, 0.0, 0.0};
  const int cch = kFinalChunkItems / nv;  // candidates per chunk; chunk item li = v * cn + (c - c0)
  for (int c0 = 0; c0 < C; c0 += cch) {
    const int cn = min(cch, C - c0), ni = cn * nv;
    if (c0 > 0) __syncthreads();  // the previous chunk is done with the shared arrays
    if (t < ni) {
      const int v = t / cn, c = c0 + (t - v * cn);
      double ax[8];
      slice_axes_jac(a.poses + 6 * c, view_lateral(a, v), a.sx, a.sy, a.sz, ax, s_jac[t]);
    }
    if (c0 == 0) pdl_wait();  // the moments kernel has completed and its records are visible
    // record sums: the thread's pairs p = t + k * 512, all their loads in one round
    const double* src[kFinalPairs];
#pragma unroll
    for (int k = 0; k < kFinalPairs; ++k) {
      const int p = t + k * kFinalThreads;
      src[k] = nullptr;
      if (p < ni * M_NGRAD) {
        const int li = p / M_NGRAD, m = p - li * M_NGRAD, v = li / cn;
        const int64_t it = static_cast<int64_t>(v) * C + c0 + (li - v * cn);
        src[k] = a.partial + it * tiles * M_NGRAD + m;
      }
    }
    double sum[kFinalPairs];
#pragma unroll
    for (int k = 0; k < kFinalPairs; ++k) sum[k] = 0.0;
    for (int r0 = 0; r0 < tiles; r0 += kFinalRecords) {
      double x[kFinalPairs][kFinalRecords];
#pragma unroll
      for (int k = 0; k < kFinalPairs; ++k)
#pragma unroll
        for (int r = 0; r < kFinalRecords; ++r)
          x[k][r] = src[k] && r0 + r < tiles ? __ldcg(src[k] + static_cast<int64_t>(r0 + r) * M_NGRAD) : 0.0;
#pragma unroll
      for (int k = 0; k < kFinalPairs; ++k)
#pragma unroll
        for (int r = 0; r < kFinalRecords; ++r) sum[k] += x[k][r];
    }
#pragma unroll
    for (int k = 0; k < kFinalPairs; ++k) {
      const int p = t + k * kFinalThreads;
      if (p < ni * M_NGRAD) {
        const int li = p / M_NGRAD, m = p - li * M_NGRAD, v = li / cn;
        s_mom[li][m] = sum[k];
        // the moment record (consecutive threads, consecutive doubles)
        a.mom[(static_cast<int64_t>(v) * C + c0 + (li - v * cn)) * kMomStride + m] = sum[k];
      }
    }
    __syncthreads();
    if (t < ni) {
      const int li = t, v = li / cn, c = c0 + (li - v * cn);
      const int64_t it = static_cast<int64_t>(v) * C + c;
      const double* m = s_mom[li];
      const double* j = s_jac[li];
      const double sq = sqrt(m[M_EP] * m[M_ET]);
      const double inv = 1.0 / (sq + 1e-8);
      const double ncc = m[M_CROSS] * inv;
      const double bb = sq > 0.0 ? -0.5 * m[M_CROSS] * m[M_ET] * inv * inv / sq : 0.0;
      const double gc = -(a.g ? static_cast<double>(a.g[v * a.g_stride]) : 1.0) / C;
      double ga[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double du = gc * (inv * m[M_AU + i] + 2.0 * bb * m[M_BU + i]) * s3[i];
        const double dv = gc * (inv * m[M_AV + i] + 2.0 * bb * m[M_BV + i]) * s3[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) ga[k] += du * j[(k * 2 + 0) * 3 + i] + dv * j[(k * 2 + 1) * 3 + i];
      }
      double* o = s_part[li];
      o[0] = ga[0];
      o[1] = ga[1];
      o[2] = ga[2];
      o[3] = gc * inv * a.kappa * m[M_PHU];
      o[4] = gc * inv * a.kappa * m[M_PHV];
      o[5] = ncc;
      a.mom[it * kMomStride + 17] = ncc;
      if (a.ncc_out) a.ncc_out[it] = static_cast<float>(ncc);
    }
    __syncthreads();
    if (t < cn) {
      const int c = c0 + t;
      double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int v = 0; v < nv; ++v) {
        const double* o = s_part[v * cn + t];
#pragma unroll
        for (int k = 0; k < 5; ++k) r[k] += o[k];
        if (v == 0) lsum[0] += o[5];
        else if (v == 1) lsum[1] += o[5];
        else if (v == 2) lsum[2] += o[5];
        else lsum[3] += o[5];
      }
      float* g = a.grad + 6 * c;
      const float rf[6] = {static_cast<float>(r[0]), static_cast<float>(r[1]), static_cast<float>(r[2]),
                           static_cast<float>(r[3]), static_cast<float>(r[4]), 0.f};
      for (int k = 0; k < 6; ++k) g[k] = a.accumulate ? g[k] + rf[k] : rf[k];
    }
  }
  // loss[v] = 1 - mean_c ncc (fixed order: per thread, per warp, across warps)
  const int lane = t & 31, w = t >> 5;
#pragma unroll
  for (int v = 0; v < kMaxViews; ++v) {
    const double sv = warp_sum(lsum[v]);
    if (lane == 0) red[v][w] = sv;
  }
  __syncthreads();
  if (t == 0) {
    double total = 0.0;
    for (int v = 0; v < nv; ++v) {
      double sv = 0.0;
      for (int k = 0; k < kFinalThreads / 32; ++k) sv += red[v][k];
      const double l = 1.0 - sv / C;
      a.loss[v] = static_cast<float>(l);
      total += l;
    }
    a.loss[nv] = static_cast<float>(total);
  }
}

// Launch the epilogue as a programmatic dependent of the kernel before it on
// the stream (plain launch where the attribute is refused).
static void launch_sncc_final(cudaStream_t s, const SnccArgs& a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(kFinalThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, tc_sncc_final_kernel, a) != cudaSuccess) {
    (void)cudaGetLastError();
    tc_sncc_final_kernel<<<1, kFinalThreads, 0, s>>>(a);
  }
}

// Record sums (fp64, fixed order) -> mom[v][c][0..NM), ncc in mom[v][c][17];
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

// pair_ok: the caller's kernels also read the x-pair storage (the moments kernels).
static int stencil_from(int dtype, const void* data, const float* scales, int64_t D, int64_t H, int64_t W,
                        Stencil* s, bool pair_ok = false) {
  if (!data || D < 1 || H < 1 || W < 1 || D > 8192 || H > 8192 || W > 8192) return FVR_ERR_ARG;
  if (dtype != FVR_F32 && dtype != FVR_BF16 && dtype != FVR_F16 &&
      !(pair_ok && (dtype == FVR_BF16_PAIR || dtype == FVR_F16_PAIR || dtype == FVR_F32_PAIR)))
    return FVR_ERR_DTYPE;
  if ((dtype == FVR_F16 || dtype == FVR_F16_PAIR) && !scales) return FVR_ERR_ARG;
  if (dtype == FVR_F32_PAIR && (reinterpret_cast<uintptr_t>(data) & 31) != 0) return FVR_ERR_ARG;  // 256-bit loads
  if ((reinterpret_cast<uintptr_t>(data) & 15) != 0) return FVR_ERR_ARG;
  *s = Stencil{data, scales, static_cast<int>(D), static_cast<int>(H), static_cast<int>(W), dtype};
  return FVR_OK;
}

static double half_extent(int64_t n) { return 0.5 * static_cast<double>(n > 1 ? n - 1 : 1); }

static int device_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    sms = (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0) ? n : 148;
  }
  return sms;
}

// Grid and tables of one moments launch: one wave of min_blocks resident
// CTAs per SM split over the (candidate, view) items in whole slice rows
// (never more CTAs than slots), at least 256 samples per CTA.
struct SnccPlan {
  dim3 grid;
  int tile_rows, tiles;
};

static SnccPlan sncc_plan(int64_t C, int64_t R, int nv, int variant) {
  const SnccVariant v = sncc_variant(variant);
  const int64_t items = C * nv, min_rows = cdiv64(kSnccThreads, R);
  int64_t tiles = (static_cast<int64_t>(v.min_blocks) * device_sms()) / items;
  tiles = std::max<int64_t>(1, std::min(tiles, R / min_rows));
  const int64_t tile_rows = cdiv64(R, tiles);
  tiles = cdiv64(R, tile_rows);
  SnccPlan p{};
  p.grid = dim3(static_cast<unsigned>(tiles), static_cast<unsigned>(C), static_cast<unsigned>(nv));
  p.tile_rows = static_cast<int>(tile_rows);
  p.tiles = static_cast<int>(tiles);
  return p;
}

// Dynamic shared memory: the tables (R columns + tile rows).
static int64_t sncc_smem(int64_t R, int tile_rows) { return (R + tile_rows) * kSnccTabEntryBytes; }
constexpr int64_t kSnccMaxSmem = 200 * 1024;

// pdl: launch as a programmatic dependent of the kernel before it on the
// stream (the moments kernel waits for that kernel's completion before its
// first read, so only the launch overlaps it); plain launch where refused.
template <int DT, bool GRAD, int VI>
static void launch_sncc_v(dim3 grid, int smem, cudaStream_t st, const SnccArgs& a, bool pdl) {
  constexpr SnccVariant v = sncc_variant(VI);
  auto k = tc_sncc_moments_kernel<DT, GRAD, v.group, v.min_blocks>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (pdl) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kSnccThreads);
    cfg.dynamicSmemBytes = static_cast<size_t>(smem);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k, a) == cudaSuccess) return;
    (void)cudaGetLastError();
  }
  k<<<grid, kSnccThreads, smem, st>>>(a);
}

template <int DT, bool GRAD>
static void launch_sncc(int variant, dim3 grid, int smem, cudaStream_t s, const SnccArgs& a, bool pdl = false) {
  switch (variant) {
#define FVR_V(n) \
  case n: launch_sncc_v<DT, GRAD, n>(grid, smem, s, a, pdl); break;
    FVR_V(0) FVR_V(1) FVR_V(2) FVR_V(3) FVR_V(4) FVR_V(5) FVR_V(6) FVR_V(7)
#undef FVR_V
    default: break;
  }
}
static_assert(kSnccVariants == 8, "launch_sncc lists every variant");

// Shared argument set-up of the moments launches.
static int sncc_setup(int dtype, const void* stencil, const float* scales, int64_t D, int64_t H, int64_t W,
                      const float* poses, int64_t C, int nviews, const int* views, const void* const* ftargs,
                      const float* hp, const float* lin, int64_t R, double kappa, int variant, SnccArgs* a,
                      dim3* grid, int64_t* smem) {
  Stencil st;
  int rc = stencil_from(dtype, stencil, scales, D, H, W, &st, true);
  if (rc) return rc;
  if (!poses || !views || !ftargs || !lin || C < 1 || R < 1 || C > 65535) return FVR_ERR_ARG;
  if (nviews < 1 || nviews > kMaxViews || R * R > (int64_t)1 << 30) return FVR_ERR_ARG;
  if (variant < 0 || variant >= kSnccVariants) return FVR_ERR_ARG;
  if ((D + 1) * (H + 1) * (W + 1) > INT32_MAX) return FVR_ERR_UNSUPPORTED;  // 32-bit entry index
  const SnccPlan plan = sncc_plan(C, R, nviews, variant);
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
  a->nv = nviews;
  a->tile_rows = plan.tile_rows;
  a->tiles = plan.tiles;
  *smem = sncc_smem(R, plan.tile_rows);
  if (*smem > kSnccMaxSmem) return FVR_ERR_UNSUPPORTED;
  a->kpi = kappa / 3.14159265358979323846;
  a->kappa = kappa;
  a->sx = half_extent(W);
  a->sy = half_extent(H);
  a->sz = half_extent(D);
  *grid = plan.grid;
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
// Size (about 352 KB per device): kStaticRecords partial-moment records of
// 17 doubles and kStaticItems (candidate, view) moment records of 18
// doubles.  Calls needing more -- more than 512 (candidate, view) pairs, or
// more than 2048 partial records (pairs x tiles, as the launch variant sizes
// the tiles) -- are refused with FVR_ERR_WORKSPACE before anything is
// launched.
//
// Start state: none.  The partial and moment records are written by every
// call before they are read.
//
// Set-up: the first call on each device, made with that device current,
// resolves the array's device address with cudaGetSymbolAddress and caches
// it; make that first call before any stream capture begins.  The cached
// address belongs to the device's primary context of that moment: a process
// that calls cudaDeviceReset (or otherwise destroys that context) while the
// library is loaded must not call this entry point on that device again,
// since the module is loaded anew into the next context and the cached
// address no longer names the array.
//
// Record bound: sncc_plan gives each (candidate, view) item
// max(1, floor(min_blocks * SMs / items)) tiles, so one call needs at most
// max(items, min_blocks * SMs) partial records; with items <= 512 and the
// largest min_blocks of the variant table on a 148-SM B200 that stays within
// kStaticRecords (static_assert below; the run-time check refuses anything
// else before launching).
//
// Races: one array per device is shared by every caller in the process.
// Calls on the same device must be ordered (one stream, or explicit
// synchronisation); two calls that overlap in time corrupt each other's
// scratch.
// ----------------------------------------------------------------------------
constexpr int64_t kStaticItems = 512;
constexpr int64_t kStaticRecords = 2048;
constexpr int64_t kStaticPartialDoubles = kStaticRecords * M_NGRAD;
constexpr int64_t kStaticMomDoubles = kStaticItems * kMomStride;
constexpr int64_t kStaticDoubles = kStaticPartialDoubles + kStaticMomDoubles;
constexpr int kStaticMaxDevices = 64;

static __device__ __align__(256) double g_sncc_static_scratch[kStaticDoubles];

constexpr int max_min_blocks() {
  int m = 0;
  for (const SnccVariant& v : kSnccVariantTable) m = v.min_blocks > m ? v.min_blocks : m;
  return m;
}
static_assert(kStaticItems <= kStaticRecords && max_min_blocks() * 148 <= kStaticRecords,
              "static scratch holds the partial records of every launch variant on a 148-SM device");

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

// Partial records: at most ceil(K / 256) tiles per (candidate, view).
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
    case FVR_BF16_PAIR: FVR_SNCC(FVR_BF16_PAIR)
    case FVR_F16_PAIR: FVR_SNCC(FVR_F16_PAIR)
    case FVR_F32_PAIR: FVR_SNCC(FVR_F32_PAIR)
  }
#undef FVR_SNCC
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

// Fused workspace: partial records | moments [nv][C][18]; both written by a
// call before they are read.
int64_t fvr_tc_sncc_fused_workspace(int64_t C, int64_t R, int64_t nviews) {
  if (C < 1 || R < 1 || nviews < 1) return 0;
  return fvr_tc_sncc_workspace(C, R, nviews) + nviews * C * kMomStride * (int64_t)sizeof(double);
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
  a.mom = reinterpret_cast<double*>(ws + fvr_tc_sncc_workspace(C, R, nviews));
  a.loss = loss;
  a.ncc_out = ncc_out;
  a.grad = grad_poses;
  a.g = g;
  a.g_stride = (int)g_stride;
  a.accumulate = accumulate;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FVR_F32: launch_sncc<FVR_F32, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_BF16: launch_sncc<FVR_BF16, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F16: launch_sncc<FVR_F16, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_BF16_PAIR: launch_sncc<FVR_BF16_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F16_PAIR: launch_sncc<FVR_F16_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F32_PAIR: launch_sncc<FVR_F32_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
  }
  FVR_LAUNCH_CHECK();
  launch_sncc_final(s, a);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_tc_sncc_finalize(const void* workspace, int64_t C, int64_t R, int nviews, int with_grad, int variant,
                         double* mom, float* loss, float* ncc_out, void* stream) {
  if (!workspace || !mom || !loss || C < 1 || R < 1 || nviews < 1 || nviews > kMaxViews) return FVR_ERR_ARG;
  if (variant < 0 || variant >= kSnccVariants) return FVR_ERR_ARG;
  const SnccPlan plan = sncc_plan(C, R, nviews, variant);
  tc_sncc_finalize_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const double*>(workspace), (int)C, nviews, plan.tiles, with_grad ? M_NGRAD : 3, mom, loss, ncc_out);
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
  if (items > kStaticItems || items * a.tiles > kStaticRecords) return FVR_ERR_WORKSPACE;
  double* scratch = nullptr;
  rc = static_scratch(&scratch);
  if (rc) return rc;
  a.partial = scratch;
  a.mom = scratch + kStaticPartialDoubles;
  a.loss = loss;
  a.ncc_out = ncc_out;
  a.grad = grad_poses;
  a.g = g;
  a.g_stride = (int)g_stride;
  a.accumulate = accumulate;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case FVR_F32: launch_sncc<FVR_F32, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_BF16: launch_sncc<FVR_BF16, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F16: launch_sncc<FVR_F16, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_BF16_PAIR: launch_sncc<FVR_BF16_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F16_PAIR: launch_sncc<FVR_F16_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
    case FVR_F32_PAIR: launch_sncc<FVR_F32_PAIR, true>(variant, grid, (int)smem, s, a, true); break;
  }
  FVR_LAUNCH_CHECK();
  launch_sncc_final(s, a);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"

FVR_CHECK_ACCESSOR(check_word_tc)
