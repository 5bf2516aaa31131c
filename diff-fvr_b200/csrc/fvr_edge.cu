// Edge-dominant gradient NCC (src/fvr/cone_beam_fvr.py:71-112), sm_100a.
//
// For each image pair (pred a, target b) and channel: Sobel x / y responses
// (zero padding) on the interior [crop, H-crop) x [crop, W-crop), their NCC
// per direction, averaged; optionally the same on 3x3 box-blurred images
// (zero padding, divisor 9) weighted by w.  Everything is expressed through
// five moments per (direction, scale) -- S_u, S_v, S_uu, S_vv, S_uv -- so the
// forward pass is one tiled stencil + reduction and the adjoint is one tiled
// stencil that applies the transposed Sobel and box filters in shared memory.
#include "fvr_common.cuh"

namespace fvr {

constexpr int kEdgeTile = 32;      // output tile edge
constexpr int kEdgeThreads = 256;  // 8 rows of 32
constexpr int kEdgeMom = 5;        // S_u, S_v, S_uu, S_vv, S_uv
constexpr int kEdgeCombos = 4;     // fine x, fine y, coarse x, coarse y

struct EdgeArgs {
  const float* a;  // [B][C][H][W]
  const float* b;  // [Bt][C][H][W], Bt = 1 (broadcast) or B
  int B, Bt, Cch, H, W, crop;
  int coarse;       // 1: blurred scale enabled
  int tiles_x, tiles_y;
};

// Sobel responses at smem position (i, j) of a tile `t` with row pitch p:
// gx = sum kx * t, kx = [-1 0 1; -2 0 2; -1 0 1]; gy with ky = kx^T.
__device__ __forceinline__ void sobel(const float* t, int p, int i, int j, float& gx, float& gy) {
  const float* r0 = t + (i - 1) * p + j;
  const float* r1 = t + i * p + j;
  const float* r2 = t + (i + 1) * p + j;
  gx = (r0[1] - r0[-1]) + 2.f * (r1[1] - r1[-1]) + (r2[1] - r2[-1]);
  gy = (r2[-1] + 2.f * r2[0] + r2[1]) - (r0[-1] + 2.f * r0[0] + r0[1]);
}

// Zero-padded image window [r0, r0+n) x [c0, c0+n) into smem (pitch n).
__device__ __forceinline__ void load_window(const float* img, int H, int W, int r0, int c0, int n, float* s) {
  for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
    const int i = k / n, j = k - i * n;
    const int r = r0 + i, c = c0 + j;
    s[k] = (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(img + static_cast<int64_t>(r) * W + c) : 0.f;
  }
}

// Box-blurred window (pitch n) from a zero-padded window (pitch n + 2) one
// pixel wider on each side; blurred pixels outside the image are zero.
__device__ __forceinline__ void blur_window(const float* src, int H, int W, int r0, int c0, int n, float* dst) {
  const int p = n + 2;
  for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
    const int i = k / n, j = k - i * n;
    const int r = r0 + i, c = c0 + j;
    float v = 0.f;
    if (r >= 0 && r < H && c >= 0 && c < W) {
      const float* q = src + i * p + j;
      v = (q[0] + q[1] + q[2] + q[p] + q[p + 1] + q[p + 2] + q[2 * p] + q[2 * p + 1] + q[2 * p + 2]) * (1.f / 9.f);
    }
    dst[k] = v;
  }
}

// Moments of one 32 x 32 tile of the interior -> partial[pair][tile][20] (fp64).
__global__ void __launch_bounds__(kEdgeThreads) edge_moments_kernel(EdgeArgs a, double* __restrict__ partial) {
  constexpr int T = kEdgeTile;
  constexpr int NA = T + 4, NB = T + 2;
  __shared__ float sa[NA * NA], sb[NA * NA], ba[NB * NB], bb[NB * NB];
  __shared__ double red[kEdgeCombos * kEdgeMom * (kEdgeThreads / 32)];
  const int pair = blockIdx.z;
  const int bi = pair / a.Cch, ch = pair - bi * a.Cch;
  const int bt = a.Bt == 1 ? 0 : bi;
  const int64_t plane = static_cast<int64_t>(a.H) * a.W;
  const float* img_a = a.a + (static_cast<int64_t>(bi) * a.Cch + ch) * plane;
  const float* img_b = a.b + (static_cast<int64_t>(bt) * a.Cch + ch) * plane;
  const int r0 = a.crop + blockIdx.y * T, c0 = a.crop + blockIdx.x * T;
  const int r_end = a.H - a.crop, c_end = a.W - a.crop;
  load_window(img_a, a.H, a.W, r0 - 2, c0 - 2, NA, sa);
  load_window(img_b, a.H, a.W, r0 - 2, c0 - 2, NA, sb);
  __syncthreads();
  if (a.coarse) {
    blur_window(sa, a.H, a.W, r0 - 1, c0 - 1, NB, ba);
    blur_window(sb, a.H, a.W, r0 - 1, c0 - 1, NB, bb);
    __syncthreads();
  }
  float acc[kEdgeCombos * kEdgeMom];
#pragma unroll
  for (int m = 0; m < kEdgeCombos * kEdgeMom; ++m) acc[m] = 0.f;
  const int tj = threadIdx.x & 31;
  for (int ti = threadIdx.x >> 5; ti < T; ti += kEdgeThreads / 32) {
    const int r = r0 + ti, c = c0 + tj;
    if (r >= r_end || c >= c_end) continue;
    float u[4], v[4];
    sobel(sa, NA, ti + 2, tj + 2, u[0], u[1]);
    sobel(sb, NA, ti + 2, tj + 2, v[0], v[1]);
    if (a.coarse) {
      sobel(ba, NB, ti + 1, tj + 1, u[2], u[3]);
      sobel(bb, NB, ti + 1, tj + 1, v[2], v[3]);
    } else {
      u[2] = u[3] = v[2] = v[3] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < kEdgeCombos; ++k) {
      float* m = acc + k * kEdgeMom;
      m[0] += u[k];
      m[1] += v[k];
      m[2] = fmaf(u[k], u[k], m[2]);
      m[3] = fmaf(v[k], v[k], m[3]);
      m[4] = fmaf(u[k], v[k], m[4]);
    }
  }
  // fp64 cross-lane / cross-warp sums
  constexpr int NM = kEdgeCombos * kEdgeMom;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = kEdgeThreads / 32;
#pragma unroll
  for (int m = 0; m < NM; ++m) {
    const double s = warp_sum(static_cast<double>(acc[m]));
    if (lane == 0) red[m * nw + wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < NM) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[threadIdx.x * nw + w];
    const int tile = blockIdx.y * a.tiles_x + blockIdx.x;
    partial[(static_cast<int64_t>(pair) * a.tiles_x * a.tiles_y + tile) * NM + threadIdx.x] = s;
  }
}

// Per pair: tile sums -> stats[pair][20]; per batch item: the loss value
// (1 - w) * mean_c 0.5 (ncc_fx + ncc_fy) + w * (coarse), then the batch mean.
__device__ __forceinline__ double edge_ncc(const double* m, double n) {
  const double suu = m[2] - m[0] * m[0] / n, svv = m[3] - m[1] * m[1] / n, suv = m[4] - m[0] * m[1] / n;
  return suv / sqrt(fmax(suu * svv, 1e-12));
}

__global__ void edge_finalize_kernel(EdgeArgs a, const double* __restrict__ partial, float w,
                                     double* __restrict__ stats, float* __restrict__ out, int reduction_mean) {
  constexpr int NM = kEdgeCombos * kEdgeMom;
  const int tiles = a.tiles_x * a.tiles_y;
  const int npair = a.B * a.Cch;
  for (int k = threadIdx.x; k < npair * NM; k += blockDim.x) {
    const int pair = k / NM, m = k - pair * NM;
    double s = 0.0;
    for (int t = 0; t < tiles; ++t) s += partial[(static_cast<int64_t>(pair) * tiles + t) * NM + m];
    stats[k] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double n = static_cast<double>(a.H - 2 * a.crop) * static_cast<double>(a.W - 2 * a.crop);
  double total = 0.0;
  for (int bi = 0; bi < a.B; ++bi) {
    double fine = 0.0, coarse = 0.0;
    for (int ch = 0; ch < a.Cch; ++ch) {
      const double* st = stats + static_cast<int64_t>(bi * a.Cch + ch) * NM;
      fine += 0.5 * (edge_ncc(st, n) + edge_ncc(st + kEdgeMom, n));
      if (a.coarse) coarse += 0.5 * (edge_ncc(st + 2 * kEdgeMom, n) + edge_ncc(st + 3 * kEdgeMom, n));
    }
    fine /= a.Cch;
    coarse /= a.Cch;
    const double val = a.coarse ? (1.0 - w) * fine + w * coarse : fine;
    if (!reduction_mean) out[bi] = static_cast<float>(val);
    total += val;
  }
  if (reduction_mean) out[0] = static_cast<float>(total / a.B);
}

// d value / d pred (or d target with wrt_b) for one 32 x 32 output tile of the
// full image.  Interior gradient fields g_k(q) = alpha_k (v_k(q) - mean v_k)
// + beta_k (u_k(q) - mean u_k) on the interior, transposed Sobel, and for the
// blurred scale the transposed box filter.
__global__ void __launch_bounds__(kEdgeThreads) edge_grad_kernel(EdgeArgs a, const double* __restrict__ stats,
                                                                 float w, const float* __restrict__ g, int g_stride,
                                                                 int reduction_mean, int wrt_b,
                                                                 float* __restrict__ grad) {
  constexpr int T = kEdgeTile;
  constexpr int N4 = T + 8, N3 = T + 6, N2 = T + 4, N1 = T + 2;
  extern __shared__ float smem[];
  float* sa = smem;            // N4^2 : this image (differentiated), halo 4
  float* sb = sa + N4 * N4;    // N4^2 : the other image
  float* ba = sb + N4 * N4;    // N3^2 : blurred, halo 3
  float* bb = ba + N3 * N3;    // N3^2
  float* gfx = bb + N3 * N3;   // N1^2 : fine-scale fields, halo 1
  float* gfy = gfx + N1 * N1;  // N1^2
  float* gcx = gfy + N1 * N1;  // N2^2 : coarse-scale fields, halo 2
  float* gcy = gcx + N2 * N2;  // N2^2
  float* gbl = gcy + N2 * N2;  // N1^2 : gradient w.r.t. the blurred image, halo 1
  __shared__ float coef[kEdgeCombos][4];  // alpha, beta, mean u, mean v
  const int pair = blockIdx.z;
  const int bi = pair / a.Cch, ch = pair - bi * a.Cch;
  const int bt = a.Bt == 1 ? 0 : bi;
  const int64_t plane = static_cast<int64_t>(a.H) * a.W;
  const float* img_a = a.a + (static_cast<int64_t>(bi) * a.Cch + ch) * plane;
  const float* img_b = a.b + (static_cast<int64_t>(bt) * a.Cch + ch) * plane;
  if (wrt_b) {
    const float* t = img_a;
    img_a = img_b;
    img_b = t;
  }
  const int r0 = blockIdx.y * T, c0 = blockIdx.x * T;
  if (threadIdx.x < kEdgeCombos) {
    const int k = threadIdx.x;
    const double* m = stats + static_cast<int64_t>(pair) * kEdgeCombos * kEdgeMom + k * kEdgeMom;
    // u = the differentiated image's response, v = the other one's
    const double su = wrt_b ? m[1] : m[0], sv = wrt_b ? m[0] : m[1];
    const double suu_raw = wrt_b ? m[3] : m[2], svv_raw = wrt_b ? m[2] : m[3];
    const double n = static_cast<double>(a.H - 2 * a.crop) * static_cast<double>(a.W - 2 * a.crop);
    const double suu = suu_raw - su * su / n, svv = svv_raw - sv * sv / n, suv = m[4] - m[0] * m[1] / n;
    const double prod = suu * svv;
    const double den = sqrt(fmax(prod, 1e-12));
    const double gv = static_cast<double>(g[g_stride * bi]) * (reduction_mean ? 1.0 / a.B : 1.0);
    const double sw = k < 2 ? (a.coarse ? 1.0 - w : 1.0) : (a.coarse ? w : 0.0);
    const double wk = gv * sw * 0.5 / a.Cch;
    coef[k][0] = static_cast<float>(wk / den);
    coef[k][1] = prod > 1e-12 ? static_cast<float>(-wk * suv * svv / (den * den * den)) : 0.f;
    coef[k][2] = static_cast<float>(su / n);
    coef[k][3] = static_cast<float>(sv / n);
  }
  load_window(img_a, a.H, a.W, r0 - 4, c0 - 4, N4, sa);
  load_window(img_b, a.H, a.W, r0 - 4, c0 - 4, N4, sb);
  __syncthreads();
  if (a.coarse) {
    blur_window(sa, a.H, a.W, r0 - 3, c0 - 3, N3, ba);
    blur_window(sb, a.H, a.W, r0 - 3, c0 - 3, N3, bb);
  }
  const int ilo = a.crop, ihi = a.H - a.crop, jlo = a.crop, jhi = a.W - a.crop;
  // fine fields at halo 1 (window origin r0 - 1)
  for (int k = threadIdx.x; k < N1 * N1; k += blockDim.x) {
    const int i = k / N1, j = k - i * N1;
    const int r = r0 - 1 + i, c = c0 - 1 + j;
    float fx = 0.f, fy = 0.f;
    if (r >= ilo && r < ihi && c >= jlo && c < jhi) {
      float ux, uy, vx, vy;
      sobel(sa, N4, i + 3, j + 3, ux, uy);
      sobel(sb, N4, i + 3, j + 3, vx, vy);
      fx = coef[0][0] * (vx - coef[0][3]) + coef[0][1] * (ux - coef[0][2]);
      fy = coef[1][0] * (vy - coef[1][3]) + coef[1][1] * (uy - coef[1][2]);
    }
    gfx[k] = fx;
    gfy[k] = fy;
  }
  __syncthreads();
  if (a.coarse) {
    // coarse fields at halo 2 (window origin r0 - 2)
    for (int k = threadIdx.x; k < N2 * N2; k += blockDim.x) {
      const int i = k / N2, j = k - i * N2;
      const int r = r0 - 2 + i, c = c0 - 2 + j;
      float fx = 0.f, fy = 0.f;
      if (r >= ilo && r < ihi && c >= jlo && c < jhi) {
        float ux, uy, vx, vy;
        sobel(ba, N3, i + 1, j + 1, ux, uy);
        sobel(bb, N3, i + 1, j + 1, vx, vy);
        fx = coef[2][0] * (vx - coef[2][3]) + coef[2][1] * (ux - coef[2][2]);
        fy = coef[3][0] * (vy - coef[3][3]) + coef[3][1] * (uy - coef[3][2]);
      }
      gcx[k] = fx;
      gcy[k] = fy;
    }
    __syncthreads();
    // gradient w.r.t. the blurred image at halo 1: transposed Sobel, in-image only
    for (int k = threadIdx.x; k < N1 * N1; k += blockDim.x) {
      const int i = k / N1, j = k - i * N1;
      const int r = r0 - 1 + i, c = c0 - 1 + j;
      float s = 0.f;
      if (r >= 0 && r < a.H && c >= 0 && c < a.W) {
        const float* px = gcx + (i + 1) * N2 + (j + 1);
        const float* py = gcy + (i + 1) * N2 + (j + 1);
        // sum_d g(m - d) k[d]: kx[d] = dj (1 + (di == 0)), ky[d] = di (1 + (dj == 0))
        s = (px[N2 - 1] - px[N2 + 1]) + 2.f * (px[-1] - px[1]) + (px[-N2 - 1] - px[-N2 + 1]);
        s += (py[-N2 - 1] + 2.f * py[-N2] + py[-N2 + 1]) - (py[N2 - 1] + 2.f * py[N2] + py[N2 + 1]);
      }
      gbl[k] = s;
    }
    __syncthreads();
  }
  const int tj = threadIdx.x & 31;
  const int64_t out_base = (static_cast<int64_t>(bi) * a.Cch + ch) * plane;
  for (int ti = threadIdx.x >> 5; ti < T; ti += kEdgeThreads / 32) {
    const int r = r0 + ti, c = c0 + tj;
    if (r >= a.H || c >= a.W) continue;
    const float* px = gfx + (ti + 1) * N1 + (tj + 1);
    const float* py = gfy + (ti + 1) * N1 + (tj + 1);
    float s = (px[N1 - 1] - px[N1 + 1]) + 2.f * (px[-1] - px[1]) + (px[-N1 - 1] - px[-N1 + 1]);
    s += (py[-N1 - 1] + 2.f * py[-N1] + py[-N1 + 1]) - (py[N1 - 1] + 2.f * py[N1] + py[N1 + 1]);
    if (a.coarse) {
      const float* q = gbl + (ti + 1) * N1 + (tj + 1);
      s += (q[-N1 - 1] + q[-N1] + q[-N1 + 1] + q[-1] + q[0] + q[1] + q[N1 - 1] + q[N1] + q[N1 + 1]) * (1.f / 9.f);
    }
    grad[out_base + static_cast<int64_t>(r) * a.W + c] = s;
  }
}

constexpr int64_t kEdgeGradSmem =
    (2 * (kEdgeTile + 8) * (kEdgeTile + 8) + 2 * (kEdgeTile + 6) * (kEdgeTile + 6) +
     3 * (kEdgeTile + 2) * (kEdgeTile + 2) + 2 * (kEdgeTile + 4) * (kEdgeTile + 4)) *
    static_cast<int64_t>(sizeof(float));

static int edge_args(const float* a, const float* b, int64_t B, int64_t Bt, int64_t C, int64_t H, int64_t W,
                     int64_t crop, float w, EdgeArgs* e) {
  if (!a || !b || B < 1 || C < 1 || H < 3 || W < 3 || (Bt != 1 && Bt != B) || crop < 0) return FVR_ERR_ARG;
  if (H - 2 * crop < 1 || W - 2 * crop < 1 || B * C > 65535 || H > 32768 || W > 32768) return FVR_ERR_ARG;
  e->a = a;
  e->b = b;
  e->B = (int)B;
  e->Bt = (int)Bt;
  e->Cch = (int)C;
  e->H = (int)H;
  e->W = (int)W;
  e->crop = (int)crop;
  e->coarse = (w > 0.f && W >= 96) ? 1 : 0;  // the reference tests the last dim (cone_beam_fvr.py:86, 107)
  e->tiles_x = (int)cdiv64(W - 2 * crop, kEdgeTile);
  e->tiles_y = (int)cdiv64(H - 2 * crop, kEdgeTile);
  return FVR_OK;
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int64_t fvr_edge_ncc_workspace(int64_t B, int64_t C, int64_t H, int64_t W, int64_t crop) {
  if (B < 1 || C < 1 || H - 2 * crop < 1 || W - 2 * crop < 1) return 0;
  return B * C * cdiv64(H - 2 * crop, kEdgeTile) * cdiv64(W - 2 * crop, kEdgeTile) * kEdgeCombos * kEdgeMom *
         (int64_t)sizeof(double);
}

int64_t fvr_edge_ncc_stats_count(void) { return kEdgeCombos * kEdgeMom; }

int fvr_edge_ncc_forward(const float* a, const float* b, int64_t B, int64_t Bt, int64_t C, int64_t H, int64_t W,
                         int64_t crop, float ms_weight, int reduction_mean, void* workspace, int64_t ws_bytes,
                         double* stats, float* out, void* stream) {
  EdgeArgs e;
  int rc = edge_args(a, b, B, Bt, C, H, W, crop, ms_weight, &e);
  if (rc) return rc;
  if (!workspace || !stats || !out) return FVR_ERR_ARG;
  if (ws_bytes < fvr_edge_ncc_workspace(B, C, H, W, crop)) return FVR_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  dim3 grid(e.tiles_x, e.tiles_y, static_cast<unsigned>(B * C));
  edge_moments_kernel<<<grid, kEdgeThreads, 0, s>>>(e, static_cast<double*>(workspace));
  FVR_LAUNCH_CHECK();
  edge_finalize_kernel<<<1, 256, 0, s>>>(e, static_cast<const double*>(workspace), ms_weight, stats, out,
                                         reduction_mean);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

int fvr_edge_ncc_backward(const float* a, const float* b, int64_t B, int64_t Bt, int64_t C, int64_t H, int64_t W,
                          int64_t crop, float ms_weight, int reduction_mean, const double* stats, const float* g,
                          int64_t g_stride, int wrt_b, float* grad, void* stream) {
  EdgeArgs e;
  int rc = edge_args(a, b, B, Bt, C, H, W, crop, ms_weight, &e);
  if (rc) return rc;
  if (!stats || !g || !grad) return FVR_ERR_ARG;
  // the shared-memory opt-in is a per-device setting: made before every launch
  if (cudaFuncSetAttribute(edge_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEdgeGradSmem) !=
      cudaSuccess)
    return FVR_ERR_CUDA;
  dim3 grid(static_cast<unsigned>(cdiv64(W, kEdgeTile)), static_cast<unsigned>(cdiv64(H, kEdgeTile)),
            static_cast<unsigned>(B * C));
  edge_grad_kernel<<<grid, kEdgeThreads, kEdgeGradSmem, static_cast<cudaStream_t>(stream)>>>(
      e, stats, ms_weight, g, (int)g_stride, reduction_mean, wrt_b, grad);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
