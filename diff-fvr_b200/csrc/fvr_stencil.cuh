// Stencil ("corner-cube") spectrum layout and the trilinear fetch built on it.
//
// A centred complex spectrum of D x H x W voxels is stored as an entry grid of
// (D+1) x (H+1) x (W+1) entries.  Entry (ez, ey, ex) holds the 8 complex
// corners of the cell whose low corner is voxel (ez-1, ey-1, ex-1), ordered
// c = dz*4 + dy*2 + dx, with corners outside the volume stored as zero.  A
// trilinear sample at p therefore reads exactly one aligned entry:
//   f32 : 64 B (4 x 16-byte vector loads, two 32-byte sectors)
//   bf16: 32 B (2 x 16-byte vector loads, one 32-byte sector)
//   f16 : 32 B + one per-16^3-entry-brick power-of-two scale (exact rescale)
// This spends 8x the HBM of a plain array (180 GB per B200 makes that cheap)
// to turn the 8 scattered corner reads of the reference gather
// (src/fvr/triton_slice.py:38-44, 119-138: 16 scalar loads per sample, real
// and imaginary planes far apart) into one fully used sector (bf16) or two
// (f32), and removes all per-corner bounds checks: zero padding outside the
// volume is materialised in the entries.
#pragma once

#include "fvr_common.cuh"

namespace fvr {

constexpr int kBrick = 16;  // f16 scale brick edge, in entries

struct Stencil {
  const void* data;
  const float* scales;  // f16 only: [ceil(D1/16)][ceil(H1/16)][ceil(W1/16)]
  int D, H, W;          // spectrum (voxel) dims
  int dtype;            // FVR_F32 / FVR_BF16 / FVR_F16
};

struct Sample8 {
  float re[8], im[8];
};

// Trilinear value and spatial derivatives from the 8 corners (nested lerps).
struct Interp {
  float sr, si;                        // value
  float dxr, dxi, dyr, dyi, dzr, dzi;  // d/dx, d/dy, d/dz
};

template <bool DERIV>
__device__ __forceinline__ void trilerp(const Sample8& v, float tx, float ty, float tz, Interp& o) {
  float ar[4], ai[4], xr[4], xi[4];
#pragma unroll
  for (int zy = 0; zy < 4; ++zy) {
    const float r0 = v.re[2 * zy], r1 = v.re[2 * zy + 1], i0 = v.im[2 * zy], i1 = v.im[2 * zy + 1];
    xr[zy] = r1 - r0;
    xi[zy] = i1 - i0;
    ar[zy] = fmaf(tx, xr[zy], r0);
    ai[zy] = fmaf(tx, xi[zy], i0);
  }
  // zy index = dz*2 + dy
  const float byr0 = ar[1] - ar[0], byi0 = ai[1] - ai[0], byr1 = ar[3] - ar[2], byi1 = ai[3] - ai[2];
  const float br0 = fmaf(ty, byr0, ar[0]), bi0 = fmaf(ty, byi0, ai[0]);
  const float br1 = fmaf(ty, byr1, ar[2]), bi1 = fmaf(ty, byi1, ai[2]);
  o.dzr = br1 - br0;
  o.dzi = bi1 - bi0;
  o.sr = fmaf(tz, o.dzr, br0);
  o.si = fmaf(tz, o.dzi, bi0);
  if (DERIV) {
    o.dyr = fmaf(tz, byr1 - byr0, byr0);
    o.dyi = fmaf(tz, byi1 - byi0, byi0);
    const float cxr0 = fmaf(ty, xr[1] - xr[0], xr[0]), cxi0 = fmaf(ty, xi[1] - xi[0], xi[0]);
    const float cxr1 = fmaf(ty, xr[3] - xr[2], xr[2]), cxi1 = fmaf(ty, xi[3] - xi[2], xi[2]);
    o.dxr = fmaf(tz, cxr1 - cxr0, cxr0);
    o.dxi = fmaf(tz, cxi1 - cxi0, cxi0);
  }
}

// ---- packed (re, im) form: sm_100 FP32x2 arithmetic ------------------------
//
// Every step of the trilinear lerp treats the real and imaginary parts alike,
// so a corner kept as a float2 (re, im) pair goes through one fma.rn.f32x2 /
// add.rn.f32x2 per step instead of two scalar instructions.  Each component
// is rounded exactly as the scalar form rounds it: a - b is formed as
// fma(b, -1, a), a single rounding of the exact difference.

__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

struct Sample8c {
  float2 c[8];  // corner (re, im), c = dz*4 + dy*2 + dx
};

struct Interp2 {
  float2 s;           // value
  float2 d[3];        // d/dx, d/dy, d/dz
};

// trilerp in packed form: the same nested lerps, component for component.
template <bool DERIV>
__device__ __forceinline__ void trilerp2(const Sample8c& v, float tx, float ty, float tz, Interp2& o) {
  const float2 TX = f2(tx), TY = f2(ty), TZ = f2(tz);
  float2 a[4], x[4];
#pragma unroll
  for (int zy = 0; zy < 4; ++zy) {
    x[zy] = sub2(v.c[2 * zy + 1], v.c[2 * zy]);
    a[zy] = fma2(TX, x[zy], v.c[2 * zy]);
  }
  const float2 by0 = sub2(a[1], a[0]), by1 = sub2(a[3], a[2]);
  const float2 b0 = fma2(TY, by0, a[0]), b1 = fma2(TY, by1, a[2]);
  o.d[2] = sub2(b1, b0);
  o.s = fma2(TZ, o.d[2], b0);
  if (DERIV) {
    o.d[1] = fma2(TZ, sub2(by1, by0), by0);
    const float2 cx0 = fma2(TY, sub2(x[1], x[0]), x[0]);
    const float2 cx1 = fma2(TY, sub2(x[3], x[2]), x[2]);
    o.d[0] = fma2(TZ, sub2(cx1, cx0), cx0);
  }
}

// ---- split load / decode, so a thread can put several samples' loads in flight

// One 256-bit read-only load (sm_100 ld.global.nc.v8): a whole 32-byte stencil
// entry (16-bit storage) or half of one (f32) per instruction.  `p` must be
// 32-byte aligned (entries are 32 or 64 bytes, the buffer base is aligned).
__device__ __forceinline__ void ldg256(const void* p, uint4& a, uint4& b) {
  asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
               : "l"(p));
}
__device__ __forceinline__ void ldg256(const float4* p, float4& a, float4& b) {
  uint4 ua, ub;
  ldg256(static_cast<const void*>(p), ua, ub);
  a = make_float4(__uint_as_float(ua.x), __uint_as_float(ua.y), __uint_as_float(ua.z), __uint_as_float(ua.w));
  b = make_float4(__uint_as_float(ub.x), __uint_as_float(ub.y), __uint_as_float(ub.z), __uint_as_float(ub.w));
}

template <int DT>
struct Raw;
template <>
struct Raw<FVR_F32> {
  float4 q[4];
};
template <>
struct Raw<FVR_BF16> {
  uint4 q[2];
};
template <>
struct Raw<FVR_F16> {
  uint4 q[2];
  float sc;
};
// x-pair storage (16-bit): q[0] = entry ex (the cell's x = 0 corners), q[1] =
// entry ex + 1 (x = 1), each ordered dz*2 + dy; f16: the scale of their
// (z, y) slab, which spans every x.
template <>
struct Raw<FVR_BF16_PAIR> {
  uint4 q[2];
};
template <>
struct Raw<FVR_F16_PAIR> {
  uint4 q[2];
  float sc;
};
// f32 x-pair: q[0..1] = entry ex, q[2..3] = entry ex + 1 (two complex each).
template <>
struct Raw<FVR_F32_PAIR> {
  float4 q[4];
};

constexpr bool is_pair(int dt) { return dt == FVR_BF16_PAIR || dt == FVR_F16_PAIR || dt == FVR_F32_PAIR; }

// x-pair entry grid: (D+1)(H+1)(W+2) entries; f16 scales per (z, y) slab of
// kBrick x kBrick entry rows.
__device__ __forceinline__ int64_t pair_entries(const Stencil& s) {
  return static_cast<int64_t>(s.D + 1) * (s.H + 1) * (s.W + 2);
}
__device__ __forceinline__ int64_t pair_scales(const Stencil& s) {
  return static_cast<int64_t>((s.D + kBrick) / kBrick) * ((s.H + kBrick) / kBrick);
}

// Two 128-bit read-only loads of the 32 contiguous bytes at p (16-byte aligned).
__device__ __forceinline__ void ldg128x2(const uint4* p, uint4& a, uint4& b) {
  a = __ldg(p);
  b = __ldg(p + 1);
}

// The two x-pair entries of cell index e (entry ex of its row; e + 1 is
// entry ex + 1), f16 with the scale of the cell's (z, y) slab; zeros and a
// zero scale when e < 0 or (checked build) out of bounds.
template <int DT>
__device__ __forceinline__ void pair_load(const Stencil& s, int64_t e, int ez, int ey, Raw<DT>& r) {
  if (e < 0 || !fvr_checked(e + 1, pair_entries(s), kSiteStencilEntry)) {
    if constexpr (DT == FVR_F32_PAIR) {
#pragma unroll
      for (int i = 0; i < 4; ++i) r.q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      r.q[0] = r.q[1] = make_uint4(0u, 0u, 0u, 0u);
      if constexpr (DT == FVR_F16_PAIR) r.sc = 0.f;
    }
    return;
  }
  if constexpr (DT == FVR_F32_PAIR) {
    const float4* p = static_cast<const float4*>(s.data) + e * 2;  // 32-byte entries
    ldg256(p, r.q[0], r.q[1]);
    ldg256(p + 2, r.q[2], r.q[3]);
  } else {
    ldg128x2(static_cast<const uint4*>(s.data) + e, r.q[0], r.q[1]);
    if constexpr (DT == FVR_F16_PAIR) {
      const unsigned by = static_cast<unsigned>(s.H + kBrick) / kBrick;
      const unsigned si = (static_cast<unsigned>(ez) / kBrick) * by + static_cast<unsigned>(ey) / kBrick;
      r.sc = fvr_checked(si, pair_scales(s), kSiteStencilScale) ? __ldg(s.scales + si) : 0.f;
    }
  }
}

// Cell address of p (FP64 voxel coordinates; zero-padding partial or hard cut-off).
struct Cell {
  int64_t e;           // entry index, -1 when no corner is inside
  float tx, ty, tz;    // fractional position inside the cell
  int ez, ey, ex;      // entry coordinates (for the f16 brick scale)
};

template <bool HARD>
__device__ __forceinline__ Cell stencil_cell(const Stencil& s, double px, double py, double pz) {
  Cell c;
  bool ok;
  if (HARD) {
    ok = (px >= 0.0) && (px <= static_cast<double>(s.W - 1)) && (py >= 0.0) &&
         (py <= static_cast<double>(s.H - 1)) && (pz >= 0.0) && (pz <= static_cast<double>(s.D - 1));
  } else {
    ok = (px >= -1.0) && (px < static_cast<double>(s.W)) && (py >= -1.0) && (py < static_cast<double>(s.H)) &&
         (pz >= -1.0) && (pz < static_cast<double>(s.D));
  }
  if (!ok) {
    c.e = -1;
    c.tx = c.ty = c.tz = 0.f;
    c.ez = c.ey = c.ex = 0;
    return c;
  }
  const double fx = floor(px), fy = floor(py), fz = floor(pz);
  c.tx = static_cast<float>(px - fx);
  c.ty = static_cast<float>(py - fy);
  c.tz = static_cast<float>(pz - fz);
  c.ex = static_cast<int>(fx) + 1;
  c.ey = static_cast<int>(fy) + 1;
  c.ez = static_cast<int>(fz) + 1;
  c.e = (static_cast<int64_t>(c.ez) * (s.H + 1) + c.ey) * (s.W + 1) + c.ex;
  return c;
}

__device__ __forceinline__ int64_t stencil_entries(const Stencil& s) {
  return static_cast<int64_t>(s.D + 1) * (s.H + 1) * (s.W + 1);
}
__device__ __forceinline__ int64_t stencil_scales(const Stencil& s) {
  return static_cast<int64_t>((s.D + kBrick) / kBrick) * ((s.H + kBrick) / kBrick) * ((s.W + kBrick) / kBrick);
}

template <int DT>
__device__ __forceinline__ void raw_load(const Stencil& s, const Cell& c, Raw<DT>& r) {
  if constexpr (DT == FVR_F32) {
    if (c.e < 0 || !fvr_checked(c.e, stencil_entries(s), kSiteStencilEntry)) {
#pragma unroll
      for (int i = 0; i < 4; ++i) r.q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      return;
    }
    const float4* p = static_cast<const float4*>(s.data) + c.e * 4;
    ldg256(p, r.q[0], r.q[1]);
    ldg256(p + 2, r.q[2], r.q[3]);
  } else {
    if (c.e < 0 || !fvr_checked(c.e, stencil_entries(s), kSiteStencilEntry)) {
      r.q[0] = r.q[1] = make_uint4(0u, 0u, 0u, 0u);
      if constexpr (DT == FVR_F16) r.sc = 0.f;
      return;
    }
    const uint4* p = static_cast<const uint4*>(s.data) + c.e * 2;
    ldg256(p, r.q[0], r.q[1]);
    if constexpr (DT == FVR_F16) {
      const int bx = (s.W + 1 + kBrick - 1) / kBrick, by = (s.H + 1 + kBrick - 1) / kBrick;
      const int64_t si = (static_cast<int64_t>(c.ez / kBrick) * by + c.ey / kBrick) * bx + c.ex / kBrick;
      r.sc = fvr_checked(si, stencil_scales(s), kSiteStencilScale) ? __ldg(s.scales + si) : 0.f;
    }
  }
}

template <int DT>
__device__ __forceinline__ void raw_decode(const Raw<DT>& r, Sample8& v) {
  if constexpr (DT == FVR_F32) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v.re[2 * i] = r.q[i].x;
      v.im[2 * i] = r.q[i].y;
      v.re[2 * i + 1] = r.q[i].z;
      v.im[2 * i + 1] = r.q[i].w;
    }
  } else {
    const uint32_t w[8] = {r.q[0].x, r.q[0].y, r.q[0].z, r.q[0].w, r.q[1].x, r.q[1].y, r.q[1].z, r.q[1].w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if constexpr (DT == FVR_BF16) {
        v.re[i] = bf_lo(w[i]);
        v.im[i] = bf_hi(w[i]);
      } else {
        v.re[i] = h_lo(w[i]) * r.sc;
        v.im[i] = h_hi(w[i]) * r.sc;
      }
    }
  }
}

// Sample the stencil spectrum at p (FP64 voxel coords x=W, y=H, z=D): value
// and, with DERIV, derivatives.
// HARD=false: zero-padding partial interpolation (grid_sample padding 'zeros').
// HARD=true : scipy map_coordinates(order=1, mode='constant'): zero unless
//             0 <= p <= n-1 on every axis.
template <int DT, bool DERIV, bool HARD>
__device__ __forceinline__ bool stencil_sample_d(const Stencil& s, double px, double py, double pz, Interp& o) {
  const Cell c = stencil_cell<HARD>(s, px, py, pz);
  Raw<DT> r;
  raw_load<DT>(s, c, r);
  Sample8 v;
  raw_decode<DT>(r, v);
  trilerp<DERIV>(v, c.tx, c.ty, c.tz, o);
  return c.e >= 0;
}

// ---- per-CTA split-position tables (shared by the slice kernels) ---------

// Per-CTA sample tables.  The slice position s + ku*u + kv*v is split into a
// row part (s + ku*u, ku = lin[i]) and a column part (kv*v, kv = lin[j]); each
// is formed in FP64 once per CTA and kept as an integer cell index plus a
// float fraction in [0, 1], so a sample's position (their sum) is the FP64
// position to within 2^-24 of a cell with integer adds and one float add per
// axis.  The phase ramp factorises the same way:
//   e^{i pi kpi (ku tx + kv ty)} = e^{i pi kpi ku tx} . e^{i pi kpi kv ty},
// each factor from FP64 sincospi.  Entry n < R is column n; entry R + r is row
// row0 + r.  (Kernels without a phase ramp leave ph unused.)
struct AxisTables {
  int4* idx;    // (floor x, floor y, floor z, -)
  float4* frac; // (frac x, frac y, frac z, k)
  float2* ph;   // (cos, sin)
};

__device__ __forceinline__ AxisTables axis_tables(unsigned char* smem, int n_tab) {
  AxisTables t;
  t.idx = reinterpret_cast<int4*>(smem);
  t.frac = reinterpret_cast<float4*>(smem + 16 * n_tab);
  t.ph = reinterpret_cast<float2*>(smem + 32 * n_tab);
  return t;
}

// Cell of sample (row entry a, column entry b); e = -1 when no corner of the
// cell is inside (zero-padding partial: -1 <= p < n on every axis).
struct TabCell {
  int e;
  float tx, ty, tz;
  int ex, ey, ez;
};

__device__ __forceinline__ TabCell tab_cell(const Stencil& s, int4 ia, float4 fa, int4 ib, float4 fb) {
  TabCell c;
  c.tx = fa.x + fb.x;
  c.ty = fa.y + fb.y;
  c.tz = fa.z + fb.z;
  int ix = ia.x + ib.x, iy = ia.y + ib.y, iz = ia.z + ib.z;
  if (c.tx >= 1.f) { c.tx -= 1.f; ++ix; }
  if (c.ty >= 1.f) { c.ty -= 1.f; ++iy; }
  if (c.tz >= 1.f) { c.tz -= 1.f; ++iz; }
  c.ex = ix + 1;
  c.ey = iy + 1;
  c.ez = iz + 1;
  const bool ok = static_cast<unsigned>(c.ex) <= static_cast<unsigned>(s.W) &&
                  static_cast<unsigned>(c.ey) <= static_cast<unsigned>(s.H) &&
                  static_cast<unsigned>(c.ez) <= static_cast<unsigned>(s.D);
  c.e = ok ? (c.ez * (s.H + 1) + c.ey) * (s.W + 1) + c.ex : -1;
  return c;
}

// Entry load without the f16 brick scale applied (it multiplies the
// interpolated value and derivatives instead: 8 products, not 16).
template <int DT>
__device__ __forceinline__ void tab_load(const Stencil& s, const TabCell& c, Raw<DT>& r) {
  if constexpr (DT == FVR_F32) {
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
      const int bx = (s.W + kBrick) / kBrick, by = (s.H + kBrick) / kBrick;
      const int si = ((c.ez / kBrick) * by + c.ey / kBrick) * bx + c.ex / kBrick;
      r.sc = fvr_checked(si, stencil_scales(s), kSiteStencilScale) ? __ldg(s.scales + si) : 0.f;
    }
  }
}

template <int DT>
__device__ __forceinline__ void tab_decode(const Raw<DT>& r, Sample8& v) {
  if constexpr (DT == FVR_F16) {
    const uint32_t w[8] = {r.q[0].x, r.q[0].y, r.q[0].z, r.q[0].w, r.q[1].x, r.q[1].y, r.q[1].z, r.q[1].w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v.re[i] = h_lo(w[i]);
      v.im[i] = h_hi(w[i]);
    }
  } else {
    raw_decode<DT>(r, v);
  }
}

// Corners as (re, im) pairs, f16 without its brick scale (as tab_decode).
template <int DT>
__device__ __forceinline__ void tab_decode2(const Raw<DT>& r, Sample8c& v) {
  if constexpr (DT == FVR_F32_PAIR) {
    // corner c = dz*4 + dy*2 + dx: x = 0 corners from entry ex, x = 1 from ex + 1
    v.c[0] = make_float2(r.q[0].x, r.q[0].y);
    v.c[2] = make_float2(r.q[0].z, r.q[0].w);
    v.c[4] = make_float2(r.q[1].x, r.q[1].y);
    v.c[6] = make_float2(r.q[1].z, r.q[1].w);
    v.c[1] = make_float2(r.q[2].x, r.q[2].y);
    v.c[3] = make_float2(r.q[2].z, r.q[2].w);
    v.c[5] = make_float2(r.q[3].x, r.q[3].y);
    v.c[7] = make_float2(r.q[3].z, r.q[3].w);
  } else if constexpr (is_pair(DT)) {
    // corner c = dz*4 + dy*2 + dx: x = 0 corners from q[0], x = 1 from q[1]
    const uint32_t w0[4] = {r.q[0].x, r.q[0].y, r.q[0].z, r.q[0].w};
    const uint32_t w1[4] = {r.q[1].x, r.q[1].y, r.q[1].z, r.q[1].w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if constexpr (DT == FVR_BF16_PAIR) {
        v.c[2 * k] = make_float2(bf_lo(w0[k]), bf_hi(w0[k]));
        v.c[2 * k + 1] = make_float2(bf_lo(w1[k]), bf_hi(w1[k]));
      } else {
        v.c[2 * k] = make_float2(h_lo(w0[k]), h_hi(w0[k]));
        v.c[2 * k + 1] = make_float2(h_lo(w1[k]), h_hi(w1[k]));
      }
    }
  } else if constexpr (DT == FVR_F32) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v.c[2 * i] = make_float2(r.q[i].x, r.q[i].y);
      v.c[2 * i + 1] = make_float2(r.q[i].z, r.q[i].w);
    }
  } else {
    const uint32_t w[8] = {r.q[0].x, r.q[0].y, r.q[0].z, r.q[0].w, r.q[1].x, r.q[1].y, r.q[1].z, r.q[1].w};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if constexpr (DT == FVR_BF16)
        v.c[i] = make_float2(bf_lo(w[i]), bf_hi(w[i]));
      else
        v.c[i] = make_float2(h_lo(w[i]), h_hi(w[i]));
    }
  }
}

template <int DT>
__device__ __forceinline__ float raw_scale(const Raw<DT>& r) {
  if constexpr (DT == FVR_F16 || DT == FVR_F16_PAIR)
    return r.sc;
  else
    return 1.f;
}

}  // namespace fvr
