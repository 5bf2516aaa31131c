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

template <int DT>
__device__ __forceinline__ void stencil_load(const Stencil& s, int ez, int ey, int ex, Sample8& v) {
  const int64_t e = (static_cast<int64_t>(ez) * (s.H + 1) + ey) * (s.W + 1) + ex;
  if constexpr (DT == FVR_F32) {
    const float4* p = static_cast<const float4*>(s.data) + e * 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float4 f = __ldg(p + i);
      v.re[2 * i] = f.x;
      v.im[2 * i] = f.y;
      v.re[2 * i + 1] = f.z;
      v.im[2 * i + 1] = f.w;
    }
  } else {
    const uint4* p = static_cast<const uint4*>(s.data) + e * 2;
    uint4 a = __ldg(p), b = __ldg(p + 1);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    if constexpr (DT == FVR_BF16) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        v.re[i] = bf_lo(w[i]);
        v.im[i] = bf_hi(w[i]);
      }
    } else {
      const int bx = (s.W + 1 + kBrick - 1) / kBrick, by = (s.H + 1 + kBrick - 1) / kBrick;
      const float sc = __ldg(s.scales + (static_cast<int64_t>(ez / kBrick) * by + ey / kBrick) * bx + ex / kBrick);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        v.re[i] = h_lo(w[i]) * sc;
        v.im[i] = h_hi(w[i]) * sc;
      }
    }
  }
}

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

// Sample the stencil spectrum at p (voxel coords x=W, y=H, z=D).
// HARD=false: zero-padding partial interpolation (grid_sample padding 'zeros').
// HARD=true : scipy map_coordinates(order=1, mode='constant'): zero unless
//             0 <= p <= n-1 on every axis.
// Returns false (and a zero sample) when nothing of the stencil is inside.
template <int DT, bool DERIV, bool HARD>
__device__ __forceinline__ bool stencil_sample(const Stencil& s, float px, float py, float pz, Interp& o) {
  bool ok;
  if (HARD) {
    ok = (px >= 0.f) && (px <= static_cast<float>(s.W - 1)) && (py >= 0.f) &&
         (py <= static_cast<float>(s.H - 1)) && (pz >= 0.f) && (pz <= static_cast<float>(s.D - 1));
  } else {
    ok = (px >= -1.f) && (px < static_cast<float>(s.W)) && (py >= -1.f) && (py < static_cast<float>(s.H)) &&
         (pz >= -1.f) && (pz < static_cast<float>(s.D));
  }
  if (!ok) {
    o = Interp{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    return false;
  }
  const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  const int ix = static_cast<int>(fx), iy = static_cast<int>(fy), iz = static_cast<int>(fz);
  Sample8 v;
  stencil_load<DT>(s, iz + 1, iy + 1, ix + 1, v);
  trilerp<DERIV>(v, px - fx, py - fy, pz - fz, o);
  return true;
}

}  // namespace fvr
