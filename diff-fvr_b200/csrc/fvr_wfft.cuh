// Warp-level complex FFT of length N = 32 M (M = 2, 3, 4, 5) held in
// registers: lane l holds x[l + 32 m], m < M.  Four-step split N = M x 32:
// an M-point DFT per lane, a twiddle W_N^(l k2), then a 32-point radix-2
// decimation-in-frequency across the lanes with shuffles.  On return lane l
// holds X[k2 + M brev5(l)] in x[k2], i.e. element k of the transform sits at
// "position" brev5(k / M) + 32 (k % M) when lanes are laid out along a row
// (brev5 = 5-bit reversal), which keeps shared-memory stores of a whole warp
// contiguous.  Unnormalised; INV selects e^{+2 pi i / N}.
#pragma once

#include "fvr_dft.cuh"

namespace fvr {

__device__ __forceinline__ int brev5(int x) { return static_cast<int>(__brev(static_cast<unsigned>(x)) >> 27); }

// Storage position of transform element k (see above).
template <int M>
__device__ __forceinline__ int wfft_pos(int k) {
  return brev5(k / M) + 32 * (k % M);
}

template <int M, bool INV>
struct WarpFft {
  Cx<float> stw[5];  // stage s (half size h = 16 >> s): W_{2h}^(l mod h)
  Cx<float> itw[M];  // W_N^(l k2)

  __device__ __forceinline__ void init(int lane) {
    constexpr float sgn = INV ? 1.f : -1.f;
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const int h = 16 >> s;
      float sn, cs;
      sincospif(static_cast<float>(lane % h) / static_cast<float>(h), &sn, &cs);
      stw[s] = Cx<float>{cs, sgn * sn};
    }
#pragma unroll
    for (int k = 0; k < M; ++k) {
      float sn, cs;
      sincospif(2.f * static_cast<float>(lane * k) / static_cast<float>(32 * M), &sn, &cs);
      itw[k] = Cx<float>{cs, sgn * sn};
    }
  }

  __device__ __forceinline__ void run(Cx<float> (&x)[M], int lane) const {
    Dft<float, M>::run(x, INV);
#pragma unroll
    for (int k = 1; k < M; ++k) x[k] = cmul(x[k], itw[k]);
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const int h = 16 >> s;
      const bool upper = (lane & h) != 0;
#pragma unroll
      for (int k = 0; k < M; ++k) {
        Cx<float> p;
        p.x = __shfl_xor_sync(0xffffffffu, x[k].x, h);
        p.y = __shfl_xor_sync(0xffffffffu, x[k].y, h);
        x[k] = upper ? cmul(csub(p, x[k]), stw[s]) : cadd(x[k], p);
      }
    }
  }
};

}  // namespace fvr
