// Measurement utility (no reference counterpart): the gather ceiling of a
// cell sequence.  Reads the 32-byte stencil entries idx[0..n) with one
// 256-bit load each, UNROLL loads in flight per thread, and folds them into
// one word per thread, so its time is what the memory system needs to serve
// exactly the entries a moments launch reads, in the order it reads them,
// with no arithmetic around the loads.  Indices outside [0, n_entries) read
// nothing.
#include "fvr_stencil.cuh"

namespace fvr {

template <int UNROLL>
__global__ void __launch_bounds__(256) gather32_kernel(const uint4* __restrict__ entries, int64_t n_entries,
                                                       const int* __restrict__ idx, int64_t n,
                                                       unsigned* __restrict__ out) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  unsigned acc = 0;
  for (int64_t i0 = t; i0 < n; i0 += stride * UNROLL) {
    uint4 a[UNROLL], b[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const int64_t i = i0 + u * stride;
      const int64_t e = i < n ? static_cast<int64_t>(__ldg(idx + i)) : -1;
      if (e >= 0 && e < n_entries)
        ldg256(entries + 2 * e, a[u], b[u]);
      else
        a[u] = b[u] = make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) acc ^= a[u].x ^ a[u].y ^ a[u].z ^ a[u].w ^ b[u].x ^ b[u].y ^ b[u].z ^ b[u].w;
  }
  out[t] = acc;
}

}  // namespace fvr

using namespace fvr;

extern "C" {

int fvr_bench_gather32(const void* entries, int64_t n_entries, const int* idx, int64_t n, unsigned* out,
                       int64_t out_len, int blocks, void* stream) {
  if (!entries || !idx || !out || n_entries < 1 || n < 1 || blocks < 1) return FVR_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(entries) & 31) != 0) return FVR_ERR_ARG;
  if (out_len < static_cast<int64_t>(blocks) * 256) return FVR_ERR_WORKSPACE;
  gather32_kernel<3><<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const uint4*>(entries),
                                                                            n_entries, idx, n, out);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

}  // extern "C"
