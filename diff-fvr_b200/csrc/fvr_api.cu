// Status strings, version and device checks of the C ABI.
#include "fvr_common.cuh"

namespace {

// dst[0..n) = src[0..n); 16-byte words when both ends and n allow it.
__global__ void __launch_bounds__(256) copy_bytes_kernel(unsigned char* __restrict__ dst,
                                                         const unsigned char* __restrict__ src, int64_t n) {
  // a kernel launched after this one as its programmatic dependent may be
  // scheduled now; it still waits (griddepcontrol.wait) for this grid to
  // complete before it reads anything (no-op without such a dependent)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const bool wide = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15) == 0;
  const int64_t nw = wide ? n / 16 : 0;
  for (int64_t i = t; i < nw; i += stride)
    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
  for (int64_t i = nw * 16 + t; i < n; i += stride) dst[i] = src[i];
}

}  // namespace

#ifdef FVR_CHECK
namespace fvr {
int check_word_tc(unsigned long long* out, int clear);
int check_word_pou(unsigned long long* out, int clear);
int check_word_slice3d(unsigned long long* out, int clear);
int check_word_np(unsigned long long* out, int clear);
}  // namespace fvr
#endif

extern "C" {

int fvr_check_words(unsigned long long* out, int n, int clear) {
#ifdef FVR_CHECK
  using Reader = int (*)(unsigned long long*, int);
  const Reader readers[] = {fvr::check_word_tc, fvr::check_word_pou, fvr::check_word_slice3d, fvr::check_word_np};
  constexpr int kUnits = sizeof(readers) / sizeof(readers[0]);
  if (!out || n < kUnits) return FVR_ERR_ARG;
  for (int i = 0; i < kUnits; ++i)
    if (readers[i](out + i, clear)) return FVR_ERR_CUDA;
  return FVR_OK;
#else
  (void)out;
  (void)n;
  (void)clear;
  return FVR_ERR_UNSUPPORTED;
#endif
}

int fvr_copy_bytes(void* dst, const void* src, int64_t n, void* stream) {
  if (!dst || !src || n < 0) return FVR_ERR_ARG;
  if (n == 0) return FVR_OK;
  const int64_t blocks = (n / 16 + 255) / 256;
  copy_bytes_kernel<<<static_cast<unsigned>(blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks)), 256, 0,
                      static_cast<cudaStream_t>(stream)>>>(static_cast<unsigned char*>(dst),
                                                           static_cast<const unsigned char*>(src), n);
  FVR_LAUNCH_CHECK();
  return FVR_OK;
}

const char* fvr_status_string(int status) {
  switch (status) {
    case FVR_OK: return "ok";
    case FVR_ERR_ARG: return "invalid argument (null pointer, size, stride or alignment)";
    case FVR_ERR_DTYPE: return "unsupported dtype";
    case FVR_ERR_UNSUPPORTED: return "unsupported size (e.g. FFT length with a prime factor above 127)";
    case FVR_ERR_WORKSPACE: return "workspace too small";
    case FVR_ERR_CUDA: return "CUDA launch or driver error";
    default: return "unknown fvr status";
  }
}

int fvr_version(void) { return 100; }

int fvr_device_supported(int device) {
  int major = 0, minor = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess) return 0;
  return major == 10 ? 1 : 0;
}

int fvr_event_record(void* event, void* stream, int external) {
  if (!event) return FVR_ERR_ARG;
  cudaError_t e = external ? cudaEventRecordWithFlags(static_cast<cudaEvent_t>(event),
                                                      static_cast<cudaStream_t>(stream), cudaEventRecordExternal)
                           : cudaEventRecord(static_cast<cudaEvent_t>(event), static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? FVR_OK : FVR_ERR_CUDA;
}

}  // extern "C"
