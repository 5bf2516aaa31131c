// Status strings, version and device checks of the C ABI.
#include "fvr_common.cuh"

extern "C" {

const char* fvr_status_string(int status) {
  switch (status) {
    case FVR_OK: return "ok";
    case FVR_ERR_ARG: return "invalid argument (null pointer, size, stride or alignment)";
    case FVR_ERR_DTYPE: return "unsupported dtype";
    case FVR_ERR_UNSUPPORTED: return "unsupported size (e.g. FFT length with a prime factor above 127)";
    case FVR_ERR_WORKSPACE: return "workspace too small";
    case FVR_ERR_CUDA: return "CUDA launch or driver error";
    case FVR_ERR_TIMEOUT: return "device-side wait timed out";
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
