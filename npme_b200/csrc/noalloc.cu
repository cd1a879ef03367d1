// npme_gpu_direct_sum_device_noalloc: the short-range direct sum with its
// scratch in static device memory instead of memory from an allocator.
//
// Who needs it: a caller that cannot call cudaMalloc at the moment it wants
// the direct sum.  Examples are code running under another framework's
// memory manager that has reserved the device's memory up front (an extra
// cudaMalloc can fail or fragment that pool), and latency-critical callers
// that must not let an allocation synchronise the device while other streams
// are busy.  Those callers still create and set up the handle beforehand;
// this entry point itself calls no cudaMalloc, cudaFree or allocating library
// routine.
//
// The only per-call scratch of the direct sum is the caller's charges
// gathered into the direct-sum order.  Here it lives in g_direct_scratch, a
// file-scope __device__ array of kNoAllocScratchBytes (8 MiB), which every GPU
// that loads this library holds until the process exits.  Limits: n points
// fit when n * (4 bytes FP32 | 8 bytes FP64) * (1 real | 2 complex) <= 8 MiB,
// i.e. 2,097,152 points (FP32 real), 1,048,576 (FP32 complex or FP64 real),
// 524,288 (FP64 complex); larger systems are rejected with NPME_EINVAL.
//
// In host code g_direct_scratch is only a host-side stand-in for the device
// symbol, never a device address.  Every call (with the handle's device
// current) looks the address up with cudaGetSymbolAddress, which allocates
// nothing once this module is on the device.  The module, and with it the
// 8 MiB array, is loaded onto a device when npme_gpu_setup first runs there
// (CUDA loads modules lazily by default): set-up is the point where the
// caller still allows allocation, so the first no-allocation call does not
// make the driver reserve memory.  Looking the address up on every call also
// keeps it right after cudaDeviceReset or a new primary context.  All calls
// on a device share the one array and it keeps the last call's contents: the
// gather overwrites every byte the sum reads, so nothing has to start at
// zero, but calls whose work overlaps on the GPU (two streams, or two
// handles) race on the array.  Serialise them.
#include <cuda_runtime.h>

#include <string>

#include "internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
__device__ __align__(256) unsigned char g_direct_scratch[kNoAllocScratchBytes];

int scratch_address(void **ptr, std::string &err) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
  if (e != cudaSuccess || p == nullptr) {
    err = std::string("cudaGetSymbolAddress of the static direct-sum scratch failed: ") +
          cudaGetErrorString(e);
    return NPME_ECUDA;
  }
  *ptr = p;
  return NPME_OK;
}

}  // namespace

namespace npme {
// Loads this module (and its static array) onto the current device; called by
// npme_gpu_setup, where allocation is still allowed.
int noalloc_preload(std::string &err) {
  void *p = nullptr;
  return scratch_address(&p, err);
}
}  // namespace npme

extern "C" int npme_gpu_direct_sum_device_noalloc(npme_handle *h, double *d_V,
                                                  const double *d_charge, void *stream) {
  if (!h) return npme::record_error(nullptr, NPME_EINVAL, "null handle");
  if (!h->ready) {
    h->err = "direct_sum_noalloc before setup";
    return NPME_ESTATE;
  }
  if (!d_V || !d_charge) {
    h->err = "null buffer";
    return NPME_EINVAL;
  }
  const size_t per_point = (h->fp32 ? sizeof(float) : sizeof(double)) * (h->complex_kernel ? 2 : 1);
  const size_t need = per_point * h->n;
  if (need > kNoAllocScratchBytes) {
    h->err = "direct_sum_noalloc: " + std::to_string(h->n) + " points need " +
             std::to_string(need) + " bytes of scratch, above the static " +
             std::to_string(kNoAllocScratchBytes) + "-byte array (at most " +
             std::to_string(kNoAllocScratchBytes / per_point) +
             " points in this mode); use npme_gpu_direct_sum_device";
    return NPME_EINVAL;
  }
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) {
    h->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    return NPME_ECUDA;
  }
  void *scratch = nullptr;
  const int rc = scratch_address(&scratch, h->err);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the default stream
  h->launches = 0;
  npme::launch_gather_direct(h, d_charge, scratch, s);
  npme::DirectArgs a{scratch, d_charge, 0.0, 0.0, d_V};
  if (npme::launch_direct_args(h, a, s)) {
    h->err = "direct_sum_noalloc: launch of the caller-defined kernel failed";
    return NPME_ECUDA;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    h->err = std::string("direct_sum_noalloc launch: ") + cudaGetErrorString(e);
    return NPME_ECUDA;
  }
  return NPME_OK;
}
