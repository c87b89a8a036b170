// ssn_noalloc.cu -- ssn_gram_noalloc: the Gram products of ssn_gram with their
// scratch (the split-K partial sums) in a fixed, statically allocated device
// array instead of a caller-provided workspace.
//
// Who needs it: callers that cannot allocate device memory at the point of the
// call -- e.g. a host framework whose pooling allocator already owns the whole
// device and will not hand a raw buffer to foreign code, or a latency-critical
// caller that must never reach cudaMalloc, which can synchronise the device and
// can fail under memory pressure.  They pass inputs and outputs only.
//
// Limits and sharing rules:
//  * the scratch is kNoAllocScratchBytes (16 MiB) of device memory, held by
//    every GPU that loads this library until the process exits;
//  * a call needs batch * splits * 2 * m^2 doubles of it; the row split count is
//    lowered to fit, and a call whose batch * 2 * m^2 doubles exceed the array
//    is rejected with SSN_ERR_SCRATCH_LIMIT before anything is launched;
//  * all calls share the one array, which keeps the previous call's contents:
//    every partial sum a call reads is written by the same call first, so no
//    clearing is needed; calls that overlap on the GPU (other streams, other
//    host threads) race on it and must be serialised by the caller;
//  * the first call on each device resolves the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it per device
//    index for the life of the process; that first call should come before any
//    stream capture.  Resetting the device or recreating its primary context
//    (cudaDeviceReset) while the library stays loaded is not supported: the
//    cached address would then be stale.
#include <mutex>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_gram_scratch[kNoAllocScratchDoubles];

namespace {
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_gram_scratch on the current device (the host-side name
// is only a stand-in and must never be passed to a kernel).
cudaError_t scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_gram_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}
}  // namespace

}  // namespace ssn

extern "C" {

size_t ssn_gram_noalloc_scratch_bytes(void) { return ssn::kNoAllocScratchBytes; }

int ssn_gram_noalloc(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                     int batch, int rows, int m, ssn_stream_t stream) {
  using namespace ssn;
  if (batch < 1 || m < 2 || m > kMaxM || (m % 2) != 0 || rows < 1 || !A || !D || !Cr || !Ci ||
      ab_stride < (int64_t)rows * m || (ab_stride % 2) != 0 ||
      (reinterpret_cast<uintptr_t>(A) & 15u) != 0 || (reinterpret_cast<uintptr_t>(D) & 15u) != 0)
    return SSN_ERR_INVALID_ARGUMENT;
  const size_t per_split = (size_t)batch * 2 * m * m;   // doubles of partial sums per row split
  if (per_split > kNoAllocScratchDoubles) return SSN_ERR_SCRATCH_LIMIT;
  const int max_splits = (int)(kNoAllocScratchDoubles / per_split);
  double* scratch = nullptr;
  if (scratch_on_current_device(&scratch) != cudaSuccess) return SSN_ERR_CUDA;
  const cudaError_t e = launch_gram(A, D, ab_stride, Cr, Ci, batch, rows, m, scratch,
                                    reinterpret_cast<cudaStream_t>(stream), max_splits);
  return e == cudaSuccess ? SSN_OK : SSN_ERR_CUDA;
}

}  // extern "C"
