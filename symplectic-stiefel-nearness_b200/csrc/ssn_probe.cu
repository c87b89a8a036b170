// ssn_probe.cu -- FP64 tensor-pipe rate probe (measurement helper; no reference
// counterpart).  Each warp keeps 8 independent DMMA accumulator chains so the
// launch is limited by the FP64 pipe, not by latency.  Bounded loop, no waits.
#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

constexpr int kProbeThreads = 256;
constexpr int kProbeChains = 8;
constexpr int kProbeUnroll = 4;

__global__ void __launch_bounds__(kProbeThreads) probe_fp64_mma_kernel(double* sink, int iters) {
  const double a = 1.0 + threadIdx.x * 1e-6, b = 1.0 - threadIdx.x * 1e-7;
  double c[kProbeChains][2];
#pragma unroll
  for (int i = 0; i < kProbeChains; ++i) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kProbeUnroll; ++u)
#pragma unroll
      for (int i = 0; i < kProbeChains; ++i) dmma_8x8x4(c[i][0], c[i][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kProbeChains; ++i) s += c[i][0] + c[i][1];
  sink[(blockIdx.x * kProbeThreads + threadIdx.x) & 8191] = s;
}

cudaError_t launch_probe_fp64_mma(double* sink, int iters, double* flops, cudaStream_t stream) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaError_t err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  const int blocks = 4 * sms;
  probe_fp64_mma_kernel<<<blocks, kProbeThreads, 0, stream>>>(sink, iters);
  const double warps = (double)blocks * (kProbeThreads / 32);
  *flops = warps * iters * kProbeUnroll * kProbeChains * (2.0 * 8 * 8 * 4);
  return cudaGetLastError();
}

}  // namespace ssn
