// ssn_ozaki.cu -- split-precision (INT8 Ozaki) products on the tcgen05 tensor cores.
//
// The contraction kernels here compute FP64 products exactly enough for the
// dual Newton solve from INT8 digit slices: every FP64 operand row (or
// column) is scaled by a power of two and written as S signed 7-bit digits,
// the digit products are accumulated exactly in INT32 TMEM accumulators by
// tcgen05.mma kind::i8, and the levels s + t <= S + 1 are recombined in FP64.
//
// This file starts with the single-CTA INT8 MMA used to check the descriptor,
// TMEM and completion plumbing bit for bit against an integer reference.
#include <cuda_runtime.h>

#include "ssn_internal.h"
#include "ssn_tc.cuh"

namespace ssn {

namespace {

constexpr int kProbeThreadsS8 = 128;   // four warps: one per TMEM lane quarter

// C[128 x n] = A[128 x k] * B[n x k]^T, all row-major, int8 in, int32 out.
__global__ void __launch_bounds__(kProbeThreadsS8)
probe_s8_mma_kernel(const int8_t* __restrict__ A, const int8_t* __restrict__ B, int32_t* __restrict__ C,
                    int n, int k, int* __restrict__ stall) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t done;
  __shared__ uint32_t tmem_slot;
  uint8_t* sA = smem;
  uint8_t* sB = smem + 128 * k;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int chunks_per_row = k >> 4;

  for (int c = tid; c < 128 * chunks_per_row; c += kProbeThreadsS8) {
    const int r = c / chunks_per_row, kc = c - r * chunks_per_row;
    const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)r * k + kc * 16);
    *reinterpret_cast<uint4*>(sA + tc::core_offset(r, kc * 16, k)) = v;
  }
  for (int c = tid; c < n * chunks_per_row; c += kProbeThreadsS8) {
    const int r = c / chunks_per_row, kc = c - r * chunks_per_row;
    const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)r * k + kc * 16);
    *reinterpret_cast<uint4*>(sB + tc::core_offset(r, kc * 16, k)) = v;
  }
  const uint32_t ncols = tc::tmem_cols_for(n);
  if (tid == 0) tc::mbar_init(&done, 1);
  __syncwarp();
  if (warp == 0) tc::tmem_alloc(&tmem_slot, ncols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;

  if (tid == 0) {
    const uint32_t sbo = (uint32_t)chunks_per_row * tc::kCoreBytes;
    const uint32_t idesc = tc::idesc_s8(128, n);
    const uint32_t a0 = tc::smem_addr(sA), b0 = tc::smem_addr(sB);
    for (int s = 0; s < k / tc::kStepK; ++s)
      tc::mma_s8(tmem, tc::desc_kmajor(a0 + 256u * s, tc::kCoreBytes, sbo),
                 tc::desc_kmajor(b0 + 256u * s, tc::kCoreBytes, sbo), idesc, s > 0);
    tc::commit(&done);
  }
  __syncwarp();
  bool ok = tc::mbar_wait(&done, 0, tc::kWaitPolls);
  tc::fence_after_sync();
  if (ok) {
    const int row = warp * 32 + lane;
    for (int col = 0; col < n; col += 8) {
      uint32_t r[8];
      tc::tmem_ld8(tc::tmem_at(tmem, warp * 32, col), r);
      tc::tmem_wait8(r);
#pragma unroll
      for (int j = 0; j < 8; ++j) C[(size_t)row * n + col + j] = static_cast<int32_t>(r[j]);
    }
  } else {
    atomicExch(stall, 1);
    ok = tc::mbar_wait(&done, 0, tc::kWaitPolls);   // let the MMAs drain before TMEM is freed
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

}  // namespace

size_t probe_s8_mma_smem(int n, int k) { return (size_t)(128 + n) * k; }

cudaError_t launch_probe_s8_mma(const int8_t* A, const int8_t* B, int32_t* C, int n, int k, int* stall,
                                cudaStream_t stream) {
  const size_t smem = probe_s8_mma_smem(n, k);
  cudaError_t err = cudaFuncSetAttribute(probe_s8_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
  if (err != cudaSuccess) return err;
  probe_s8_mma_kernel<<<1, kProbeThreadsS8, smem, stream>>>(A, B, C, n, k, stall);
  return cudaGetLastError();
}

}  // namespace ssn
