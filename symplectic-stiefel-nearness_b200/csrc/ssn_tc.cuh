// Fifth-generation tensor-core (tcgen05) primitives for sm_100a, written as
// inline PTX: shared-memory matrix descriptors, the INT8 MMA with a TMEM
// accumulator, TMEM allocation and loads, mbarrier completion with a bounded
// wait, and the proxy / tcgen05 ordering fences.
//
// Operand layout used throughout: K-major, no swizzle.  A "core matrix" is
// 8 rows x 16 bytes stored contiguously (row r of the core matrix at byte
// 16 r).  An operand of R rows and K bytes is stored as core matrices
// (g, c) for row group g = r / 8 and K chunk c = k / 16 at byte offset
// (g * (K / 16) + c) * 128.  In the descriptor, the leading byte offset is
// the distance between K-adjacent core matrices (128) and the stride byte
// offset the distance between 8-row groups (K / 16 * 128).  One INT8 MMA
// consumes 32 bytes of K, i.e. two K-adjacent core matrices, so the start
// address of K step s is base + 256 s.
#pragma once

#include <cstdint>

namespace ssn {
namespace tc {

constexpr int kCoreBytes = 128;     // 8 rows x 16 bytes
constexpr int kStepK = 32;          // K bytes per kind::i8 MMA

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) of a K-major operand with kbytes bytes per row.
__host__ __device__ __forceinline__ int core_offset(int r, int k, int kbytes) {
  return ((r >> 3) * (kbytes >> 4) + (k >> 4)) * kCoreBytes + (r & 7) * 16 + (k & 15);
}

// Shared-memory matrix descriptor, sm100 format (version 1), K-major, no swizzle.
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu)
       | (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16)
       | (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32)
       | (1ull << 46);
}

// Instruction descriptor of kind::i8: signed INT8 A and B, both K-major, S32 accumulator.
__host__ __device__ constexpr uint32_t idesc_s8(int M, int N) {
  return (2u << 4)                                 // D format S32
       | (1u << 7)                                 // A format signed INT8
       | (1u << 10)                                // B format signed INT8
       | (static_cast<uint32_t>(N >> 3) << 17)
       | (static_cast<uint32_t>(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T over one 32-byte K step; issued by one thread.
__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t"
      "}\n"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on the mbarrier when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_addr(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(done) : "r"(smem_addr(mbar)), "r"(parity) : "memory");
  return done != 0;
}

// Poll the phase with the given parity at most `limit` times (each poll is itself
// time-limited by the hardware).  Returns false if the phase never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

// Whole-warp TMEM allocation; the column base is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_addr(slot)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Make this thread's generic-proxy shared-memory writes visible to the tensor core.
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Plain arrive (count 1) on the mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_addr(mbar)) : "memory");
}

// Arrive once on the mbarrier and add `bytes` to the transaction count its phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(mbar)), "r"(bytes)
               : "memory");
}

// Bulk (non-tensor) asynchronous copy of `bytes` contiguous bytes from global to this CTA's
// shared memory, completing as transactions on the mbarrier.  dst, src 16-byte aligned,
// bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mbar)) : "memory");
}

// Bulk (non-tensor) asynchronous copy of `bytes` contiguous bytes from this CTA's shared
// memory to global memory, tracked in the issuing thread's bulk group.  dst, src 16-byte
// aligned, bytes a multiple of 16.  The source must be made visible to the async proxy
// (fence_smem_to_async by the writing threads, then a barrier) before the copy is issued.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               :: "l"(dst), "r"(smem_addr(src)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until this thread's bulk groups have read their shared-memory sources.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Wait until this thread's bulk groups are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Barrier `id` (1..15) over `nthreads` threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}

// TMEM address of (lane, column).
__device__ __forceinline__ uint32_t tmem_at(uint32_t base, int lane, int col) {
  return base + (static_cast<uint32_t>(lane) << 16) + static_cast<uint32_t>(col);
}

// Warp-collective load of 32 lanes x 8 consecutive 32-bit columns: thread t gets
// lane (lane base of the address) + t.  The values are valid after tmem_wait8.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
                 "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

// Wait for this thread's TMEM loads; the registers are threaded through so that
// no use of them can be scheduled before the wait.
__device__ __forceinline__ void tmem_wait8(uint32_t (&r)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]),
                 "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
               :: "memory");
}

// Smallest power-of-two TMEM allocation (>= 32 columns) holding `cols` columns.
__host__ __device__ constexpr uint32_t tmem_cols_for(int cols) {
  return cols <= 32 ? 32u : cols <= 64 ? 64u : cols <= 128 ? 128u : cols <= 256 ? 256u : 512u;
}

constexpr uint32_t kWaitPolls = 1u << 22;   // bound on mbarrier polls before a kernel reports a stall

}  // namespace tc
}  // namespace ssn
