// ssn_ozaki.cu -- split-precision (INT8 Ozaki) products on the tcgen05 tensor cores.
//
// The contraction kernels here compute FP64 products exactly enough for the
// dual Newton solve from INT8 digit slices: every FP64 operand vector is scaled
// by a power of two and written as six balanced 8-bit digits, the digit
// products are accumulated exactly in INT32 TMEM accumulators by tcgen05.mma
// kind::i8, and the levels p + q <= 5 are recombined in FP64.
//
// Digits.  A value x of a vector with scale exponent E (|x| < 2^E for every
// entry of the vector) is written as the integer F = rint(x 2^(46-E)),
// |F| <= 2^46, in six balanced base-256 digits d_0 (most significant) .. d_5,
// each in [-128, 127]: F = sum_i d_i 256^(5-i).  Balanced digits make the
// truncation of the dropped digit products unbiased (plain unsigned low bytes
// make every dropped product positive, and the error then grows with K).
// One FMA does all of it: z = x * 2^(46-E) + (1.5 * 2^52 + C) with
// C = sum_i 128 * 256^i rounds x 2^(46-E) to the integer F and leaves F + C in
// the low 48 mantissa bits of z; byte (5-i) of F + C, XOR 0x80, is d_i.
//
// Products keep the digit pairs with p + q <= 5 (21 of 36), accumulated per
// level l = p + q in its own INT32 TMEM accumulator (exact: 6 pairs x 2^14 x K
// < 2^31 for K < 21845), and recombined in FP64 as
//     sum_l 256^(10-l) acc_l * 2^(E_a - 46) * 2^(E_b - 46).
//
// This file starts with the single-CTA INT8 MMA used to check the descriptor,
// TMEM and completion plumbing bit for bit against an integer reference.
#include <cuda_runtime.h>

#include "ssn_common.cuh"
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

// ============================================================== Ozaki digits
namespace oz {

constexpr int kDigits = 6;
constexpr int kFrac = 8 * kDigits - 2;              // 46
constexpr int kExpNonFinite = 4096;                 // exponent code of a vector with Inf / NaN
constexpr int kExpMin = -960;                       // 2^(kFrac - E) stays finite
constexpr double kMagic = 6755399441055744.0 + 141289400074368.0;   // 1.5 * 2^52 + 0x808080808080

// Exponent E with max < 2^E from the bit pattern of max |x| (sign bit clear).
__host__ __device__ __forceinline__ int exp_of_maxbits(unsigned long long bits) {
  if (bits >= 0x7FF0000000000000ull) return kExpNonFinite;
  if (bits == 0ull) return kExpMin;
  const int eb = static_cast<int>(bits >> 52);
  const int e = (eb > 0 ? eb : 1) - 1022;
  return e < kExpMin ? kExpMin : e;
}

__device__ __forceinline__ double pow2(int e) {   // exact 2^e for -1022 <= e <= 1023
  return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}

__device__ __forceinline__ unsigned long long abs_bits(double x) {
  return static_cast<unsigned long long>(__double_as_longlong(x)) & 0x7FFFFFFFFFFFFFFFull;
}

// Digit words of four values sharing the scale sc = 2^(kFrac - E): w[i] holds
// digit i of x[0..3] in bytes 0..3 (K-contiguous rows of a K-major operand).
__device__ __forceinline__ void slice4(const double (&x)[4], double sc, uint32_t (&w)[kDigits]) {
  uint32_t lo[4], hi[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double z = fma(x[q], sc, kMagic);
    lo[q] = static_cast<uint32_t>(__double2loint(z));
    hi[q] = static_cast<uint32_t>(__double2hiint(z));
  }
  // 4 x 4 byte transpose of lo, 4 x 2 of the low half of hi
  const uint32_t t0 = __byte_perm(lo[0], lo[1], 0x5140), t1 = __byte_perm(lo[0], lo[1], 0x7362);
  const uint32_t t2 = __byte_perm(lo[2], lo[3], 0x5140), t3 = __byte_perm(lo[2], lo[3], 0x7362);
  const uint32_t t4 = __byte_perm(hi[0], hi[1], 0x5140), t5 = __byte_perm(hi[2], hi[3], 0x5140);
  w[5] = __byte_perm(t0, t2, 0x5410) ^ 0x80808080u;   // byte 0 of F + C
  w[4] = __byte_perm(t0, t2, 0x7632) ^ 0x80808080u;   // byte 1
  w[3] = __byte_perm(t1, t3, 0x5410) ^ 0x80808080u;   // byte 2
  w[2] = __byte_perm(t1, t3, 0x7632) ^ 0x80808080u;   // byte 3
  w[1] = __byte_perm(t4, t5, 0x5410) ^ 0x80808080u;   // byte 4
  w[0] = __byte_perm(t4, t5, 0x7632) ^ 0x80808080u;   // byte 5 (most significant digit)
}

// An INT32 accumulator as a double, exactly: 2^52 + 2^31 + a has a + 2^31 as its low
// word, so one XOR builds it and one subtraction removes the offset (an FP64 add
// instead of an integer-to-FP64 conversion).
__device__ __forceinline__ double i32_to_f64(uint32_t a) {
  return __hiloint2double(0x43300000, static_cast<int>(a ^ 0x80000000u)) - 4503601774854144.0;
}

// sum_l 256^(5-l) acc_l (Horner), the digit-level recombination before scaling.
__device__ __forceinline__ double horner6(const uint32_t (&a)[kDigits]) {
  double v = i32_to_f64(a[0]);
#pragma unroll
  for (int l = 1; l < kDigits; ++l) v = fma(v, 256.0, i32_to_f64(a[l]));
  return v;
}

}  // namespace oz

// ============================================================== Ozaki Gram
//
// Cr = A^T A + D^T D and G = A^T D over row chunks of n: one CTA per (row chunk,
// group of 32 output columns, instance).  The MMA's M = 128 rows are the m
// columns of T (zero-padded), N = 32 the CTA's output columns, K the rows of
// the chunk, streamed in sub-tiles of 32 rows of A and 32 rows of D.  One warp
// bulk-copies the FP64 rows of each sub-tile into a ring of up to three stages;
// sixteen slicing warps turn a stage into digit planes (K-major, 64 K bytes per
// operand row: A rows then D rows) in one of two digit stages; one thread
// issues the sub-tile's 21 digit pairs x {A^T A, D^T D, A^T D} as 18 MMAs with
// stacked B digits into 12 TMEM accumulators (6 levels x {Cr, G}, 32 columns
// each) and commits them to the digit stage's mbarrier, which frees it.
// Column scales are per (chunk, column), shared by A and D so that Cr's two
// halves can share accumulators; a pre-pass computes them (and the per-row
// scales the recovery uses).  Partials go to [B][chunk][2][m][m] and are summed
// in fixed order by the FP64 Gram's finalize kernel.
namespace {

constexpr int kScaleThreads = 256;
constexpr int kScaleRows = 64;                 // rows of A and D per pre-pass block

// Pre-pass: per-(chunk, column) max |x| over the rows of A and D in the chunk (as
// bit patterns, atomicMax into a zeroed array; max is order-independent; skipped
// when col_bits is null) and the per-row scale exponent of [A_r | D_r] for the
// recovery (skipped when row_exp is null).
__global__ void __launch_bounds__(kScaleThreads)
    ozaki_scale_kernel(const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride, int rows,
                       int m, int chunk, int nchunks, unsigned long long* __restrict__ col_bits,
                       int32_t* __restrict__ row_exp) {
  __shared__ unsigned long long cmax[kScaleThreads / 32][kMaxM];
  const int b = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = blockIdx.x * kScaleRows, r1 = imin(rows, r0 + kScaleRows);
  const double* Ab = A + (size_t)b * ab_stride;
  const double* Db = D + (size_t)b * ab_stride;
  unsigned long long cm[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll 2
  for (int r = r0 + warp; r < r1; r += kScaleThreads / 32) {
    unsigned long long rm = 0ull;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int col = 2 * lane + 64 * hh;
      if (col < m) {
        const double2 a = *reinterpret_cast<const double2*>(Ab + (size_t)r * m + col);
        const double2 d = *reinterpret_cast<const double2*>(Db + (size_t)r * m + col);
        const unsigned long long c0 = max(oz::abs_bits(a.x), oz::abs_bits(d.x));
        const unsigned long long c1 = max(oz::abs_bits(a.y), oz::abs_bits(d.y));
        cm[2 * hh] = max(cm[2 * hh], c0);
        cm[2 * hh + 1] = max(cm[2 * hh + 1], c1);
        rm = max(rm, max(c0, c1));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rm = max(rm, __shfl_xor_sync(0xffffffffu, rm, o));
    if (lane == 0 && row_exp) row_exp[(size_t)b * rows + r] = oz::exp_of_maxbits(rm);
  }
#pragma unroll
  for (int hh = 0; hh < 2; ++hh) {
    const int col = 2 * lane + 64 * hh;
    if (col < m) {
      cmax[warp][col] = cm[2 * hh];
      cmax[warp][col + 1] = cm[2 * hh + 1];
    }
  }
  __syncthreads();
  const int c = r0 / chunk;        // pre-pass blocks never straddle a chunk (chunk % kScaleRows == 0)
  if (col_bits)
    for (int j = threadIdx.x; j < m; j += kScaleThreads) {
      unsigned long long mx = 0ull;
      for (int w = 0; w < kScaleThreads / 32; ++w) mx = max(mx, cmax[w][j]);
      atomicMax(&col_bits[((size_t)b * nchunks + c) * m + j], mx);
    }
}

// Warp roles.  All slicing warps work on every sub-tile in order, so every
// waiter sees every phase of the mbarriers it waits on: a parity wait is only
// unambiguous when the waiter has observed the previous phase (a consumer that
// skipped phases could see a parity match one phase early).
constexpr int kGSliceWarps = 16;
constexpr int kGSlicers = kGSliceWarps * 32;
constexpr int kGMmaWarp = kGSliceWarps;                    // warp 16: MMA issuer
constexpr int kGLoadWarp = kGSliceWarps + 1;               // warp 17: TMA producer
constexpr int kGThreads = kGSlicers + 64;
constexpr int kGSub = 32;                                  // rows of A (and of D) per sub-tile
constexpr int kGN = 32;                                    // output columns per CTA (MMA N)
constexpr int kGM = 128;                                   // MMA M: operand rows read from a digit plane
constexpr int kGKBytes = 2 * kGSub;                        // K bytes per operand row of one digit plane
constexpr int kGDStages = 2;                               // digit-plane stages
constexpr int kGFStagesMax = 3;                            // FP64 staging stages (TMA bulk copies)
constexpr int kGSmemMax = 227 * 1024 - 2304;               // opt-in limit minus the static shared memory
constexpr uint32_t kGTmemCols = 512;                       // 2 x 6 x 32 = 384 used
constexpr uint32_t kGSbo = (kGKBytes / 16) * tc::kCoreBytes;   // 512: 8-row group stride

// Shared-memory plan of the Gram kernel for m columns.  Digit planes are packed
// at mp16 rows; the M = 128 rows an MMA reads from plane p may run into plane
// p + 1 (those output rows are never read), so only the last plane is padded
// to 128 rows.  FP64 stages hold 32 rows of A then 32 rows of D.
struct GramSmem {
  int plane, bstack, dstage, fstage, fstages, total;
};
constexpr int kGBStack = oz::kDigits * kGN * kGKBytes;    // 12288: digits 0..5 of the CTA's 32 columns
__host__ __device__ inline GramSmem gram_smem(int m) {
  GramSmem g;
  const int mp16 = round_up(m, 16);
  g.plane = mp16 * kGKBytes;
  g.bstack = (oz::kDigits - 1) * g.plane + kGM * kGKBytes;   // B copy follows the A planes of a stage
  g.dstage = g.bstack + kGBStack;
  g.fstage = 2 * kGSub * m * 8;
  g.fstages = (kGSmemMax - kGDStages * g.dstage) / g.fstage;
  if (g.fstages > kGFStagesMax) g.fstages = kGFStagesMax;
  g.total = kGDStages * g.dstage + g.fstages * g.fstage;
  return g;
}

// The MMAs of one sub-tile.  For a fixed digit p of the A operand (all m columns), the
// B operand is the stack of digits q = 0 .. 5 - p of the CTA's 32 output columns
// (rows 32 q + jj of the B copy), so one MMA with N = (6 - p) 32 adds every pair
// (p, q) into the level accumulators p + q, which lie at TMEM columns 32 (p + q):
// contiguous from 32 p.  Per p: A^T A and D^T D (Cr) and A^T D (G); 18 MMAs.
template <int P>
struct GramStack {
  __device__ __forceinline__ static void issue(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t plane16,
                                               bool first_tile) {
    constexpr int N = (oz::kDigits - P) * kGN;
    constexpr uint32_t idesc = tc::idesc_s8(kGM, N);
    const uint64_t da = adesc + (uint64_t)(P * plane16);
    constexpr uint32_t col = (uint32_t)P * kGN;
    const uint32_t acc = (!first_tile || P > 0) ? 1u : 0u;
    tc::mma_s8(tmem + col, da, bdesc, idesc, acc);                                 // A^T A
    tc::mma_s8(tmem + col, da + 16, bdesc + 16, idesc, 1u);                        // + D^T D (K bytes 32..63)
    tc::mma_s8(tmem + oz::kDigits * kGN + col, da, bdesc + 16, idesc, acc);        // A^T D
    if constexpr (P + 1 < oz::kDigits) GramStack<P + 1>::issue(tmem, adesc, bdesc, plane16, first_tile);
  }
};

__global__ void __launch_bounds__(kGThreads, 1)
    ozaki_gram_kernel(const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride, int rows,
                      int m, int chunk, int nchunks, int ncg, const unsigned long long* __restrict__ col_bits,
                      double* __restrict__ partial, int* __restrict__ stall) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar_full[kGFStagesMax];     // TMA -> slicers (transaction bytes)
  __shared__ uint64_t bar_ffree[kGFStagesMax];    // slicers -> producer: FP64 stage consumed
  __shared__ uint64_t bar_ready[kGDStages];       // slicers -> MMA issuer: digit planes written
  __shared__ uint64_t bar_dfree[kGDStages];       // MMA commit -> slicers: digit planes consumed
  __shared__ uint32_t tmem_slot;
  __shared__ int s_err;
  __shared__ double s_sc[kMaxM];      // slicing scale 2^(46 - E_j)
  __shared__ double s_inv[kMaxM];     // recombination scale 2^(E_j - 26)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = blockIdx.x / ncg, h = blockIdx.x - c * ncg, b = blockIdx.y;
  const int r0 = c * chunk, r1 = imin(rows, r0 + chunk);
  const int nsub = cdiv(r1 - r0, kGSub);
  const int mp16 = round_up(m, 16);
  const GramSmem L = gram_smem(m);
  // slicing warps that work: the fewest of 8, 12, 16 that take the sub-tile's tasks (16 columns
  // x 2 row octets each) in as few rounds as 16 would, so every working warp has as many tasks
  // (m = 96: 24 tasks, 12 warps x 2 rather than 16 warps x 1 or 2)
  const int ntask_all = (mp16 / 16) * 4;
  const int rounds16 = cdiv(ntask_all, kGSliceWarps);
  const int nsl = cdiv(ntask_all, 8) == rounds16 ? 8 : cdiv(ntask_all, 12) == rounds16 ? 12 : kGSliceWarps;
  const double* Ab = A + (size_t)b * ab_stride;
  const double* Db = D + (size_t)b * ab_stride;
  uint8_t* dbase = smem;
  uint8_t* fbase = smem + kGDStages * L.dstage;

  // zero the digit stages once: rows >= mp16 of the last plane are read by the MMA, never written
  for (int i = tid * 16; i < kGDStages * L.dstage; i += kGThreads * 16)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0, 0, 0, 0);
  bool bad = false;
  if (tid < kMaxM) {
    int e = oz::kExpMin;
    if (tid < m) e = oz::exp_of_maxbits(col_bits[((size_t)b * nchunks + c) * m + tid]);
    bad = e == oz::kExpNonFinite;
    if (bad) e = 0;
    s_sc[tid] = oz::pow2(oz::kFrac - e);
    s_inv[tid] = oz::pow2(e - 26);
  }
  if (tid == 0) {
    for (int s = 0; s < kGFStagesMax; ++s) {
      tc::mbar_init(&bar_full[s], 1);
      tc::mbar_init(&bar_ffree[s], nsl);
    }
    for (int s = 0; s < kGDStages; ++s) {
      tc::mbar_init(&bar_ready[s], nsl);
      tc::mbar_init(&bar_dfree[s], 1);
    }
    s_err = 0;
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, kGTmemCols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  bad = __syncthreads_or(bad) != 0;
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;

  if (!bad) {
    if (warp == kGLoadWarp) {
      // ---- TMA producer: FP64 rows of sub-tile t of A and D into FP64 stage t % fstages
      if (lane == 0) {
        bool ok = true;
        for (int t = 0; t < nsub && ok; ++t) {
          const int f = t % L.fstages;
          if (t >= L.fstages) ok = tc::mbar_wait(&bar_ffree[f], ((t / L.fstages) - 1) & 1, tc::kWaitPolls);
          if (!ok || *reinterpret_cast<volatile int*>(&s_err)) break;
          const int rs = r0 + t * kGSub;
          const uint32_t bytes = (uint32_t)(imin(kGSub, r1 - rs) * m * 8);
          uint8_t* dst = fbase + f * L.fstage;
          tc::mbar_arrive_expect_tx(&bar_full[f], 2 * bytes);
          tc::bulk_g2s(dst, Ab + (size_t)rs * m, bytes, &bar_full[f]);
          tc::bulk_g2s(dst + kGSub * m * 8, Db + (size_t)rs * m, bytes, &bar_full[f]);
        }
        if (!ok) atomicExch(&s_err, 1);
      }
    } else if (warp == kGMmaWarp) {
      // ---- MMA issuer: the 63 MMAs of each sub-tile once its digit planes are written
      if (lane == 0) {
        const uint32_t plane16 = (uint32_t)L.plane >> 4;
        bool ok = true;
        for (int t = 0; t < nsub && ok; ++t) {
          const int d = t % kGDStages;
          ok = tc::mbar_wait(&bar_ready[d], (t / kGDStages) & 1, tc::kWaitPolls);
          if (!ok) break;
          tc::fence_after_sync();
          const uint32_t sbase = tc::smem_addr(dbase + d * L.dstage);
          const uint64_t adesc = tc::desc_kmajor(sbase, tc::kCoreBytes, kGSbo);
          const uint64_t bdesc = tc::desc_kmajor(sbase + (uint32_t)L.bstack, tc::kCoreBytes, kGSbo);
          GramStack<0>::issue(tmem, adesc, bdesc, plane16, t == 0);
          tc::commit(&bar_dfree[d]);
        }
        if (ok && nsub > 0) {
          const int tl = nsub - 1;
          ok = tc::mbar_wait(&bar_dfree[tl % kGDStages], (tl / kGDStages) & 1, tc::kWaitPolls);
        }
        if (!ok) atomicExch(&s_err, 1);
      }
    } else if (warp < nsl) {
      // ---- slicing warps: every sub-tile, FP64 stage -> digit planes and the stacked B copy
      const int ntask = (mp16 / 16) * 4;                  // warp tasks: 16 columns x 2 row octets
      for (int t = 0; t < nsub; ++t) {
        const int d = t % kGDStages, f = t % L.fstages;
        bool ok = tc::mbar_wait(&bar_full[f], (t / L.fstages) & 1, tc::kWaitPolls);
        if (ok && t >= kGDStages) ok = tc::mbar_wait(&bar_dfree[d], ((t / kGDStages) - 1) & 1, tc::kWaitPolls);
        if (!ok || *reinterpret_cast<volatile int*>(&s_err)) {
          atomicExch(&s_err, 1);
          break;
        }
        uint8_t* stage = dbase + d * L.dstage;
        const double* fs = reinterpret_cast<const double*>(fbase + f * L.fstage);
        const int nr = imin(kGSub, r1 - (r0 + t * kGSub));
        for (int g = warp; g < ntask; g += nsl) {
          // lane -> (column, K octet) so that every half-warp reads 16 distinct columns of a
          // staged row (conflict-free 8-byte loads) and writes 16 distinct bank pairs of the
          // digit planes (conflict-free 8-byte stores): lanes 8-15 take the upper 8 columns
          // of the odd octet, lanes 16-23 the upper 8 of the even one.
          const int jg = g % (mp16 / 16), kg = g / (mp16 / 16);
          const int j = jg * 16 + (lane & 7) + 8 * (((lane >> 3) ^ (lane >> 4)) & 1);
          const int k8 = kg * 2 + ((lane >> 3) & 1);      // K octet: 0..3 rows of A, 4..7 rows of D
          const int rq = (k8 & 3) * 8;
          const double* src = fs + (size_t)((k8 >> 2) * kGSub + rq) * m + j;
          double x0[4], x1[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            x0[q] = (j < m && rq + q < nr) ? src[(size_t)q * m] : 0.0;
            x1[q] = (j < m && rq + 4 + q < nr) ? src[(size_t)(q + 4) * m] : 0.0;
          }
          uint32_t w0[oz::kDigits], w1[oz::kDigits];
          oz::slice4(x0, s_sc[j], w0);
          oz::slice4(x1, s_sc[j], w1);
          const int off = tc::core_offset(j, k8 * 8, kGKBytes);
#pragma unroll
          for (int i = 0; i < oz::kDigits; ++i)
            *reinterpret_cast<uint2*>(stage + i * L.plane + off) = make_uint2(w0[i], w1[i]);
          const int jj = j - h * kGN;
          if (jj >= 0 && jj < kGN) {                      // the CTA's own columns: the stacked B copy
#pragma unroll
            for (int i = 0; i < oz::kDigits; ++i)
              *reinterpret_cast<uint2*>(stage + L.bstack + tc::core_offset(i * kGN + jj, k8 * 8, kGKBytes)) =
                  make_uint2(w0[i], w1[i]);
          }
        }
        tc::fence_smem_to_async();
        __syncwarp();
        if (lane == 0) {
          tc::mbar_arrive(&bar_ffree[f]);
          tc::mbar_arrive(&bar_ready[d]);
        }
      }
    }
  }

  // readout: warp w < 8 reads TMEM lanes 32 (w & 3) .. + 31 (output rows) of output w >> 2 (Cr, G)
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const bool ok = s_err == 0;
  if (warp < 8) {
    const int quarter = warp & 3, out = warp >> 2;
    const int i = quarter * 32 + lane;
    double* dst = partial + (((size_t)b * nchunks + c) * 2 + out) * (size_t)m * m;
    const uint32_t tbase = tc::tmem_at(tmem, quarter * 32, out * oz::kDigits * kGN);
    for (int jc = 0; jc < kGN; jc += 8) {
      uint32_t r[oz::kDigits][8];
      if (!bad && ok) {
#pragma unroll
        for (int l = 0; l < oz::kDigits; ++l) tc::tmem_ld8(tbase + l * kGN + jc, r[l]);
#pragma unroll
        for (int l = 0; l < oz::kDigits; ++l) tc::tmem_wait8(r[l]);
      }
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int col = h * kGN + jc + jj;
        if (i < m && col < m) {
          double v = __longlong_as_double(0x7FF8000000000000ll);   // NaN: non-finite input or a stall
          if (!bad && ok) {
            uint32_t a[oz::kDigits];
#pragma unroll
            for (int l = 0; l < oz::kDigits; ++l) a[l] = r[l][jj];
            v = oz::horner6(a) * s_inv[i] * s_inv[col];
          }
          dst[(size_t)i * m + col] = v;
        }
      }
    }
  }
  if (!ok && !bad) {
    if (tid == 0) atomicExch(stall, 1);
    // drain: let committed MMAs and issued copies finish before TMEM and shared memory are released
    if (tid == 0) {
      for (int s = 0; s < kGDStages; ++s) (void)tc::mbar_wait(&bar_dfree[s], 0, tc::kWaitPolls);
      for (int s = 0; s < L.fstages; ++s) (void)tc::mbar_wait(&bar_full[s], 0, tc::kWaitPolls);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, kGTmemCols);
}

struct OzGramPlan {
  int chunk, nchunks, ncg;
};

int sm_count_oz() { return current_device_sm_count(); }

// Row chunks per instance: the count minimising waves x chunk length (one CTA per
// SM), chunks a multiple of the pre-pass block and short enough for exact INT32.
OzGramPlan oz_gram_plan(int batch, int rows, int m) {
  const int sms = sm_count_oz();
  const int ncg = cdiv(m, kGN);
  const int max_chunk = 8192;                     // K = 2 chunk rows: 6 x 2^14 x 2 x 8192 < 2^31
  int best = 1;
  double best_cost = 1e300;
  for (int nc = 1; nc <= 32; ++nc) {
    const int chunk = round_up(cdiv(rows, nc), kScaleRows);
    if (chunk > max_chunk) continue;
    const int used = cdiv(rows, chunk);
    const long long ctas = (long long)batch * used * ncg;
    const double cost = (double)((ctas + sms - 1) / sms) * chunk * (1.0 + 0.01 * used);
    if (cost < best_cost) {
      best_cost = cost;
      best = nc;
    }
  }
  const ssn_tuning* tune = active_tuning();
  if (tune && tune->gram_chunks > 0 && round_up(cdiv(rows, tune->gram_chunks), kScaleRows) <= max_chunk)
    best = tune->gram_chunks;                     // autotuned
  const int chunk = round_up(cdiv(rows, best), kScaleRows);
  return OzGramPlan{chunk, cdiv(rows, chunk), ncg};
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

size_t ozaki_gram_workspace_bytes(int batch, int rows, int m) {
  const OzGramPlan pl = oz_gram_plan(batch, rows, m);
  return align256(sizeof(double) * (size_t)batch * pl.nchunks * 2 * m * m) +
         align256(sizeof(unsigned long long) * (size_t)batch * pl.nchunks * m);
}

cudaError_t launch_gram_ozaki(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                              int batch, int rows, int m, void* workspace, int32_t* row_exp, int* stall,
                              cudaStream_t stream) {
  const OzGramPlan pl = oz_gram_plan(batch, rows, m);
  double* partial = static_cast<double*>(workspace);
  unsigned long long* col_bits = reinterpret_cast<unsigned long long*>(
      static_cast<char*>(workspace) + align256(sizeof(double) * (size_t)batch * pl.nchunks * 2 * m * m));
  cudaError_t err = cudaMemsetAsync(col_bits, 0, sizeof(unsigned long long) * (size_t)batch * pl.nchunks * m, stream);
  if (err != cudaSuccess) return err;
  ozaki_scale_kernel<<<dim3(cdiv(rows, kScaleRows), batch), kScaleThreads, 0, stream>>>(
      A, D, ab_stride, rows, m, pl.chunk, pl.nchunks, col_bits, row_exp);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const int smem = gram_smem(m).total;
  err = cudaFuncSetAttribute(ozaki_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return err;
  ozaki_gram_kernel<<<dim3(pl.nchunks * pl.ncg, batch), kGThreads, smem, stream>>>(
      A, D, ab_stride, rows, m, pl.chunk, pl.nchunks, pl.ncg, col_bits, partial, stall);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  return launch_gram_finalize(partial, Cr, Ci, batch, m, pl.nchunks, stream);
}

// ============================================================== Ozaki recovery
//
// X = [A P^T + D Q^T ; D P^T - A Q^T].  With W_r = [A_r | D_r] (K = 2m) every
// entry is R[r, o] = sum_c W[r, c] B[o, c] for the 2m output columns o (Ur then
// Ui) with B rows [P_o | Q_o] (o < m) and [-Q_o' | P_o'] (o' = o - m); per-row
// scales on both sides (W rows from the Gram pre-pass, B rows from the prep
// kernel), six digits each, so X is accurate to about 2^-46 of each row's
// largest contribution.
//
// One CTA per (instance, group of 64 output columns, part of the row tiles),
// persistent over its tiles: MMA M = a 128-row tile, N = stacked digits of the
// group's 64 B rows, K = 2m in 32-byte steps.  The prep kernel slices B once per
// (instance, group) into the stacked, step-major layout the CTA bulk-loads in
// one copy; the W digits, made once by the W-digit kernel in the same layout,
// arrive one 24 KB bulk copy per (tile, K step) into a ring of up to four
// stages; the MMA warp runs a tile's steps once the eight epilogue warps have
// drained the previous tile's accumulators (six levels of 64 columns: 384 TMEM
// columns).
namespace {

constexpr int kRM = 128;                                  // rows per tile (MMA M)
constexpr int kRW = 64;                                   // output columns per CTA
constexpr int kRK = 32;                                   // K bytes per step
constexpr int kRPlane = kRM * kRK;                        // 4096: one digit plane of a step
constexpr int kRAStage = oz::kDigits * kRPlane;           // 24576: the six A planes of a step
constexpr int kRBStep = oz::kDigits * kRW * kRK;          // 12288: stacked B digits of a step
constexpr int kRStagesMax = 4;                            // digit-plane stages (bulk copies of W digits)
constexpr int kRMmaWarp = 0;                              // warp 0: MMA issuer (lane 0), TMEM allocator
constexpr int kRLoadWarp = 1;                             // warp 1: bulk copies of the W digit steps
constexpr int kREpiWarp0 = 4;                             // warps 4-19: epilogue, TMEM lane quarter = warp % 4
constexpr int kREpiWarps = 16;                            // four per lane quarter, one per 16-column quarter
constexpr int kRThreads = (kREpiWarp0 + kREpiWarps) * 32;
constexpr int kRSmemMax = 227 * 1024 - 1024;              // opt-in limit minus the static shared memory
constexpr uint32_t kRSbo = (kRK / 16) * tc::kCoreBytes;    // 256
constexpr uint32_t kRTmemCols = 512;                      // 6 x 64 = 384 used

__host__ __device__ inline int rec_groups(int m) { return cdiv(2 * m, kRW); }
__host__ __device__ inline int rec_steps(int m) { return cdiv(2 * m, kRK); }
constexpr int kRStgLd = kRW + 2;                          // staged X row stride (doubles): 528 bytes
constexpr int kRStg = kRM * kRStgLd * 8;                  // 67584: one tile's X, staged for bulk stores
__host__ __device__ inline int rec_stages(int m) {
  const int f = (kRSmemMax - rec_steps(m) * kRBStep - kRStg) / kRAStage;
  return f > kRStagesMax ? kRStagesMax : f;
}
__host__ __device__ inline int rec_smem(int m) {
  return rec_steps(m) * kRBStep + rec_stages(m) * kRAStage + kRStg;
}

// B row o, column c (o < 2m, c < 2m): rows [P_o | Q_o] (Ur), [-Q_o' | P_o'] (Ui).
__device__ __forceinline__ double rec_b(const double* P, const double* Q, int m, int o, int c) {
  if (o < m) return c < m ? P[o * m + c] : Q[o * m + c - m];
  const int oo = o - m;
  return c < m ? -Q[oo * m + c] : P[oo * m + c - m];
}

// One warp per B row: its scale exponent and its six digits, written in the
// stacked step-major layout [instance][group][step][digit q][64 rows][32 K bytes]
// (K-major core matrices), zero outside o < 2m, c < 2m.
__global__ void __launch_bounds__(256)
    ozaki_recover_prep_kernel(const double* __restrict__ P, const double* __restrict__ Q, int m,
                              uint8_t* __restrict__ bdig, int32_t* __restrict__ fexp) {
  // grid.x = group x 8: each CTA (8 warps) handles 8 of the group's 64 B rows
  const int h = blockIdx.x >> 3, b = blockIdx.y, ngrp = gridDim.x >> 3, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nks = rec_steps(m), kpad = nks * kRK;
  const double* Pb = P + (size_t)b * m * m;
  const double* Qb = Q + (size_t)b * m * m;
  uint8_t* out = bdig + ((size_t)b * ngrp + h) * nks * kRBStep;
  {
    const int jj = (blockIdx.x & 7) * 8 + warp;
    const int o = h * kRW + jj;
    unsigned long long mx = 0ull;
    if (o < 2 * m)
      for (int c = lane; c < 2 * m; c += 32) mx = max(mx, oz::abs_bits(rec_b(Pb, Qb, m, o, c)));
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, sh));
    int e = oz::exp_of_maxbits(mx);
    if (lane == 0 && o < 2 * m) fexp[(size_t)b * 2 * m + o] = e;
    if (e == oz::kExpNonFinite) e = 0;
    const double sc = oz::pow2(oz::kFrac - e);
    for (int c = lane; c < kpad; c += 32) {
      const double x = (o < 2 * m && c < 2 * m) ? rec_b(Pb, Qb, m, o, c) : 0.0;
      const double z = fma(x, sc, oz::kMagic);
      const uint32_t lo = static_cast<uint32_t>(__double2loint(z)), hi = static_cast<uint32_t>(__double2hiint(z));
      const int s = c / kRK, k = c - s * kRK;
#pragma unroll
      for (int q = 0; q < oz::kDigits; ++q) {
        const int byte = oz::kDigits - 1 - q;           // digit q is byte 5 - q of F + C
        const uint32_t word = byte < 4 ? lo : hi;
        const uint8_t d = static_cast<uint8_t>(((word >> (8 * (byte & 3))) & 0xFFu) ^ 0x80u);
        out[(size_t)s * kRBStep + tc::core_offset(q * kRW + jj, k, kRK)] = d;
      }
    }
  }
}

// The MMAs of one K step: for digit p of the tile rows, B = stacked digits
// q0 .. q0 + NQ - 1 of the group's 64 rows, accumulated at TMEM columns 64 (p + q0).
template <int P, int Q0, int NQ>
__device__ __forceinline__ void rec_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, bool first) {
  constexpr uint32_t idesc = tc::idesc_s8(kRM, NQ * kRW);
  const uint64_t da = adesc + (uint64_t)((P * kRPlane) >> 4);
  const uint64_t db = bdesc + (uint64_t)((Q0 * (kRW / 8) * kRSbo) >> 4);
  tc::mma_s8(tmem + (uint32_t)(P + Q0) * kRW, da, db, idesc, (first && P == 0) ? 0u : 1u);
}

__device__ __forceinline__ void rec_step_mmas(uint32_t tmem, uint64_t adesc, uint64_t bdesc, bool first) {
  rec_mma<0, 0, 4>(tmem, adesc, bdesc, first);
  rec_mma<0, 4, 2>(tmem, adesc, bdesc, first);
  rec_mma<1, 0, 4>(tmem, adesc, bdesc, first);
  rec_mma<1, 4, 1>(tmem, adesc, bdesc, first);
  rec_mma<2, 0, 4>(tmem, adesc, bdesc, first);
  rec_mma<3, 0, 3>(tmem, adesc, bdesc, first);
  rec_mma<4, 0, 2>(tmem, adesc, bdesc, first);
  rec_mma<5, 0, 1>(tmem, adesc, bdesc, first);
}

// W digits: one warp per row of W = [A_r | D_r]: its scale exponent (max over
// the row) and its six digits, written straight into the MMA layout of the
// recovery: [instance][tile][step][digit q][128 rows][32 K bytes] (K-major core
// matrices, zero beyond c < 2m and r < rows), so each (tile, step) is one
// contiguous 24 KB block.  Lane l handles K octet l (columns 8 l .. 8 l + 7).
__global__ void __launch_bounds__(256)
    ozaki_wdigits_kernel(const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride, int rows,
                         int m, uint8_t* __restrict__ wdig, int32_t* __restrict__ row_exp) {
  const int tile = blockIdx.x, b = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nks = rec_steps(m), ntiles = gridDim.x;
  const double* Ab = A + (size_t)b * ab_stride;
  const double* Db = D + (size_t)b * ab_stride;
  uint8_t* out = wdig + ((size_t)b * ntiles + tile) * nks * kRAStage;
  const int c0 = lane * 8;                             // this lane's K octet
  const bool active = c0 < nks * kRK;                 // octets of the padded K range
  for (int rr = warp; rr < kRM; rr += 8) {
    const int r = tile * kRM + rr;
    double x[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = c0 + 2 * i;                       // m even: a pair never straddles A and D
      double2 v = make_double2(0.0, 0.0);
      if (r < rows && c < 2 * m)
        // streaming (evict-first) loads and stores: this kernel runs beside the Newton
        // kernels, whose operands it would otherwise push out of L2
        v = c < m ? __ldcs(reinterpret_cast<const double2*>(Ab + (size_t)r * m + c))
                  : __ldcs(reinterpret_cast<const double2*>(Db + (size_t)r * m + (c - m)));
      x[2 * i] = v.x;
      x[2 * i + 1] = v.y;
    }
    unsigned long long mx = 0ull;
#pragma unroll
    for (int i = 0; i < 8; ++i) mx = max(mx, oz::abs_bits(x[i]));
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, sh));
    int e = oz::exp_of_maxbits(mx);
    if (lane == 0 && r < rows) row_exp[(size_t)b * rows + r] = e;
    if (e == oz::kExpNonFinite) e = 0;
    if (!active) continue;
    const double sc = oz::pow2(oz::kFrac - e);
    const double x0[4] = {x[0], x[1], x[2], x[3]};
    const double x1[4] = {x[4], x[5], x[6], x[7]};
    uint32_t w0[oz::kDigits], w1[oz::kDigits];
    oz::slice4(x0, sc, w0);
    oz::slice4(x1, sc, w1);
    const int s = c0 / kRK, k = c0 - s * kRK;
    uint8_t* blk = out + (size_t)s * kRAStage + tc::core_offset(rr, k, kRK);
#pragma unroll
    for (int q = 0; q < oz::kDigits; ++q) __stcs(reinterpret_cast<uint2*>(blk + q * kRPlane), make_uint2(w0[q], w1[q]));
  }
}

// Persistent over the row tiles [tile0, tile1) of one (instance, output group):
// the group's B digits are loaded once; warp 1 streams the W digit blocks of
// every (tile, step) into a ring of stages; the MMA thread runs a tile's steps
// once the epilogue has drained the previous tile's accumulators; the epilogue
// warps recombine the levels and store X through a small shared transpose
// (64-byte row segments).
__global__ void __launch_bounds__(kRThreads, 1)
    ozaki_recover_kernel(const uint8_t* __restrict__ wdig, const int32_t* __restrict__ row_exp,
                         const uint8_t* __restrict__ bdig, const int32_t* __restrict__ fexp, double* __restrict__ Ur,
                         double* __restrict__ Ui, int64_t u_stride, int rows, int m, int nparts,
                         int* __restrict__ stall) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar_b;
  __shared__ uint64_t bar_full[kRStagesMax];     // a W digit step landed
  __shared__ uint64_t bar_dfree[kRStagesMax];    // MMAs done with a stage
  __shared__ uint64_t bar_acc_full;              // MMA commit: a tile's accumulators are complete
  __shared__ uint64_t bar_acc_free;              // epilogue: a tile's accumulators have been read
  __shared__ uint32_t tmem_slot;
  __shared__ int s_err;
  __shared__ double s_finv[kRW];                 // 2^(f_o - 26); NaN marks a non-finite B row
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ngrp = rec_groups(m), nks = rec_steps(m), ntiles = cdiv(rows, kRM), nst = rec_stages(m);
  const int part = blockIdx.x % nparts, h = (blockIdx.x / nparts) % ngrp, b = blockIdx.y;
  const int per = cdiv(ntiles, nparts);
  const int tile0 = part * per, tile1 = imin(ntiles, tile0 + per);
  const int ntl = imax(0, tile1 - tile0);
  const int32_t* rexp = row_exp + (size_t)b * rows;
  uint8_t* bsm = smem;                                              // nks x kRBStep
  uint8_t* asm_ = smem + nks * kRBStep;                             // nst x kRAStage
  double* stg = reinterpret_cast<double*>(asm_ + nst * kRAStage);   // kRM x kRStgLd: the tile's X
  const double nan = __longlong_as_double(0x7FF8000000000000ll);

  if (tid < kRW) {
    const int o = h * kRW + tid;
    const int e = o < 2 * m ? fexp[(size_t)b * 2 * m + o] : oz::kExpMin;
    s_finv[tid] = e == oz::kExpNonFinite ? nan : oz::pow2(e - 26);
  }
  if (tid == 0) {
    tc::mbar_init(&bar_b, 1);
    for (int s = 0; s < kRStagesMax; ++s) {
      tc::mbar_init(&bar_full[s], 1);
      tc::mbar_init(&bar_dfree[s], 1);
    }
    tc::mbar_init(&bar_acc_full, 1);
    tc::mbar_init(&bar_acc_free, kREpiWarps);
    s_err = 0;
  }
  if (warp == kRMmaWarp) tc::tmem_alloc(&tmem_slot, kRTmemCols);
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const int nsteps = ntl * nks;

  if (warp == kRMmaWarp) {
    // ---- MMA thread: the group's B digits once, then per tile 8 MMAs per K step
    if (lane == 0 && ntl > 0) {
      const uint32_t bbytes = (uint32_t)(nks * kRBStep);
      tc::mbar_arrive_expect_tx(&bar_b, bbytes);
      tc::bulk_g2s(bsm, bdig + ((size_t)b * ngrp + h) * bbytes, bbytes, &bar_b);
      bool ok = tc::mbar_wait(&bar_b, 0, tc::kWaitPolls);
      int g = 0;                                                      // K step counter over all tiles
      for (int it = 0; it < ntl && ok; ++it) {
        if (it > 0) ok = tc::mbar_wait(&bar_acc_free, (it - 1) & 1, tc::kWaitPolls);
        tc::fence_after_sync();
        for (int s = 0; s < nks && ok; ++s, ++g) {
          const int d = g % nst;
          ok = tc::mbar_wait(&bar_full[d], (g / nst) & 1, tc::kWaitPolls);
          if (!ok) break;
          const uint64_t adesc = tc::desc_kmajor(tc::smem_addr(asm_ + d * kRAStage), tc::kCoreBytes, kRSbo);
          const uint64_t bdesc = tc::desc_kmajor(tc::smem_addr(bsm + s * kRBStep), tc::kCoreBytes, kRSbo);
          rec_step_mmas(tmem, adesc, bdesc, s == 0);
          tc::commit(&bar_dfree[d]);
        }
        if (ok) tc::commit(&bar_acc_full);
      }
      if (!ok) atomicExch(&s_err, 1);
    }
  } else if (warp == kRLoadWarp) {
    // ---- W digit steps: one 24 KB bulk copy per (tile, step) into the stage ring
    if (lane == 0) {
      for (int g = 0; g < nsteps; ++g) {
        const int d = g % nst;
        if (g >= nst && !tc::mbar_wait(&bar_dfree[d], ((g / nst) - 1) & 1, tc::kWaitPolls)) {
          atomicExch(&s_err, 1);
          break;
        }
        if (*reinterpret_cast<volatile int*>(&s_err)) break;
        const int it = g / nks, s = g - it * nks;
        const uint8_t* src = wdig + (((size_t)b * ntiles + tile0 + it) * nks + s) * kRAStage;
        tc::mbar_arrive_expect_tx(&bar_full[d], kRAStage);
        tc::bulk_g2s(asm_ + d * kRAStage, src, kRAStage, &bar_full[d]);
      }
    }
  } else if (warp >= kREpiWarp0) {
    // ---- epilogue warps: TMEM lane quarter (warp % 4), 16 of the 64 output columns, 32 rows.
    // Each lane recombines its row's levels into the staged tile; then one lane per row
    // stores the row's segment of X (in Ur and/or Ui) with a bulk copy.
    const int ew = warp - kREpiWarp0, quarter = warp & 3;
    const int c0 = (ew >> 2) * (kRW / 4);
    const uint32_t tbase = tc::tmem_at(tmem, quarter * 32, 0);
    const int rr = quarter * 32 + lane;
    double* srow = stg + rr * kRStgLd;
    const int o0 = h * kRW, o1 = imin(o0 + kRW, 2 * m);
    const int ur1 = imin(o1, m), ui0 = imax(o0, m);  // Ur columns [o0, ur1), Ui columns [ui0, o1) - m
    const bool issuer = ew < 4;                         // one warp per lane quarter stores its rows
    for (int it = 0; it < ntl; ++it) {
      bool ok = tc::mbar_wait(&bar_acc_full, it & 1, tc::kWaitPolls) && !*reinterpret_cast<volatile int*>(&s_err);
      tc::fence_after_sync();
      const int r = (tile0 + it) * kRM + rr;
      const int e = r < rows ? __ldg(rexp + r) : oz::kExpMin;
      const double rinv = e == oz::kExpNonFinite ? nan : oz::pow2(e - 26);
      if (issuer) tc::bulk_wait_read();                 // the previous tile's stores have read the staging
      tc::named_sync(1, kREpiWarps * 32);
#pragma unroll 1
      for (int jc = c0; jc < c0 + kRW / 4; jc += 8) {
        uint32_t v[oz::kDigits][8];
        if (ok) {
#pragma unroll
          for (int l = 0; l < oz::kDigits; ++l) tc::tmem_ld8(tbase + l * kRW + jc, v[l]);
#pragma unroll
          for (int l = 0; l < oz::kDigits; ++l) tc::tmem_wait8(v[l]);
        }
        if (jc + 8 == c0 + kRW / 4) {               // all of this warp's TMEM reads of the tile are done
          tc::fence_before_sync();
          __syncwarp();
          if (lane == 0) tc::mbar_arrive(&bar_acc_free);
        }
#pragma unroll
        for (int jj = 0; jj < 8; jj += 2) {
          double corr[2] = {nan, nan};
          if (ok) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              uint32_t a[oz::kDigits];
#pragma unroll
              for (int l = 0; l < oz::kDigits; ++l) a[l] = v[l][jj + q];
              corr[q] = oz::horner6(a) * rinv * s_finv[jc + jj + q];
            }
          }
          *reinterpret_cast<double2*>(srow + jc + jj) = make_double2(corr[0], corr[1]);
        }
      }
      tc::fence_smem_to_async();
      tc::named_sync(1, kREpiWarps * 32);
      if (issuer && r < rows) {
        // m and o0 are even: every segment starts 16-byte aligned and has an even length
        const size_t rowoff = (size_t)b * u_stride + (size_t)r * m;
        if (o0 < ur1) tc::bulk_s2g(Ur + rowoff + o0, srow, (uint32_t)(ur1 - o0) * 8u);
        if (ui0 < o1) tc::bulk_s2g(Ui + rowoff + (ui0 - m), srow + (ui0 - o0), (uint32_t)(o1 - ui0) * 8u);
        tc::bulk_commit();
      }
    }
    if (issuer) tc::bulk_wait_all();
  }

  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (s_err && tid == 0) {
    atomicExch(stall, 1);
    // drain: let committed MMAs and issued copies finish before TMEM and shared memory are released
    for (int s = 0; s < nst; ++s) (void)tc::mbar_wait(&bar_dfree[s], 0, tc::kWaitPolls);
    for (int s = 0; s < nst; ++s) (void)tc::mbar_wait(&bar_full[s], 0, tc::kWaitPolls);
    (void)tc::mbar_wait(&bar_b, 0, tc::kWaitPolls);
  }
  __syncthreads();
  if (warp == kRMmaWarp) tc::tmem_dealloc(tmem, kRTmemCols);
}

}  // namespace

size_t ozaki_recover_workspace_bytes(int batch, int rows, int m) {
  return align256(sizeof(int32_t) * (size_t)batch * rows) +
         align256((size_t)batch * cdiv(rows, kRM) * rec_steps(m) * kRAStage) +
         align256((size_t)batch * rec_groups(m) * rec_steps(m) * kRBStep) +
         align256(sizeof(int32_t) * (size_t)batch * 2 * m) + 256;
}

namespace {
struct RecWs {
  int32_t* row_exp;
  uint8_t* wdig;
  uint8_t* bdig;
  int32_t* fexp;
  int* stall;
};
RecWs rec_ws(void* workspace, int batch, int rows, int m) {
  char* ws = static_cast<char*>(workspace);
  RecWs w;
  w.row_exp = reinterpret_cast<int32_t*>(ws);
  ws += align256(sizeof(int32_t) * (size_t)batch * rows);
  w.wdig = reinterpret_cast<uint8_t*>(ws);
  ws += align256((size_t)batch * cdiv(rows, kRM) * rec_steps(m) * kRAStage);
  w.bdig = reinterpret_cast<uint8_t*>(ws);
  ws += align256((size_t)batch * rec_groups(m) * rec_steps(m) * kRBStep);
  w.fexp = reinterpret_cast<int32_t*>(ws);
  ws += align256(sizeof(int32_t) * (size_t)batch * 2 * m);
  w.stall = reinterpret_cast<int*>(ws);
  return w;
}
}  // namespace

cudaError_t launch_recover_wdigits(const double* A, const double* D, int64_t ab_stride, int batch, int rows, int m,
                                   void* workspace, cudaStream_t stream) {
  const RecWs w = rec_ws(workspace, batch, rows, m);
  ozaki_wdigits_kernel<<<dim3(cdiv(rows, kRM), batch), 256, 0, stream>>>(A, D, ab_stride, rows, m, w.wdig,
                                                                          w.row_exp);
  return cudaGetLastError();
}

cudaError_t launch_recover_products(const double* P, const double* Q, double* Ur, double* Ui, int64_t u_stride,
                                    int batch, int rows, int m, void* workspace, cudaStream_t stream) {
  const RecWs w = rec_ws(workspace, batch, rows, m);
  ozaki_recover_prep_kernel<<<dim3(rec_groups(m) * 8, batch), 256, 0, stream>>>(P, Q, m, w.bdig, w.fexp);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const int smem = rec_smem(m);
  err = cudaFuncSetAttribute(ozaki_recover_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return err;
  // tiles of an (instance, group) split into parts: about four CTAs per SM over the grid
  const int ntiles = cdiv(rows, kRM), pairs = batch * rec_groups(m);
  const ssn_tuning* tune = active_tuning();
  const int want = (tune && tune->recover_parts > 0) ? tune->recover_parts : cdiv(4 * sm_count_oz(), pairs);
  const int nparts = imax(1, imin(ntiles, want));
  ozaki_recover_kernel<<<dim3(nparts * rec_groups(m), batch), kRThreads, smem, stream>>>(
      w.wdig, w.row_exp, w.bdig, w.fexp, Ur, Ui, u_stride, rows, m, nparts, w.stall);
  return cudaGetLastError();
}

cudaError_t launch_recover_ozaki(const double* A, const double* D, int64_t ab_stride, const double* P,
                                 const double* Q, double* Ur, double* Ui, int64_t u_stride, int batch, int rows,
                                 int m, void* workspace, cudaStream_t stream) {
  cudaError_t err = launch_recover_wdigits(A, D, ab_stride, batch, rows, m, workspace, stream);
  if (err != cudaSuccess) return err;
  return launch_recover_products(P, Q, Ur, Ui, u_stride, batch, rows, m, workspace, stream);
}

}  // namespace ssn
