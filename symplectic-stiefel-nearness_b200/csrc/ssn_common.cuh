// ssn_common.cuh -- shared device helpers for the sm_100a symplectic Stiefel solver.
//
// * FP64 tensor-core fragments: mma.sync m8n8k4 f64 (DMMA).  On B200 it runs at
//   the same 37 TFLOP/s as SIMT DFMA but issues 256 FMAs per warp instruction and
//   reuses register fragments, so products reach the FP64 pipe limit with far
//   fewer issue slots and shared-memory reads.  tcgen05 has no f64 kind.
// * cp.async 16-byte global->shared copies for K-panel double buffering.
// * Deterministic CTA reductions: fixed shuffle tree + fixed-order warp sum, so
//   every thread of a CTA sees bit-identical scalars and takes the same branch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ssn.h"

namespace ssn {

constexpr int kMaxM = 128;      // m = 2k <= 128
constexpr int kThreads = 512;   // CTA size of the Newton / component kernels
constexpr int kWarps = kThreads / 32;
constexpr int kPanelK = 16;     // K extent of one staged panel
constexpr int kMinorLd = 20;    // leading dim of K-minor panels (== 4 mod 16)

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ constexpr int round_up(int a, int b) { return cdiv(a, b) * b; }
// Smallest leading dimension >= x with ld == 4 (mod 16) doubles: DMMA fragment
// loads (8 rows x 4 k, or 4 k x 8 cols) then hit 16 distinct bank pairs per half-warp.
__host__ __device__ constexpr int frag_ld(int x) { return x + (((4 - x) % 16) + 16) % 16; }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int imin(int a, int b) { return a < b ? a : b; }

// m-bucket: products are tiled for mp <= 32*MB.
__host__ __device__ constexpr int bucket_of(int m) { return m <= 32 ? 1 : m <= 64 ? 2 : m <= 96 ? 3 : 4; }

// ---------------------------------------------------------------- PTX wrappers
// D = A(8x4, row) * B(4x8, col) + C.  Lane l: g = l>>2, t = l&3;
// a = A[g][t], b = B[t][g], {c0,c1} = C[g][2t], C[g][2t+1].
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async_16(void* smem_dst, const void* gmem_src) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; every thread returns the same bits.  red: >= kWarps doubles.
template <int THREADS = kThreads>
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < THREADS / 32; ++w) s += red[w];
  return s;
}

// Two sums with one pair of barriers.  red: >= 2*kWarps doubles.
template <int THREADS = kThreads>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = a;
    red[THREADS / 32 + (threadIdx.x >> 5)] = b;
  }
  __syncthreads();
  double sa = 0.0, sb = 0.0;
#pragma unroll
  for (int w = 0; w < THREADS / 32; ++w) {
    sa += red[w];
    sb += red[THREADS / 32 + w];
  }
  a = sa;
  b = sb;
}

// ---------------------------------------------------------------- product engine
// One operand of a product: op = stored or stored^T, stored row-major with
// leading dimension ld.  alias >= 0 (B operands only): reuse the smem panel of
// A operand `alias` (same stored data and the same K-major layout); valid only
// when that A operand is transposed and the product runs in one row pass with
// R == N, so the A panel covers exactly the B columns.
struct MatOp {
  const double* ptr;
  int ld;
  int trans;
  int alias;
};

__device__ __forceinline__ MatOp op_n(const double* p, int ld) { return MatOp{p, ld, 0, -1}; }
__device__ __forceinline__ MatOp op_t(const double* p, int ld) { return MatOp{p, ld, 1, -1}; }

// Coefficient table: 2 bits per (out, a, b): 1 = +, 2 = -.  Index (o*4 + a*2 + b).
__host__ __device__ constexpr uint32_t coef_bit(int o, int a, int b, int s) {
  return static_cast<uint32_t>(s) << (2 * (o * 4 + a * 2 + b));
}
__host__ __device__ constexpr int coef_get(uint32_t c, int o, int a, int b) {
  return static_cast<int>((c >> (2 * (o * 4 + a * 2 + b))) & 3u);
}

// Copy one K-panel [k0, k0+16) of an operand into a shared slot, zero-filling
// outside [0,outer) x [0,K) up to the padded extent.
//   kminor: slot[o * kMinorLd + kk] = stored[o][k0+kk]   (o < outer_pad)
//   kmajor: slot[kk * pld + o]      = stored[k0+kk][o]
__device__ __forceinline__ void load_panel(double* slot, const double* ptr, int ld, bool kminor,
                                           int outer, int outer_pad, int pld, int k0, int K) {
  if (kminor) {
    const int chunks = outer_pad * (kPanelK / 2);
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
      const int o = c >> 3, kk = (c & 7) * 2, k = k0 + kk;
      double* dst = slot + o * kMinorLd + kk;
      if (o < outer && k + 1 < K) {
        cp_async_16(dst, ptr + (size_t)o * ld + k);
      } else {
        dst[0] = (o < outer && k < K) ? ptr[(size_t)o * ld + k] : 0.0;
        dst[1] = 0.0;
      }
    }
  } else {
    const int half = outer_pad / 2;
    const int chunks = kPanelK * half;
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
      const int kk = c / half, o = (c - kk * half) * 2, k = k0 + kk;
      double* dst = slot + kk * pld + o;
      if (k < K && o + 1 < outer) {
        cp_async_16(dst, ptr + (size_t)k * ld + o);
      } else {
        dst[0] = (k < K && o < outer) ? ptr[(size_t)k * ld + o] : 0.0;
        dst[1] = 0.0;
      }
    }
  }
}

// Doubles of one staged K-panel of an operand with `rows` (a multiple of 8) outer
// rows, in either layout: K-minor rows x kMinorLd, or K-major kPanelK x frag_ld(rows).
__host__ __device__ constexpr int panel_slot(int rows) {
  return (rows * kMinorLd > kPanelK * frag_ld(rows)) ? rows * kMinorLd : kPanelK * frag_ld(rows);
}

// CTA-wide product engine (kThreads threads, warps on a 4x4 grid).
//   out_o[r][c] = sum_{a,b} sign(o,a,b) * op(A_a)[r][:] . op(B_b)[:][c]
// for r < R, c < N, contraction K, with R, N <= 128.  Each warp owns a
// (WR*8) x (WC*8) tile; row passes of 4*WR*8 rows cover R.  Results are handed
// to epi(o, r, c, value) for every valid (r, c).
//
// K-panels stream through ST stages of shared memory, each [A_0 A_1 B_0 B_1]
// with slotA doubles per A slot (>= panel_slot of the rows of one pass) and
// slotB per B slot (>= panel_slot(N padded to 8)): ST - 1 panels are in flight
// while one is consumed, and one barrier per panel both publishes the landed
// panel and retires the stage that the next copy overwrites.  All threads must
// call it; it ends with __syncthreads().
template <int WR, int WC, int NA, int NB, int NOUT, uint32_t COEF, int ST, class Epi>
__device__ __forceinline__ void tile_product_staged(const MatOp (&A)[NA], const MatOp (&B)[NB], int R, int N,
                                                    int K, double* smem, int slotA, int slotB, Epi& epi) {
  static_assert(NA >= 1 && NA <= 2 && NB >= 1 && NB <= 2 && NOUT >= 1 && NOUT <= 2, "engine arity");
  static_assert(ST >= 2 && ST <= 4, "pipeline depth");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wrow = warp >> 2, wcol = warp & 3;
  constexpr int RP = 4 * WR * 8;
  const int npanel = cdiv(K, kPanelK);
  const int N_pad = round_up(N, 8);
  const int pldB = frag_ld(N_pad);
  const int stage_sz = 2 * slotA + 2 * slotB;
  auto a_slot = [&](int stage, int a) { return smem + stage * stage_sz + a * slotA; };
  auto b_slot = [&](int stage, int b) { return smem + stage * stage_sz + 2 * slotA + b * slotB; };

  for (int r0 = 0; r0 < R; r0 += RP) {
    const int Rp = imin(RP, R - r0);
    const int Rp_pad = round_up(Rp, 8);
    const int pldA = frag_ld(Rp_pad);
    double acc[NOUT][WR][WC][2];
#pragma unroll
    for (int o = 0; o < NOUT; ++o)
#pragma unroll
      for (int i = 0; i < WR; ++i)
#pragma unroll
        for (int j = 0; j < WC; ++j) acc[o][i][j][0] = acc[o][i][j][1] = 0.0;

    auto issue = [&](int stage, int k0) {
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const bool kminor = !A[a].trans;
        const double* base = A[a].trans ? A[a].ptr + r0 : A[a].ptr + (size_t)r0 * A[a].ld;
        load_panel(a_slot(stage, a), base, A[a].ld, kminor, Rp, Rp_pad, pldA, k0, K);
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        if (B[b].alias >= 0) continue;
        const bool kminor = B[b].trans;
        load_panel(b_slot(stage, b), B[b].ptr, B[b].ld, kminor, N, N_pad, pldB, k0, K);
      }
      cp_async_commit();
    };

    const int row_base = wrow * WR * 8;
    const int col_base = wcol * WC * 8;
#pragma unroll
    for (int sp = 0; sp < ST - 1; ++sp) {
      if (sp < npanel) issue(sp, sp * kPanelK);
      else cp_async_commit();
    }
    for (int kp = 0; kp < npanel; ++kp) {
      cp_async_wait<ST - 2>();      // this thread's copies of panel kp have landed
      __syncthreads();              // everyone's have; every warp is done with panel kp - 1
      {
        const int nk = kp + ST - 1;  // refill the stage panel kp - 1 used
        if (nk < npanel) issue(nk % ST, nk * kPanelK);
        else cp_async_commit();
      }
      const int stage = kp % ST;
      if (row_base < Rp && col_base < N) {
#pragma unroll
        for (int ks = 0; ks < kPanelK / 4; ++ks) {
          const int kk = ks * 4 + t;
          double af[NA][WR], bf[NB][WC];
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            const double* s = a_slot(stage, a);
#pragma unroll
            for (int i = 0; i < WR; ++i) {
              // sub-tiles past the padded row extent are never read (they may lie past the slot)
              const int r = row_base + i * 8 + g;
              af[a][i] = (row_base + i * 8 < Rp) ? (A[a].trans ? s[kk * pldA + r] : s[r * kMinorLd + kk]) : 0.0;
            }
          }
#pragma unroll
          for (int b = 0; b < NB; ++b) {
            const double* s = B[b].alias >= 0 ? a_slot(stage, B[b].alias) : b_slot(stage, b);
            const int ld = B[b].alias >= 0 ? pldA : pldB;
            const bool kminor = B[b].alias >= 0 ? false : (B[b].trans != 0);
#pragma unroll
            for (int j = 0; j < WC; ++j) {
              const int c = col_base + j * 8 + g;
              bf[b][j] = (col_base + j * 8 < N) ? (kminor ? s[c * kMinorLd + kk] : s[kk * ld + c]) : 0.0;
            }
          }
#pragma unroll
          for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
              for (int b = 0; b < NB; ++b) {
                const int sg = coef_get(COEF, o, a, b);
                if (sg == 0) continue;
#pragma unroll
                for (int i = 0; i < WR; ++i) {
                  if (row_base + i * 8 >= Rp) continue;
                  const double av = sg == 2 ? -af[a][i] : af[a][i];
#pragma unroll
                  for (int j = 0; j < WC; ++j) {
                    if (col_base + j * 8 >= N) continue;
                    dmma_8x8x4(acc[o][i][j][0], acc[o][i][j][1], av, bf[b][j]);
                  }
                }
              }
        }
      }
    }
    cp_async_wait<0>();
    __syncthreads();   // every warp is done with the panels: epilogues may write over the stages
    // epilogue
#pragma unroll
    for (int o = 0; o < NOUT; ++o)
#pragma unroll
      for (int i = 0; i < WR; ++i)
#pragma unroll
        for (int j = 0; j < WC; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int r = row_base + i * 8 + g;
            const int c = col_base + j * 8 + 2 * t + e;
            if (r < Rp && c < N) epi(o, r0 + r, c, acc[o][i][j][e]);
          }
    __syncthreads();   // epilogue writes are visible; the stages are free for the next pass
  }
}

// Two stages of four equal slots of `slot` doubles (8 * slot doubles of smem).
template <int WR, int WC, int NA, int NB, int NOUT, uint32_t COEF, class Epi>
__device__ __forceinline__ void tile_product(const MatOp (&A)[NA], const MatOp (&B)[NB], int R, int N, int K,
                                   double* smem, int slot, Epi& epi) {
  tile_product_staged<WR, WC, NA, NB, NOUT, COEF, 2>(A, B, R, N, K, smem, slot, slot, epi);
}

// Warp-tile shape for bucket MB (mp <= 32*MB) and NOUT accumulator sets,
// keeping NOUT*WR*WC*2 <= 36 doubles of accumulators per thread.
template <int MB, int NOUT>
struct Tile {
  static constexpr int WC = MB;
  static constexpr int WR = imin(MB == 1 ? 4 : MB, imax(1, 18 / (NOUT * WC)));
  static constexpr int ROWS = 4 * WR * 8;  // rows per pass
};

// Shared-memory slot size (doubles) for bucket MB.
__host__ __device__ constexpr int slot_doubles(int MB) {
  return imax(32 * MB * kMinorLd, kPanelK * frag_ld(32 * MB));
}
__host__ __device__ constexpr int slot_doubles_rows(int rows, int MB) {
  return imax(imax(rows, 32 * MB) * kMinorLd, kPanelK * frag_ld(imax(rows, 32 * MB)));
}

}  // namespace ssn

namespace ssn {

// ---------------------------------------------------------------- shared-memory products
// out(i, j) for i < R, j < N of op(A)[R x K] * op(B)[K x N] with both operands
// already in shared memory (row-major, leading dims lda/ldb, K a multiple of 4,
// R and N multiples of 8).  Each warp computes 16 x 16 output blocks (2 x 2
// DMMA tiles) in turn and hands every element to fn(i, j, value).  No barrier.
// Leading dimensions == 4 (mod 16) keep the fragment loads conflict-free.
template <bool AT, bool BT, class Fn>
__device__ __forceinline__ void smem_product(int R, int N, int K, const double* A, int lda,
                                             const double* B, int ldb, Fn&& fn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int br = cdiv(R, 16), bc = cdiv(N, 16);
  for (int blk = warp; blk < br * bc; blk += nwarps) {
    const int r0 = (blk / bc) * 16, c0 = (blk % bc) * 16;
    double acc[2][2][2] = {};
    for (int k = 0; k < K; k += 4) {
      double af[2], bf[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = r0 + 8 * i + g;
        af[i] = (r0 + 8 * i < R) ? (AT ? A[(k + t) * lda + r] : A[r * lda + k + t]) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int c = c0 + 8 * j + g;
        bf[j] = (c0 + 8 * j < N) ? (BT ? B[c * ldb + k + t] : B[(k + t) * ldb + c]) : 0.0;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = r0 + 8 * i + g, c = c0 + 8 * j + 2 * t + e;
          if (r0 + 8 * i < R && c0 + 8 * j < N) fn(r, c, acc[i][j][e]);
        }
  }
}

// One 16 x 16 block (rows r0.., columns c0..) of op(A)[R x 16] * op(B)[16 x N],
// handed to fn(i, j, value); the same DMMA sequence as smem_product's blocks.
template <bool AT, bool BT, class Fn>
__device__ __forceinline__ void smem_block16(int r0, int c0, const double* A, int lda, const double* B, int ldb,
                                             Fn&& fn) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[2][2][2] = {};
#pragma unroll
  for (int k = 0; k < 16; k += 4) {
    double af[2], bf[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = r0 + 8 * i + g;
      af[i] = AT ? A[(k + t) * lda + r] : A[r * lda + k + t];
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = c0 + 8 * j + g;
      bf[j] = BT ? B[c * ldb + k + t] : B[(k + t) * ldb + c];
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) fn(r0 + 8 * i + g, c0 + 8 * j + 2 * t + e, acc[i][j][e]);
}

// Rank-16 update out(i, j) = X[i][:16] . U[:16][j] over an mp x mp square (mp = 32 WT),
// one (8 WT) x (8 WT) tile per warp of a 4 x 4 warp grid (kThreads threads): WT^2
// independent accumulators per warp, and each 8x8 fragment sees the same DMMA
// sequence as in smem_product, so the results are the same bits.
template <int WT, class Fn>
__device__ __forceinline__ void smem_rank16_tiled(const double* X, int ldx, const double* U, int ldu, Fn&& fn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = (warp >> 2) * 8 * WT, c0 = (warp & 3) * 8 * WT;
  double acc[WT][WT][2];
#pragma unroll
  for (int i = 0; i < WT; ++i)
#pragma unroll
    for (int j = 0; j < WT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
  for (int k = 0; k < 16; k += 4) {
    double af[WT], bf[WT];
#pragma unroll
    for (int i = 0; i < WT; ++i) af[i] = X[(r0 + 8 * i + g) * ldx + k + t];
#pragma unroll
    for (int j = 0; j < WT; ++j) bf[j] = U[(k + t) * ldu + c0 + 8 * j + g];
#pragma unroll
    for (int i = 0; i < WT; ++i)
#pragma unroll
      for (int j = 0; j < WT; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
  }
#pragma unroll
  for (int i = 0; i < WT; ++i)
#pragma unroll
    for (int j = 0; j < WT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) fn(r0 + 8 * i + g, c0 + 8 * j + 2 * t + e, acc[i][j][e]);
}

// Inverse of a symmetric positive definite matrix held in shared memory,
// in place, by block Gauss-Jordan sweeps over 16 x 16 pivot blocks:
//   Dinv = K_PP^-1,  U = Dinv K_PQ,  W = K_QP Dinv,
//   K_QQ -= K_QP U,  K_PQ = U,  K_QP = -W,  K_PP = Dinv,
// for each pivot block P (Q = the other indices).  The small inverse is a
// scalar sweep run by warp 0 whose pivots are the Schur-complement diagonals:
// they are all positive exactly when K is positive definite (the test
// torch.linalg.cholesky_ex applies).  K: mp x mp (mp = m rounded up to 16;
// the caller pads the tail with the identity), leading dim ld == 4 (mod 16).
// scratch: 16 * ld + 2 * mp * 20 doubles.  Returns the same bool in every thread.
__host__ __device__ constexpr int spd_region_doubles(int m) {
  return round_up(m, 16) * frag_ld(round_up(m, 16)) + 16 * frag_ld(round_up(m, 16)) + 2 * round_up(m, 16) * 20;
}

__device__ __forceinline__ bool spd_inverse_blocked(double* K, int mp, int ld, double* scratch,
                                                    int* flag) {
  constexpr int b = 16;
  double* U = scratch;               // b x ld   : U[p][j]
  double* W = scratch + b * ld;      // mp x b   stored as W[j][p] with leading dim 20
  double* X = W + mp * 20;           // mp x b   old K_:,P, leading dim 20
  if (threadIdx.x == 0) *flag = 1;
  for (int k0 = 0; k0 < mp; k0 += b) {
    // (1) warp 0 inverts the b x b diagonal block (scalar sweep operator) in
    // registers: lane (i, h) = (lane & 15, lane >> 4) holds row i, columns
    // 8h .. 8h+7; the pivot row, a_ik and the pivot are broadcast by shuffles,
    // so the sequential pivot chain never goes through shared memory.
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x, i = lane & 15, h = lane >> 4;
      double r[8];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) r[jj] = K[(k0 + i) * ld + k0 + 8 * h + jj];
      bool ok = true;
#pragma unroll
      for (int k = 0; k < b; ++k) {
        const int hk = k >> 3, ck = k & 7;              // column k lives in half hk, slot ck
        const double piv = __shfl_sync(0xffffffffu, r[ck], k + 16 * hk);
        const double aik = __shfl_sync(0xffffffffu, r[ck], i + 16 * hk);
        double rowk[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) rowk[jj] = __shfl_sync(0xffffffffu, r[jj], k + 16 * h);
        ok = ok && (piv > 0.0) && isfinite(piv);
        const double inv = 1.0 / piv;
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const bool col_k = (h == hk) && (jj == ck);
          double v;
          if (i == k) v = col_k ? inv : rowk[jj] * inv;
          else if (col_k) v = -aik * inv;
          else v = r[jj] - aik * (rowk[jj] * inv);
          r[jj] = v;
        }
      }
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) K[(k0 + i) * ld + k0 + 8 * h + jj] = r[jj];
      if (lane == 0 && !ok) *flag = 0;
    }
    __syncthreads();
    if (*flag == 0) return false;
    // (2) U = Dinv K_P,:, W = K_:,P Dinv (their 16 x 16 blocks spread over all warps in one
    // pass), and a copy X = K_:,P (old) for the update
    const double* Dinv = K + k0 * ld + k0;
    {
      const int nb = mp / 16, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
      for (int blk = warp; blk < 2 * nb; blk += nwarps) {
        if (blk < nb)
          smem_block16<false, false>(0, blk * 16, Dinv, ld, K + k0 * ld, ld,
                                     [&](int p, int j, double v) { U[p * ld + j] = v; });
        else
          smem_block16<false, false>((blk - nb) * 16, 0, K + k0, ld, Dinv, ld,
                                     [&](int j, int p, double v) { W[j * 20 + p] = v; });
      }
    }
    for (int j = threadIdx.x >> 4; j < mp; j += blockDim.x >> 4) X[j * 20 + (threadIdx.x & 15)] = K[j * ld + k0 + (threadIdx.x & 15)];
    __syncthreads();
    // (3) K_QQ -= X U, K_PQ = U, K_QP = -W  (disjoint entries, one phase)
    auto update = [&](int i, int j, double v) {
      const bool ip = i >= k0 && i < k0 + b, jp = j >= k0 && j < k0 + b;
      if (!ip && !jp) K[i * ld + j] -= v;
    };
    if (blockDim.x == kThreads && mp == 96) smem_rank16_tiled<3>(X, 20, U, ld, update);
    else if (blockDim.x == kThreads && mp == 128) smem_rank16_tiled<4>(X, 20, U, ld, update);
    else if (blockDim.x == kThreads && mp == 64) smem_rank16_tiled<2>(X, 20, U, ld, update);
    else smem_product<false, false>(mp, mp, b, X, 20, U, ld, update);
    for (int p = threadIdx.x >> 5; p < b; p += blockDim.x >> 5)
      for (int j = threadIdx.x & 31; j < mp; j += 32) {
        if (j >= k0 && j < k0 + b) continue;
        K[(k0 + p) * ld + j] = U[p * ld + j];
        K[j * ld + k0 + p] = -W[j * 20 + p];
      }
    __syncthreads();
  }
  return true;
}

}  // namespace ssn
