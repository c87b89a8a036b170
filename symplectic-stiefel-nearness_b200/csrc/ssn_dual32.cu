// ssn_dual32.cu -- FP32 early Newton-CG phase of the split-precision form.
//
// The split-precision form runs the dual Newton-CG of dual_batch
// (src/symplectic_projection/dual_recommended_hvp.py:99-191) in three launches:
//  1. dual_kernel, set-up only: the rotated Gram CrE = sym(V^T Cr V)/s,
//     Ce = skew(V^T Ci V)/s and Je = skew(V^T J V)/s in FP64, into the workspace;
//  2. this kernel: the early Newton steps entirely in FP32 -- sandwich,
//     gradient and residual, PCG with HVPs, the trial's positive-definiteness
//     test and inverse, Armijo with the exact objective change -- while the
//     FP32 residual is at least switch_tol (1e-5; FP32 resolves the residual
//     of these problems to about 1e-7) and still improving (three steps
//     without a new best, or half the Newton cap, hand over: ill-conditioned
//     targets can have an FP32 residual floor above switch_tol).  It writes
//     omega in FP64 and the number of Newton updates it took;
//  3. dual_kernel warm-started from that omega: P = (I + omega^2)^-1 in FP64
//     with the positive-definiteness test, then the last Newton step(s) with
//     FP64 sandwich, residual, trial inverse and line search, and convergence
//     declared only on the FP64 residual.  The returned omega, P, Q and the
//     acceptance of the result are FP64 throughout.
// The FP32 steps follow the reference's Newton-CG step for step (the direct
// first step, the CG tolerance clamp(sqrt(res), 1e-8, 0.1) ||g||, the
// non-descent fallback, Armijo halving with the 1e-4 t slope test).
//
// Layout.  One CTA, or a 2-CTA cluster, per instance: CTA c owns rows (and,
// for the symmetric and antisymmetric matrices, columns) [c H, (c+1) H) of
// every MP x MP matrix (MP = m padded to 32 MB with zero, or identity, rows;
// H = MP / CL).  The state stays on chip:
//  * shared memory: full copies of P and Q (Q's space holds the trial omega,
//    P's the trial K and its inverse, in the line search) and of the CG
//    direction p (or the Newton direction d) in every CTA; this CTA's columns
//    of Sr and Si and of the HVP's intermediates; the constant rotated Gram,
//    staged from L2 once per step;
//  * registers: each thread owns one 4 x 4 tile of this CTA's rows of omega,
//    d, r, p (and of the adaptive preconditioner), and computes exactly that
//    tile (or its transpose, for column-split products) in every product, so
//    the element-wise PCG work needs no shared-memory traffic.
// Products run on the tensor cores (mma.sync m16n8k8 TF32): each warp computes
// the 16 x 32 (or 32 x 16) block of the product that its 32 threads' 4 x 4
// tiles make up, and hands the tiles out through a small per-warp staging area.
// The products that set the iterate -- Q = -omega P, the sandwich and the trial
// K -- use the 3xTF32 split (hi*hi + hi*lo + lo*hi, about 2^-21 relative per
// term); the CG's HVPs and the line search's change, whose errors only perturb
// the inexact Newton direction and the Armijo test, use one TF32 product.
// Symmetric and antisymmetric operands are read through their transposes
// (P^T = P, Q^T = -Q, ...), so every operand is a row segment.
//
// All decisions (convergence, CG stop, acceptance) follow reductions summed
// in FP64 in a fixed order, identical in both CTAs of a cluster, so all
// threads branch together.  Every loop is bounded (max_newton, max_cg,
// max_backtrack, 16-wide pivot blocks).
#include <cooperative_groups.h>
#include <float.h>
#include <math.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace cg = cooperative_groups;

namespace ssn {

namespace {

// Workspace slots of the dual workspace (the enumeration of ssn_dual.cu).
constexpr int kSlotCe = 0, kSlotJe = 1, kSlotW = 2, kSlotT1 = 15, kSlotX2 = 20, kSlotAux = 22;

template <int MB, int CL>
struct G32 {
  static constexpr int MP = 32 * MB;          // padded order
  static constexpr int H = MP / CL;           // rows / columns owned by one CTA
  static constexpr int LDF = MP + 4;          // leading dim of full and own-row buffers (floats)
  static constexpr int LDO = H + 4;           // leading dim of own-column buffers
  static constexpr int TA = H / 4, TB = MP / 4;
  static constexpr int THREADS = TA * TB;     // one 4 x 4 tile per thread
  static constexpr int WARPS = THREADS / 32;
  static constexpr int NWB = TB / 8;
  static constexpr int FULL = MP * LDF, OWNC = MP * LDO, OWNR = H * LDF;
  static constexpr int YF = imax(2 * OWNC, FULL);
  static constexpr int SS = YF;
  static constexpr int NRED = 5;              // values of the widest fused reduction
  // offsets in floats
  static constexpr int STAGE = 384;           // floats per warp: tensor-core product tiles -> 4 x 4 tiles
  static constexpr int O_P = 0, O_Q = O_P + FULL, O_X = O_Q + FULL, O_Y = O_X + FULL, O_Z = O_Y + YF,
                       O_S = O_Z + OWNC, O_LAM = O_S + SS, O_PD = O_LAM + MP, O_SD = O_PD + MP,
                       O_ST = round_up(O_SD + MP, 4), FLOATS = O_ST + STAGE * WARPS;
  static constexpr size_t bytes() {
    return sizeof(float) * FLOATS + sizeof(double) * (NRED * WARPS + 4 * NRED) + 64;
  }
  static_assert(THREADS % 32 == 0 && TA % 4 == 0 && TB % 8 == 0, "tile grid");
  static_assert(32 * LDF <= OWNC, "the inverse's pivot panels fit the Z buffer");
  static_assert(OWNR <= OWNC, "own rows of Si' fit the Z buffer");
};

__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ float comp(const float4& v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}
__device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// 1 / x from the hardware approximation and one Newton-Raphson step r (2 - x r), which
// squares its relative error: the pivot reciprocal of the trial inverse, on its latency chain.
__device__ __forceinline__ float rcp_nr(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;\n" : "=f"(r) : "f"(x));
  return r * fmaf(-x, r, 2.0f);
}

// ---- products on the tensor cores: mma.sync m16n8k8 TF32 in the 3xTF32 form.
// Each FP32 operand x is split as hi = tf32(x), lo = tf32(x - hi), and a product is
// hi*hi + hi*lo + lo*hi with FP32 accumulation: about 2^-21 relative per product term
// (the lo*lo term and the rounding of lo are below it), against 2^-24 for FFMA.
__device__ __forceinline__ uint32_t lds1(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.b32 %0, [%1];\n" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ void split_tf32(uint32_t x, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(hi) : "f"(__uint_as_float(x)));
  const float r = __uint_as_float(x) - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(lo) : "f"(r));
}
__device__ __forceinline__ uint32_t to_tf32(uint32_t x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(__uint_as_float(x)));
  return r;
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// acc[o][x][y] = sum_k sum_(a,b) sign(o,a,b) A_a[k][4u + x] B_b[k][4v + y]: the 4 x 4 tile
// (u, v) of sum op(A) op(B), with every operand given as K row segments (shared-memory
// byte addresses, leading dims in floats), for the kernel's thread layout: lane l of a warp owns the
// 4 x 4 tile (u, v) with u = u0 + (l >> 3), v = v0 + (l & 7) (TR = false: a 16 x 32 warp
// tile, one m16 x four n8 MMA tiles) or u = u0 + (l & 7), v = v0 + (l >> 3) (TR = true:
// 32 x 16, two m16 x two n8).  The accumulator fragments go through the warp's STAGE
// floats of shared memory (one half of the warp tile at a time) into the 4 x 4 tiles.
// All 32 lanes of the warp call it together.
template <int NA, int NB, int NOUT, uint32_t COEF, int K, bool TR, bool X3 = true>
__device__ __forceinline__ void outer_tc(const uint32_t (&A)[NA], int lda, int u, const uint32_t (&B)[NB], int ldb,
                                         int v, float* stage, float (&acc)[NOUT][4][4]) {
  constexpr int MT = TR ? 2 : 1, NT = TR ? 2 : 4;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int lr = TR ? (lane & 7) : (lane >> 3), lc = TR ? (lane >> 3) : (lane & 7);
  const uint32_t R0 = 4u * (uint32_t)(u - lr), C0 = 4u * (uint32_t)(v - lc);   // warp tile origin
  float c[NOUT][MT * NT][4];
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int q = 0; q < MT * NT; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) c[o][q][e] = 0.0f;
#pragma unroll 2
  for (int k = 0; k < K; k += 8) {
#pragma unroll
    for (int mi = 0; mi < MT; ++mi) {
      // A fragments: a0 = (row g, k t), a1 = (g + 8, t), a2 = (g, t + 4), a3 = (g + 8, t + 4)
      uint32_t ah[NA][4], al[NA][X3 ? 4 : 1];
#pragma unroll
      for (int ia = 0; ia < NA; ++ia) {
        const uint32_t base = A[ia] + 4u * ((uint32_t)(k + t) * lda + R0 + 16u * mi + g);
        const uint32_t x0 = lds1(base), x1 = lds1(base + 32u);
        const uint32_t x2 = lds1(base + 16u * lda), x3 = lds1(base + 16u * lda + 32u);
        if constexpr (X3) {
          split_tf32(x0, ah[ia][0], al[ia][0]);
          split_tf32(x1, ah[ia][1], al[ia][1]);
          split_tf32(x2, ah[ia][2], al[ia][2]);
          split_tf32(x3, ah[ia][3], al[ia][3]);
        } else {
          ah[ia][0] = to_tf32(x0);
          ah[ia][1] = to_tf32(x1);
          ah[ia][2] = to_tf32(x2);
          ah[ia][3] = to_tf32(x3);
        }
      }
#pragma unroll
      for (int nj = 0; nj < NT; ++nj) {
#pragma unroll
        for (int ib = 0; ib < NB; ++ib) {
          // B fragment: b0 = (k t, column g), b1 = (k t + 4, g)
          const uint32_t base = B[ib] + 4u * ((uint32_t)(k + t) * ldb + C0 + 8u * nj + g);
          uint32_t bh0, bl0 = 0u, bh1, bl1 = 0u;
          if constexpr (X3) {
            split_tf32(lds1(base), bh0, bl0);
            split_tf32(lds1(base + 16u * ldb), bh1, bl1);
          } else {
            bh0 = to_tf32(lds1(base));
            bh1 = to_tf32(lds1(base + 16u * ldb));
          }
#pragma unroll
          for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int ia = 0; ia < NA; ++ia) {
              const int sg = coef_get(COEF, o, ia, ib);
              if (sg == 0) continue;
              const uint32_t f = sg == 2 ? 0x80000000u : 0u;   // negate the A operand
              float (&cc)[4] = c[o][mi * NT + nj];
              if constexpr (X3) {
                mma_tf32(cc, al[ia][0] ^ f, al[ia][1] ^ f, al[ia][2] ^ f, al[ia][3] ^ f, bh0, bh1);
                mma_tf32(cc, ah[ia][0] ^ f, ah[ia][1] ^ f, ah[ia][2] ^ f, ah[ia][3] ^ f, bl0, bl1);
              }
              mma_tf32(cc, ah[ia][0] ^ f, ah[ia][1] ^ f, ah[ia][2] ^ f, ah[ia][3] ^ f, bh0, bh1);
            }
        }
      }
    }
  }
  // fragments (row g / g + 8, columns 2 t, 2 t + 1 of each n8 tile) -> 4 x 4 tiles
  constexpr int LD = TR ? 24 : 40;
  float* st = stage + (threadIdx.x >> 5) * 384;
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      __syncwarp();
      if constexpr (!TR) {
        // half h: rows 8 h .. 8 h + 7 of the 16 x 32 tile
#pragma unroll
        for (int nj = 0; nj < NT; ++nj)
          *reinterpret_cast<float2*>(st + g * LD + 8 * nj + 2 * t) =
              make_float2(c[o][nj][2 * h], c[o][nj][2 * h + 1]);
        __syncwarp();
        // every lane reads (rows clamped into the half)
        const bool mine = (lr >> 1) == h;
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const float4 w = ld4(st + ((4 * lr + x) & 7) * LD + 4 * lc);
          // the first half is taken by every lane (so no earlier value of acc stays live),
          // the second only by its owners
          if (h == 0 || mine) { acc[o][x][0] = w.x; acc[o][x][1] = w.y; acc[o][x][2] = w.z; acc[o][x][3] = w.w; }
        }
      } else {
        // half h: m16 tile h, rows 16 h .. 16 h + 15 of the 32 x 16 tile
#pragma unroll
        for (int nj = 0; nj < NT; ++nj) {
          *reinterpret_cast<float2*>(st + g * LD + 8 * nj + 2 * t) =
              make_float2(c[o][h * NT + nj][0], c[o][h * NT + nj][1]);
          *reinterpret_cast<float2*>(st + (g + 8) * LD + 8 * nj + 2 * t) =
              make_float2(c[o][h * NT + nj][2], c[o][h * NT + nj][3]);
        }
        __syncwarp();
        const bool mine = (lr >> 2) == h;
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const float4 w = ld4(st + ((4 * lr + x) & 15) * LD + 4 * lc);
          // the first half is taken by every lane (so no earlier value of acc stays live),
          // the second only by its owners
          if (h == 0 || mine) { acc[o][x][0] = w.x; acc[o][x][1] = w.y; acc[o][x][2] = w.z; acc[o][x][3] = w.w; }
        }
      }
    }
  __syncwarp();
}

// The CTAs of one instance: sync() is the phase barrier; sumv() sums N values over the
// CTA in FP64 (fixed shuffle tree, fixed warp order) and, for CL = 2, adds both CTAs'
// partials in a fixed order through distributed shared memory, so both CTAs hold the
// same bits and branch together.
template <int CL, int THREADS, int NMAX>
struct Clu {
  static constexpr int WARPS = THREADS / 32;
  int rank;
  double* red;        // NMAX * WARPS doubles
  double* xch;        // [2 parities][NMAX values][2 ranks]
  double* xch_peer;
  int parity;
  __device__ __forceinline__ void sync() {
    if constexpr (CL == 1) __syncthreads();
    else cg::this_cluster().sync();
  }
  template <int N>
  __device__ __forceinline__ void sumv(double (&v)[N]) {
    static_assert(N <= NMAX, "reduction width");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = warp_sum(v[q]);
    __syncthreads();                       // the previous reduction's readers are done with red
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < N; ++q) red[q * WARPS + warp] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < N; ++q) {
      double s = 0.0;
#pragma unroll
      for (int w = 0; w < WARPS; ++w) s += red[q * WARPS + w];
      v[q] = s;
    }
    if constexpr (CL == 2) {
      double* slot = xch + parity * 2 * NMAX;
      double* peer = xch_peer + parity * 2 * NMAX;
      if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < N; ++q) {
          slot[2 * q + rank] = v[q];
          peer[2 * q + rank] = v[q];
        }
      cg::this_cluster().sync();
#pragma unroll
      for (int q = 0; q < N; ++q) v[q] = slot[2 * q] + slot[2 * q + 1];
      parity ^= 1;
    }
  }
};

}  // namespace

template <int MB, int CL, bool ADAPTIVE>
__global__ void __launch_bounds__(G32<MB, CL>::THREADS, 1) dual32_kernel(Dual32Args args) {
  using G = G32<MB, CL>;
  constexpr int MP = G::MP, H = G::H, LDF = G::LDF, LDO = G::LDO, THREADS = G::THREADS;
  extern __shared__ __align__(16) float sm[];
  const int m = args.m, mm = m * m;
  const int mr = round_up(m, 4);
  const int rank = CL == 1 ? 0 : (int)cg::this_cluster().block_rank();
  const int inst = blockIdx.x / CL;
  const int r0 = rank * H;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ta = 4 * (warp / G::NWB) + (lane >> 3);    // tile row block (own rows / own columns)
  const int tb = 8 * (warp % G::NWB) + (lane & 7);     // tile column block (all columns / all rows)

  float* Pf = sm + G::O_P;        // P (full); in the line search K and its inverse
  float* Qf = sm + G::O_Q;        // Q (full), or the trial omega in the line search
  float* Xf = sm + G::O_X;        // CG direction p or Newton direction d (full); Sr' own rows
  float* Yf = sm + G::O_Y;        // [2] own columns: Y^T, HVP intermediates, d Sr and d Si; CrE staging
  float* Zb = sm + G::O_Z;        // own columns: omega^T, Z; Si' own rows; the inverse's pivot panels
  float* Ss = sm + G::O_S;        // [2] own columns: Sr^T, Si^T; Ce staging
  float* lam = sm + G::O_LAM;     // diagonal of the rotated Gram (1 on the padding)
  float* pdg = sm + G::O_PD;      // diag(P), diag(Sr): the adaptive preconditioner
  float* sdg = sm + G::O_SD;
  float* stg = sm + G::O_ST;      // per-warp staging of the tensor-core product tiles
  double* red = reinterpret_cast<double*>(sm + G::FLOATS);
  double* xch = red + G::NRED * G::WARPS;
  int* flags = reinterpret_cast<int*>(xch + 4 * G::NRED);   // pivot-block outcome of the inverse

  Clu<CL, THREADS, G::NRED> cl{rank, red, xch, xch, 0};
  float* peer = sm;
  if constexpr (CL == 2) {
    cl.xch_peer = cg::this_cluster().map_shared_rank(xch, rank ^ 1);
    peer = cg::this_cluster().map_shared_rank(sm, rank ^ 1);
  }

  double* ws = args.work + (size_t)inst * kDualMats * mm;
  const double* Ce64 = ws + (size_t)kSlotCe * mm;
  const double* Je64 = ws + (size_t)kSlotJe * mm;
  const double* Cr64 = ws + (size_t)kSlotX2 * mm;       // the full rotated Gram (approximate basis)
  double* Wout = ws + (size_t)kSlotW * mm;
  float* g32 = reinterpret_cast<float*>(ws + (size_t)kSlotT1 * mm);   // [3][m][mr]: CrE, Ce, Je in FP32
  float* gCr = g32;
  float* gCe = g32 + (size_t)m * mr;
  float* gJe = g32 + 2 * (size_t)m * mr;
  int32_t* aux = reinterpret_cast<int32_t*>(ws + (size_t)kSlotAux * mm);   // updates, steps, hvps, trials, fallbacks
  const double s = args.scale[inst];
  const int status_in = args.eig_status ? args.eig_status[inst] : SSN_INSTANCE_CONVERGED;

  // own-row tile element (x, y): row r0 + 4 ta + x, column 4 tb + y
  const int ib = r0 + 4 * ta, jb = 4 * tb;

  // ---- set-up: FP32 copies of this CTA's rows of CrE, Ce, Je; lambda; P = I, Q = 0, omega = 0
  for (int e = tid; e < H * mr; e += THREADS) {
    const int i = r0 + e / mr, j = e - (e / mr) * mr;
    if (i >= m) continue;
    const bool in = j < m;
    gCr[(size_t)i * mr + j] = in ? (float)Cr64[(size_t)i * m + j] : 0.0f;
    gCe[(size_t)i * mr + j] = in ? (float)Ce64[(size_t)i * m + j] : 0.0f;
    gJe[(size_t)i * mr + j] = in ? (float)Je64[(size_t)i * m + j] : 0.0f;
  }
  for (int i = tid; i < MP; i += THREADS) lam[i] = i < m ? (float)Cr64[(size_t)i * m + i] : 1.0f;
  for (int e = tid; e < MP * LDF; e += THREADS) {
    const int i = e / LDF, j = e - i * LDF;
    Pf[e] = (i == j) ? 1.0f : 0.0f;
    Qf[e] = 0.0f;
  }
  // stall bookkeeping of the FP32 residual (best so far, steps since), double-buffered by step
  __shared__ float s_best[2];
  __shared__ int s_since[2];
  if (tid == 0) {
    s_best[0] = INFINITY;
    s_since[0] = 0;
  }
  __threadfence();
  cl.sync();

  // one row segment of a global [rows][mr] FP32 matrix as 4 floats (zero past m)
  auto grow4 = [&](const float* gmat, int i, int j0) -> float4 {
    if (i >= m || j0 >= mr) return make_float4(0.f, 0.f, 0.f, 0.f);
    return *reinterpret_cast<const float4*>(gmat + (size_t)i * mr + j0);
  };
  // full MP x MP copy of a global FP32 matrix into a shared buffer (cp.async; zero padding)
  auto stage_full = [&](float* dst, const float* gmat) {
    constexpr int C4 = MP / 4;
    for (int e = tid; e < MP * C4; e += THREADS) {
      const int i = e / C4, c = e - i * C4;
      float* d = dst + i * LDF + 4 * c;
      if (i < m && 4 * c < mr) cp_async_16(d, gmat + (size_t)i * mr + 4 * c);
      else st4(d, 0.f, 0.f, 0.f, 0.f);
    }
    cp_async_commit();
  };
  // own-row tile -> rows of a full buffer (and the peer's copy)
  auto put_rows_full = [&](float* buf, const float (&v)[4][4]) {
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      float* p = buf + (ib + x) * LDF + jb;
      st4(p, v[x][0], v[x][1], v[x][2], v[x][3]);
      if constexpr (CL == 2) {
        float* q = peer + (p - sm);
        st4(q, v[x][0], v[x][1], v[x][2], v[x][3]);
      }
    }
  };
  // own-row tile -> own-column buffer, transposed: buf[(4 tb + y) LDO + 4 ta + x] = v[x][y]
  auto put_rows_T = [&](float* buf, const float (&v)[4][4]) {
#pragma unroll
    for (int y = 0; y < 4; ++y) st4(buf + (jb + y) * LDO + 4 * ta, v[0][y], v[1][y], v[2][y], v[3][y]);
  };
  // own-column tile (rows 4 tb + x, own columns 4 ta + y) -> own-column buffer
  auto put_cols = [&](float* buf, const float (&c)[4][4]) {
#pragma unroll
    for (int x = 0; x < 4; ++x) st4(buf + (jb + x) * LDO + 4 * ta, c[x][0], c[x][1], c[x][2], c[x][3]);
  };

  float om[4][4], dd[4][4], rr[4][4], pp[4][4];
  float dn_reg[ADAPTIVE ? 4 : 1][ADAPTIVE ? 4 : 1] = {};   // the adaptive preconditioner's denominators
  // preconditioner denominator of tile element (x, y): lambda_i + lambda_j, or the Hessian diagonal
  auto den = [&](int x, int y) -> float {
    if constexpr (ADAPTIVE) return dn_reg[x][y];
    else return lam[ib + x] + lam[jb + y];
  };
  // the gradient g = Je - Si of this thread's tile, from the global Je copy and this CTA's Si^T
  auto load_g = [&](float (&g)[4][4]) {
#pragma unroll
    for (int yy = 0; yy < 4; ++yy) {
      const float4 sit = ld4(Ss + G::OWNC + (jb + yy) * LDO + 4 * ta);
#pragma unroll
      for (int x = 0; x < 4; ++x) g[x][yy] = -comp(sit, x);
    }
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const float4 je = grow4(gJe, ib + x, jb);
#pragma unroll
      for (int yy = 0; yy < 4; ++yy) g[x][yy] += comp(je, yy);
    }
  };
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) om[x][y] = 0.0f;
  int iterations = 0, n_step = 0, n_hvp = 0, n_trial = 0, n_fallback = 0;
  const double sqrt_m = sqrt((double)m);
  const bool go = status_in == SSN_INSTANCE_CONVERGED;

  for (int step = 0; go && step < args.max_newton; ++step) {
    ++n_step;
    // ---- Sr, Si in this CTA's rows (registers sr, si), stored transposed into Ss
    float sr[4][4], si[4][4];
    if (step == 0) {
      // omega = 0: Sr = CrE, Si = Ce (dual_recommended_hvp.py:119-122, full rotated Gram)
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const float4 a = grow4(gCr, ib + x, jb), c = grow4(gCe, ib + x, jb);
        sr[x][0] = a.x; sr[x][1] = a.y; sr[x][2] = a.z; sr[x][3] = a.w;
        si[x][0] = c.x; si[x][1] = c.y; si[x][2] = c.z; si[x][3] = c.w;
      }
    } else {
      // Q = -omega P (:124): own rows, A = omega^T (own columns, in Zb), B = P
      put_rows_T(Zb, om);
      __syncthreads();
      {
        float q[1][4][4];
        const uint32_t A[1] = {saddr(Zb)};
        const uint32_t B[1] = {saddr(Pf)};
        outer_tc<1, 1, 1, coef_bit(0, 0, 0, 2), MP, false>(A, LDO, ta, B, LDF, tb, stg, q);
        put_rows_full(Qf, q[0]);
      }
      // the constant rotated Gram, staged for the sandwich
      stage_full(Yf, gCr);
      stage_full(Ss, gCe);
      cp_async_wait<0>();
      cl.sync();
      // Y = (P + iQ)(CrE + i Ce) in this CTA's rows; row segments of P^T = P and Q^T = -Q:
      //   Yr = P CrE - Q Ce = A0 B0 + A1 B1,  Yi = P Ce + Q CrE = A0 B1 - A1 B0
      float y[2][4][4];
      {
        const uint32_t A[2] = {saddr(Pf + r0), saddr(Qf + r0)};
        const uint32_t B[2] = {saddr(Yf), saddr(Ss)};
        constexpr uint32_t C = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1) | coef_bit(1, 0, 1, 1) |
                               coef_bit(1, 1, 0, 2);
        outer_tc<2, 2, 2, C, MP, false>(A, LDF, ta, B, LDF, tb, stg, y);
      }
      __syncthreads();                      // the staged Gram is consumed
      put_rows_T(Yf, y[0]);
      put_rows_T(Yf + G::OWNC, y[1]);
      __syncthreads();
      // S' = Y K^-H (recover_block on m x m, :70): Sr' = Yr P^T + Yi Q^T, Si' = Yi P^T - Yr Q^T;
      // B row segments: P^T -> P, Q^T -> -Q
      {
        const uint32_t A[2] = {saddr(Yf), saddr(Yf + G::OWNC)};
        const uint32_t B[2] = {saddr(Pf), saddr(Qf)};
        constexpr uint32_t C = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 2) | coef_bit(1, 1, 0, 1) |
                               coef_bit(1, 0, 1, 1);
        outer_tc<2, 2, 2, C, MP, false>(A, LDO, ta, B, LDF, tb, stg, y);
      }
      // Sr = sym(Sr'), Si = skew(Si') with the transposed entries from the CTA owning them:
      // this CTA's rows of Sr' in Xf, of Si' in Zb (own-row layout, leading dim LDF)
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        st4(Xf + (4 * ta + x) * LDF + jb, y[0][x][0], y[0][x][1], y[0][x][2], y[0][x][3]);
        st4(Zb + (4 * ta + x) * LDF + jb, y[1][x][0], y[1][x][1], y[1][x][2], y[1][x][3]);
      }
      cl.sync();
      {
        const int cj = jb / H;
        const bool mine = CL == 1 || cj == rank;
        const float* srcr = mine ? Xf : peer + G::O_X;
        const float* srci = mine ? Zb : peer + G::O_Z;
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
          const float4 tr = ld4(srcr + (jb + yy - cj * H) * LDF + ib);
          const float4 ti = ld4(srci + (jb + yy - cj * H) * LDF + ib);
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            sr[x][yy] = (y[0][x][yy] + comp(tr, x)) * 0.5f;
            si[x][yy] = (y[1][x][yy] - comp(ti, x)) * 0.5f;
          }
        }
      }
    }
    put_rows_T(Ss, sr);
    put_rows_T(Ss + G::OWNC, si);

    // ---- preconditioner denominators: lambda_i + lambda_j, or the Hessian diagonal (step > 0)
    if constexpr (ADAPTIVE) {
      if (step > 0) {
        // diag(P) from the full copy; diag(Sr) from each CTA's own rows, shared with the peer
        for (int i = tid; i < MP; i += THREADS) pdg[i] = Pf[i * LDF + i];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy)
            if (ib + x == jb + yy) {
              sdg[ib + x] = sr[x][yy];
              if constexpr (CL == 2) peer[G::O_SD + ib + x] = sr[x][yy];
            }
        cl.sync();
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) {
            const int i = ib + x, j = jb + yy;
            const int a0 = imin(i, j), b0 = imax(i, j);
            // the same expression for (i, j) and (j, i): Sr and Si are exactly (anti)symmetric,
            // P and Q are the same full copies in both CTAs, so den is exactly symmetric
            const float sab = sr[x][yy];
            const float iab = i <= j ? si[x][yy] : -si[x][yy];
            float dn = pdg[a0] * sdg[b0] + pdg[b0] * sdg[a0] - 2.0f * Pf[a0 * LDF + b0] * sab +
                       2.0f * Qf[a0 * LDF + b0] * iab;
            if (!(dn > 0.0f)) dn = lam[a0] + lam[b0];
            dn_reg[x][yy] = (i == j) ? 1.0f : dn;
          }
      } else {
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) dn_reg[x][yy] = lam[ib + x] + lam[jb + yy];
      }
    }

    // ---- gradient g = Je - Si, the residual ||g|| s / sqrt(m) (:126-128) and, in the same
    // reduction, <g, g / den> (the first CG step's rz, and minus the direct step's slope)
    double gn2, ggd;
    {
      float gg[4][4];
      load_g(gg);                                   // this thread's own Si^T entries: no barrier needed
      double v[2] = {0.0, 0.0};
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
          v[0] += (double)gg[x][yy] * gg[x][yy];
          v[1] += (double)gg[x][yy] * (gg[x][yy] / den(x, yy));
        }
      cl.sumv(v);
      gn2 = v[0];
      ggd = v[1];
    }
    const double gnorm = sqrt(gn2);
    const double residual = gnorm * s / sqrt_m;
    if (!(residual >= args.switch_tol)) break;      // converged far enough for FP32, or non-finite
    // stalled: on ill-conditioned targets the FP32 residual can have a floor above switch_tol;
    // three steps without a new best residual, or half the Newton cap spent, hand over to the
    // FP64 iteration.  Every thread reads the same bookkeeping (slot step & 1, written by
    // thread 0 one step earlier, many barriers ago) and both CTAs hold the same FP64 sums,
    // so all leave together.
    {
      const int par = step & 1;
      const bool better = (float)residual < s_best[par];
      const int since = better ? 0 : s_since[par] + 1;
      if (threadIdx.x == 0) {
        s_best[par ^ 1] = better ? (float)residual : s_best[par];
        s_since[par ^ 1] = since;
      }
      if (since >= 3 || 2 * step >= args.max_newton) break;
    }
    ++iterations;

    // ---- search direction (:137-164); g, r, d, p are exactly antisymmetric, den symmetric
    double slope;
    if (step == 0) {
      // one preconditioner application solves H(E) = E L + L E exactly (:138-140)
      load_g(dd);
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) dd[x][yy] = -dd[x][yy] / den(x, yy);
      slope = -ggd;
    } else {
      // PCG (:142-161), r = -g, z = r / den, p = z; one fused reduction per iteration: with
      // c = <p, Hp>, alpha = rz / c, the next ||r||^2 and <r, z> follow from <r, Hp>,
      // <Hp, Hp>, <z, Hp> and <Hp, Hp / den> (FP64 sums of the FP32 vectors)
      double rz = ggd, rn2 = gn2;
      load_g(rr);
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
          rr[x][yy] = -rr[x][yy];
          pp[x][yy] = rr[x][yy] / den(x, yy);
          dd[x][yy] = 0.0f;
        }
      const double tol = fmin(fmax(sqrt(residual), 1e-8), 0.1) * gnorm;
      for (int it = 0; it < args.max_cg; ++it) {
        put_rows_full(Xf, pp);
        cl.sync();
        // W1 = p Sr, W2 = p Si in this CTA's columns: A row segments p^T = -p; B row segments
        // Sr[k][j] = Sr^T rows (+), Si[k][j] = -(Si^T rows) (-), so W1 takes -, W2 takes +
        {
          float w[2][4][4];
          const uint32_t A[1] = {saddr(Xf)};
          const uint32_t B[2] = {saddr(Ss), saddr(Ss + G::OWNC)};
          constexpr uint32_t C = coef_bit(0, 0, 0, 2) | coef_bit(1, 0, 1, 1);
          outer_tc<1, 2, 2, C, MP, true, false>(A, LDF, tb, B, LDO, ta, stg, w);
          put_cols(Yf, w[0]);
          put_cols(Yf + G::OWNC, w[1]);
        }
        __syncthreads();
        // Z = P W1 - Q W2 in this CTA's columns (A row segments P^T = P, Q^T = -Q)
        float z[1][4][4];
        {
          const uint32_t A[2] = {saddr(Pf), saddr(Qf)};
          const uint32_t B[2] = {saddr(Yf), saddr(Yf + G::OWNC)};
          constexpr uint32_t C = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1);
          outer_tc<2, 2, 1, C, MP, true, false>(A, LDF, tb, B, LDO, ta, stg, z);
          put_cols(Zb, z[0]);
        }
        cl.sync();
        ++n_hvp;
        // Hp = Z - Z^T in this CTA's rows: Z[i][j] from the CTA owning column j, Z[j][i] is
        // this thread's own column tile transposed
        float hp[4][4];
        {
          const int cj = jb / H;
          const float* src = (CL == 1 || cj == rank) ? Zb : peer + G::O_Z;
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            const float4 zr = ld4(src + (ib + x) * LDO + (jb - cj * H));
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) hp[x][yy] = comp(zr, yy) - z[0][yy][x];
          }
        }
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) {
            const double h = hp[x][yy], hd = hp[x][yy] / den(x, yy);
            v[0] += (double)pp[x][yy] * h;
            v[1] += (double)rr[x][yy] * h;
            v[2] += h * h;
            v[3] += (double)rr[x][yy] * hd;
            v[4] += h * hd;
          }
        cl.sumv(v);
        const double curv = v[0];
        if (!(curv > 0.0)) break;                   // cg_active &= curvature > 0 (:152)
        const double al = rz / curv;
        const float alpha = (float)al;
        const double rn2_next = rn2 - 2.0 * al * v[1] + al * al * v[2];
        const double rz_next = rz - 2.0 * al * v[3] + al * al * v[4];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) {
            dd[x][yy] = fmaf(alpha, pp[x][yy], dd[x][yy]);
            rr[x][yy] = fmaf(-alpha, hp[x][yy], rr[x][yy]);
          }
        if (!(sqrt(fmax(rn2_next, 0.0)) > tol)) break;   // (:155-157)
        const float beta = (float)(rz_next / rz);
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) pp[x][yy] = fmaf(beta, pp[x][yy], rr[x][yy] / den(x, yy));
        rz = rz_next;
        rn2 = rn2_next;
      }
      double sl[1] = {0.0};
      load_g(rr);                                   // r is no longer needed: g into its registers
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) sl[0] += (double)rr[x][yy] * dd[x][yy];
      cl.sumv(sl);
      slope = sl[0];
      if (slope >= 0.0) {                           // non-descent fallback (:163-164)
        ++n_fallback;
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) dd[x][yy] = -rr[x][yy] / den(x, yy);
        slope = -ggd;
      }
    }

    // ---- Armijo backtracking with the exact change (:166-190).  With delta = t d:
    //   change = t <g, d> + t^2 <P_t d, d Sr + W_t (d Si)>,
    // where d Sr and d Si do not depend on t and are formed once.
    put_rows_full(Xf, dd);
    cl.sync();
    {
      float w[2][4][4];
      const uint32_t A[1] = {saddr(Xf)};
      const uint32_t B[2] = {saddr(Ss), saddr(Ss + G::OWNC)};
      constexpr uint32_t C = coef_bit(0, 0, 0, 2) | coef_bit(1, 0, 1, 1);
      outer_tc<1, 2, 2, C, MP, true, false>(A, LDF, tb, B, LDO, ta, stg, w);
      put_cols(Yf, w[0]);                           // d Sr  (this CTA's columns)
      put_cols(Yf + G::OWNC, w[1]);                 // d Si
    }
    float* Ub = Zb;                                 // [16][LDF] pivot-row panel of the inverse
    float* Xb = Zb + 16 * LDF;                      // [16][LDF] pivot columns, transposed
    float t = 1.0f;
    bool accepted = false;
    for (int bt = 0; bt < args.max_backtrack; ++bt) {
      ++n_trial;
      float wt[4][4];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) wt[x][yy] = fmaf(t, dd[x][yy], om[x][yy]);
      put_rows_full(Qf, wt);
      cl.sync();
      // K = I + W_t W_t: this CTA's rows (A row segments W_t^T = -W_t), written into the full
      // copy Pf of both CTAs (P is not needed in the line search)
      {
        float k[1][4][4];
        const uint32_t A[1] = {saddr(Qf + r0)};
        const uint32_t B[1] = {saddr(Qf)};
        outer_tc<1, 1, 1, coef_bit(0, 0, 0, 2), MP, false>(A, LDF, ta, B, LDF, tb, stg, k);
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy)
            if (ib + x == jb + yy) k[0][x][yy] += 1.0f;
        put_rows_full(Pf, k[0]);
      }
      // U3 = W_t (d Si) in this CTA's columns (A row segments W_t^T = -W_t)
      float u3[1][4][4];
      {
        const uint32_t A[1] = {saddr(Qf)};
        const uint32_t B[1] = {saddr(Yf + G::OWNC)};
        outer_tc<1, 1, 1, coef_bit(0, 0, 0, 2), MP, true, false>(A, LDF, tb, B, LDO, ta, stg, u3);
      }
      cl.sync();                                    // K complete in both CTAs
      // Positive-definiteness test and inverse: Gauss-Jordan over 16-wide pivot blocks on the
      // whole K in every CTA (the same arithmetic on the same bits: the same inverse and the
      // same outcome in both, with no cluster barrier per block).  The pivots are the Schur-
      // complement diagonals, all positive exactly when K is positive definite (the test
      // cholesky_ex applies).
      bool valid = true;
      for (int kb = 0; kb < MP; kb += 16) {
        if (warp == 0) {
          // the 16 x 16 pivot block in registers: lane (i, h) holds row i, columns 8h..8h+7;
          // pivot row, a_ik and pivot broadcast by shuffles
          const int i = lane & 15, h = lane >> 4;
          float rw[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) rw[jj] = Pf[(kb + i) * LDF + kb + 8 * h + jj];
          bool ok = true;
#pragma unroll
          for (int kk = 0; kk < 16; ++kk) {
            const int hk = kk >> 3, ck = kk & 7;
            const float piv = __shfl_sync(0xffffffffu, rw[ck], kk + 16 * hk);
            const float aik = __shfl_sync(0xffffffffu, rw[ck], i + 16 * hk);
            float rowk[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) rowk[jj] = __shfl_sync(0xffffffffu, rw[jj], kk + 16 * h);
            ok = ok & (piv > 0.0f) & (piv < INFINITY);
            const float inv = rcp_nr(piv);
            const float mik = aik * inv;            // the row multiplier: one rounding on the chain
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const bool colk = (h == hk) && (jj == ck);
              float v;
              if (i == kk) v = colk ? inv : rowk[jj] * inv;
              else if (colk) v = -mik;
              else v = fmaf(-mik, rowk[jj], rw[jj]);
              rw[jj] = v;
            }
          }
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) Ub[i * LDF + kb + 8 * h + jj] = rw[jj];
          ok = __all_sync(0xffffffffu, ok);
          if (lane == 0) flags[0] = ok ? 1 : 0;
        }
        __syncthreads();
        if (flags[0] == 0) {
          valid = false;
          break;
        }
        // U = Dinv K[pivot rows][:] outside the pivot block; X = K[:][pivot columns] (old)
        {
          constexpr int C4 = MP / 4;
          for (int e = tid; e < 16 * C4; e += THREADS) {
            const int p = e / C4, j0 = 4 * (e - p * C4);
            if (j0 >= kb && j0 < kb + 16) continue;
            float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const float dq = Ub[p * LDF + kb + q];
              const float4 kq = ld4(Pf + (kb + q) * LDF + j0);
              a0 = fmaf(dq, kq.x, a0);
              a1 = fmaf(dq, kq.y, a1);
              a2 = fmaf(dq, kq.z, a2);
              a3 = fmaf(dq, kq.w, a3);
            }
            st4(Ub + p * LDF + j0, a0, a1, a2, a3);
          }
          for (int e = tid; e < 4 * MP; e += THREADS) {
            const int i = e >> 2, c = e & 3;
            const float4 xv = ld4(Pf + i * LDF + kb + 4 * c);
            Xb[(4 * c + 0) * LDF + i] = xv.x;
            Xb[(4 * c + 1) * LDF + i] = xv.y;
            Xb[(4 * c + 2) * LDF + i] = xv.z;
            Xb[(4 * c + 3) * LDF + i] = xv.w;
          }
        }
        __syncthreads();
        // every element is read and rewritten by one thread: K[i][j] = U[i - kb][j] on the pivot
        // rows, else K[i][j] - X_i U[:, j], the pivot columns (U = Dinv there) starting from 0
#pragma unroll
        for (int hh = 0; hh < CL; ++hh) {
          const int i0 = hh * H + 4 * ta;
          const bool prow = i0 >= kb && i0 < kb + 16;
          const bool pcol = jb >= kb && jb < kb + 16;
          float acc[4][4];
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            const float4 base = prow ? ld4(Ub + (i0 + x - kb) * LDF + jb)
                                     : (pcol ? make_float4(0.f, 0.f, 0.f, 0.f) : ld4(Pf + (i0 + x) * LDF + jb));
            acc[x][0] = base.x; acc[x][1] = base.y; acc[x][2] = base.z; acc[x][3] = base.w;
          }
          if (!prow) {
#pragma unroll 4
            for (int q = 0; q < 16; ++q) {
              const float4 xv = ld4(Xb + q * LDF + i0);
              const float4 uv = ld4(Ub + q * LDF + jb);
#pragma unroll
              for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int yy = 0; yy < 4; ++yy) acc[x][yy] = fmaf(-comp(xv, x), comp(uv, yy), acc[x][yy]);
            }
          }
#pragma unroll
          for (int x = 0; x < 4; ++x) st4(Pf + (i0 + x) * LDF + jb, acc[x][0], acc[x][1], acc[x][2], acc[x][3]);
        }
        __syncthreads();
      }
      if (valid) {
        // tail = <P_t d, d Sr + W_t (d Si)> over this CTA's columns (line_change, hvp_fused.cu:259-371)
        float v[1][4][4];
        {
          const uint32_t A[1] = {saddr(Pf)};
          const uint32_t B[1] = {saddr(Xf + r0)};
          outer_tc<1, 1, 1, coef_bit(0, 0, 0, 1), MP, true, false>(A, LDF, tb, B, LDF, ta, stg, v);
        }
        double tail[1] = {0.0};
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const float4 dsr = ld4(Yf + (jb + x) * LDO + 4 * ta);
#pragma unroll
          for (int yy = 0; yy < 4; ++yy) tail[0] += (double)v[0][x][yy] * (comp(dsr, yy) + u3[0][x][yy]);
        }
        cl.sumv(tail);
        const double td = (double)t;
        const double change = td * slope + td * td * tail[0];
        if (change <= 1e-4 * td * slope) {
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) om[x][yy] = wt[x][yy];
          accepted = true;
          break;
        }
      }
      t *= 0.5f;
    }
    if (!accepted) break;             // the FP64 phase continues from the last accepted omega
  }

  // ---- omega (working basis) and the counts for the FP64 phase
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int yy = 0; yy < 4; ++yy) {
      const int i = ib + x, j = jb + yy;
      if (i < m && j < m) Wout[(size_t)i * m + j] = (double)om[x][yy];
    }
  if (tid == 0 && rank == 0) {
    aux[0] = iterations;
    aux[1] = n_step;
    aux[2] = n_hvp;
    aux[3] = n_trial;
    aux[4] = n_fallback;
  }
  if constexpr (CL == 2) cg::this_cluster().sync();   // no CTA leaves while its peer may read its shared memory
}

template <int MB, int CL, bool ADAPTIVE>
static cudaError_t launch_dual32_mb(const Dual32Args& args, int batch, cudaStream_t stream) {
  using G = G32<MB, CL>;
  const size_t smem = G::bytes();
  cudaError_t err = cudaFuncSetAttribute(dual32_kernel<MB, CL, ADAPTIVE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(batch * CL);
  cfg.blockDim = dim3(G::THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, dual32_kernel<MB, CL, ADAPTIVE>, args);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// The FP32 phase runs where its state fits on chip: m <= 64 with one CTA or a cluster,
// 64 < m <= 96 with a 2-CTA cluster.
bool dual32_supported(int m, int cluster) {
  const int mb = bucket_of(m);
  return mb <= 2 || (mb == 3 && cluster == 2);
}

template <bool ADAPTIVE>
static cudaError_t launch_dual32_t(const Dual32Args& args, int batch, int cluster, cudaStream_t stream) {
  switch (bucket_of(args.m)) {
    case 1: return launch_dual32_mb<1, 1, ADAPTIVE>(args, batch, stream);
    case 2: return cluster == 2 ? launch_dual32_mb<2, 2, ADAPTIVE>(args, batch, stream)
                                : launch_dual32_mb<2, 1, ADAPTIVE>(args, batch, stream);
    case 3: return cluster == 2 ? launch_dual32_mb<3, 2, ADAPTIVE>(args, batch, stream) : cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_dual32(const Dual32Args& args, int batch, int cluster, cudaStream_t stream) {
  return args.adaptive ? launch_dual32_t<true>(args, batch, cluster, stream)
                       : launch_dual32_t<false>(args, batch, cluster, stream);
}

}  // namespace ssn
