// ssn_dual.cu -- persistent FP64 dual Newton-CG kernel (one CTA per instance).
//
// Replaces dual_batch (src/symplectic_projection/dual_recommended_hvp.py:99-191)
// and, through it, the reference kernels hvp_inner / hvp_outer* /
// hvp_sandwich_front / hvp_line_partial / hvp_line_finish / hvp_precondition /
// hvp_cg_update / hvp_cg_next (hvp_fused.cu), recover_fused on m x m operands
// (recovery_fused.cu) and the torch cholesky_ex / cholesky_solve calls.
//
// The whole Newton loop of an instance -- sandwich, gradient, PCG with HVPs,
// non-descent fallback, Armijo backtracking with the exact objective change,
// positive-definiteness test and inverse of the trial -- runs inside one CTA
// with no host synchronisation: every convergence / acceptance decision comes
// from a deterministic CTA reduction, so all threads branch identically.  The
// per-instance m x m state lives in an L2-resident workspace; products stream
// 16-wide K-panels into shared memory and run on DMMA fragments.
//
// Semantics per instance match the batched reference: instances are
// independent there too (masks only), so per-instance exit is equivalent.
#include <float.h>
#include <math.h>

#include <cooperative_groups.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace cg = cooperative_groups;

namespace ssn {

enum Mat {
  M_CE = 0, M_JE, M_W, M_WT, M_P, M_PT, M_Q, M_SR, M_SI, M_G, M_D, M_R, M_PP, M_HP, M_DL,
  M_T1, M_T2, M_T3, M_X0, M_X1, M_X2, M_DEN, M_AUX
};
static_assert(M_AUX + 1 == kDualMats, "workspace matrix count");
// The FP32 phase (ssn_dual32.cu) reads the set-up from, and writes its omega and counters
// to, these slots; it uses M_T1..M_T3 as scratch.
static_assert(M_CE == 0 && M_JE == 1 && M_W == 2 && M_T1 == 15 && M_X2 == 20 && M_AUX == 22,
              "slots shared with the FP32 phase");

constexpr uint32_t C_ONE = coef_bit(0, 0, 0, 1);
constexpr uint32_t C_SHARED_B = coef_bit(0, 0, 0, 1) | coef_bit(1, 1, 0, 1);
constexpr uint32_t C_SHARED_A = coef_bit(0, 0, 0, 1) | coef_bit(1, 0, 1, 1);
constexpr uint32_t C_DIFF = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 2);
constexpr uint32_t C_CPLX = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1) | coef_bit(1, 1, 0, 1) |
                            coef_bit(1, 0, 1, 2);
// (P + iQ)(C + iE): out0 = P C - Q E, out1 = P E + Q C
constexpr uint32_t C_SANDF = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 2) | coef_bit(1, 0, 1, 1) |
                             coef_bit(1, 1, 0, 1);
// out0 = A0 B0 + A1 B1
constexpr uint32_t C_SHARED_SUM = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1);

// Warp-tile shape of a CL-way row split for bucket MB: each CTA computes at most
// round_up(32*MB / CL, 8) rows of every m x m product.
template <int MB, int CL, int NOUT>
struct SplitTile {
  static constexpr int WC = MB;
  static constexpr int WR = CL == 1 ? Tile<MB, NOUT>::WR : imax(1, cdiv(16 * MB, 32));
};

// The CTAs that work on one instance: CL = 1 (one CTA) or CL = 2 (a thread-block
// cluster splitting every m x m product and pass by rows).  sync() is the phase
// barrier; sum() is a CTA reduction followed, for CL = 2, by a fixed-order sum of
// the two CTA partials exchanged through distributed shared memory, so both
// CTAs obtain identical bits and branch identically.
template <int CL>
struct Team {
  int rank, r0, r1;       // rows [r0, r1) of every m x m matrix belong to this CTA
  double* red;            // 2*kWarps doubles (CTA reduction)
  double* xch;            // [2 parities][2 values][CL ranks] exchange slots (local)
  double* xch_peer;       // the same slots in the peer CTA (CL = 2)
  int parity;

  __device__ __forceinline__ void sync() {
    if constexpr (CL == 1) {
      __syncthreads();
    } else {
      cg::this_cluster().sync();
    }
  }
  __device__ __forceinline__ void sum2(double& a, double& b) {
    block_sum2(a, b, red);
    if constexpr (CL == 2) {
      double* slot = xch + parity * 4;
      double* peer = xch_peer + parity * 4;
      if (threadIdx.x == 0) {
        slot[rank] = a;
        slot[2 + rank] = b;
        peer[rank] = a;
        peer[2 + rank] = b;
      }
      cg::this_cluster().sync();
      a = slot[0] + slot[1];
      b = slot[2] + slot[3];
      parity ^= 1;
    }
  }
  __device__ __forceinline__ double sum(double a) {
    double b = 0.0;
    sum2(a, b);
    return a;
  }
};

// Panel staging of the Newton kernel's products: A slots hold the rows of one CTA
// (half of m for CL = 2), B slots all m columns; as many stages (up to 4) as fit
// in 200 KB, since the operands come from L2 and the panel latency must be hidden.
__host__ __device__ constexpr int dual_slot_a(int MB, int CL) { return panel_slot(CL == 2 ? 16 * MB : 32 * MB); }
__host__ __device__ constexpr int dual_slot_b(int MB) { return panel_slot(32 * MB); }
__host__ __device__ constexpr int dual_stages(int MB, int CL) {
  return imax(2, imin(4, 25600 / (2 * dual_slot_a(MB, CL) + 2 * dual_slot_b(MB))));
}
__host__ __device__ constexpr int dual_region_doubles(int MB, int CL) {
  return imax(dual_stages(MB, CL) * (2 * dual_slot_a(MB, CL) + 2 * dual_slot_b(MB)), spd_region_doubles(32 * MB));
}

template <int MB, int CL>
struct Dual {
  int m;
  double* smem;
  int r0, rows;

  // rows [r0, r0 + rows) of sum_{a,b} +-op(A_a) op(B_b); epi gets global row indices
  template <int NA, int NB, int NOUT, uint32_t COEF, class Epi>
  __device__ __forceinline__ void mul(const MatOp (&A)[NA], const MatOp (&B)[NB], Epi& epi) const {
    using TL = SplitTile<MB, CL, NOUT>;
    MatOp As[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      As[a] = A[a];
      As[a].ptr = A[a].trans ? A[a].ptr + r0 : A[a].ptr + (size_t)r0 * A[a].ld;
    }
    const int off = r0;
    auto shifted = [&](int o, int i, int j, double v) { epi(o, i + off, j, v); };
    ssn::tile_product_staged<TL::WR, TL::WC, NA, NB, NOUT, COEF, dual_stages(MB, CL)>(
        As, B, rows, m, m, smem, dual_slot_a(MB, CL), dual_slot_b(MB), shifted);
  }

  // All m rows by this CTA alone, in 32-row passes so that the A panels fit the A
  // slots (sized for this CTA's own rows, >= 32 for every bucket a cluster runs).
  // Each output entry sees the same DMMA sequence as in mul, so the same bits.
  template <int NA, int NB, int NOUT, uint32_t COEF, class Epi>
  __device__ __forceinline__ void mul_all(const MatOp (&A)[NA], const MatOp (&B)[NB], Epi& epi) const {
    static_assert(CL == 1 || MB >= 2, "A slots hold at least 32 rows");
    ssn::tile_product_staged<1, MB, NA, NB, NOUT, COEF, dual_stages(MB, CL)>(
        A, B, m, m, m, smem, dual_slot_a(MB, CL), dual_slot_b(MB), epi);
  }
};

// Element loops over this CTA's rows without integer division: warp w owns rows
// r0 + w, r0 + w + 16, ..., lane l owns columns l, l+32, ...
#define SSN_FOR_IJ(T_, m_, BODY)                                                      \
  for (int i = (T_).r0 + (int)(threadIdx.x >> 5); i < (T_).r1; i += kWarps)          \
    for (int j = (int)(threadIdx.x & 31); j < (m_); j += 32) {                        \
      const int e = i * (m_) + j;                                                     \
      (void)e;                                                                        \
      BODY                                                                            \
    }

// The same element order, with every operand of a group of rows per warp
// loaded before any element is used: load(i, j, e) returns the operands of
// (i, j) (a scalar or a small struct), use(i, j, e, operands) computes and
// stores.  The working matrices live in L2, and a loop that loads, stores and
// loads again pays one L2 round trip per element; batching the loads pays one
// per group.  The visiting order, and so every per-thread partial sum, is that
// of SSN_FOR_IJ.
template <int CPL, class Team_, class Load, class Use>
__device__ __forceinline__ void each_ij(const Team_& tm, int m, Load&& load, Use&& use) {
  using V = decltype(load(0, 0, 0));
  // rows per group: about 18 doubles of operands per thread, so the group stays in registers
  constexpr int QG = imax(1, imin(3, 6 / (int)(sizeof(V) / sizeof(double))));
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  for (int i0 = tm.r0 + warp; i0 < tm.r1; i0 += QG * kWarps) {
    V v[QG][CPL];
#pragma unroll
    for (int q = 0; q < QG; ++q)
#pragma unroll
      for (int p = 0; p < CPL; ++p) {
        // out-of-range slots load a valid element (never used), so every slot is defined
        const int i = imin(i0 + q * kWarps, tm.r1 - 1), j = imin(lane + 32 * p, m - 1);
        v[q][p] = load(i, j, i * m + j);
      }
#pragma unroll
    for (int q = 0; q < QG; ++q)
#pragma unroll
      for (int p = 0; p < CPL; ++p) {
        const int i = i0 + q * kWarps, j = lane + 32 * p;
        if (i < tm.r1 && j < m) use(i, j, i * m + j, v[q][p]);
      }
  }
}

struct D2 { double x, y; };
struct D3 { double x, y, z; };
struct D4 { double x, y, z, w; };
struct D5 { double x, y, z, w, u; };
struct D6 { double x, y, z, w, u, d; };

template <int MB, int CL>
__global__ void __launch_bounds__(kThreads, 1) dual_kernel(DualArgs a) {
  extern __shared__ __align__(16) double smem[];
  const int m = a.m, mm = m * m;
  const int rank = CL == 1 ? 0 : (int)cg::this_cluster().block_rank();
  const int inst = blockIdx.x / CL;
  constexpr int region = dual_region_doubles(MB, CL);
  double* red = smem + region;                // 2*kWarps doubles
  double* lam = red + 2 * kWarps;             // kMaxM doubles
  double* pdg = lam + kMaxM;                  // kMaxM doubles: diag(P) (adaptive preconditioner)
  double* sdg = pdg + kMaxM;                  // kMaxM doubles: diag(Sr)
  double* xch = sdg + kMaxM;                  // 8 doubles
  int* flag = reinterpret_cast<int*>(xch + 8);
  int* vflag = flag + 1;                      // cluster: the trial inverse's outcome, written by CTA 0
  int* vflag_peer = vflag;
  int* perm_col = flag + 2;                   // kMaxM: permutation basis, V[perm_col[a]][a] = 1
  int* perm_row = perm_col + kMaxM;           // kMaxM: V[r][perm_row[r]] = 1
  double* Zs = smem;                          // this CTA's rows of the HVP outer product
  const int zld = m + 1;

  const int half = round_up(cdiv(m, CL), 8);
  Team<CL> team;
  team.rank = rank;
  team.r0 = imin(m, rank * half);
  team.r1 = imin(m, (rank + 1) * half);
  team.red = red;
  team.xch = xch;
  team.xch_peer = xch;
  team.parity = 0;
  const double* Zpeer = Zs;
  int peer_r0 = 0;
  if constexpr (CL == 2) {
    team.xch_peer = cg::this_cluster().map_shared_rank(xch, rank ^ 1);
    Zpeer = cg::this_cluster().map_shared_rank(Zs, rank ^ 1);
    vflag_peer = cg::this_cluster().map_shared_rank(vflag, rank ^ 1);
    peer_r0 = imin(m, (rank ^ 1) * half);
  }
  Dual<MB, CL> eng{m, smem, team.r0, team.r1 - team.r0};
  // Z(j, i) for any row j: this CTA's rows from local shared memory, the others from the peer's
  auto zval = [&](int j, int i) -> double {
    if (CL == 1 || (j >= team.r0 && j < team.r1)) return Zs[(j - team.r0) * zld + i];
    return Zpeer[(j - peer_r0) * zld + i];
  };

  double* ws = a.work + (size_t)inst * kDualMats * mm;
  const double* Ci = a.Ci + (size_t)inst * mm;
  const double* V = a.vectors + (size_t)inst * mm;
  const double s = a.scale[inst];
  int status = a.eig_status ? a.eig_status[inst] : SSN_INSTANCE_CONVERGED;
  for (int i = threadIdx.x; i < m; i += kThreads) lam[i] = a.values[(size_t)inst * m + i];
  __syncthreads();

  double* Ce = ws + (size_t)M_CE * mm;
  double* Je = ws + (size_t)M_JE * mm;
  double* Wm = ws + (size_t)M_W * mm;
  double* Wt = ws + (size_t)M_WT * mm;
  double* Pm = ws + (size_t)M_P * mm;
  double* Pt = ws + (size_t)M_PT * mm;
  double* Qm = ws + (size_t)M_Q * mm;
  double* Sr = ws + (size_t)M_SR * mm;
  double* Si = ws + (size_t)M_SI * mm;
  double* G = ws + (size_t)M_G * mm;
  double* Dd = ws + (size_t)M_D * mm;
  double* Rr = ws + (size_t)M_R * mm;
  double* Pp = ws + (size_t)M_PP * mm;
  double* Dl = ws + (size_t)M_DL * mm;
  double* T1 = ws + (size_t)M_T1 * mm;
  double* T2 = ws + (size_t)M_T2 * mm;
  double* T3 = ws + (size_t)M_T3 * mm;
  double* Kg = ws + (size_t)M_X0 * mm;        // K = I + trial trial, staged through L2 for CL = 2
  double* Dn = ws + (size_t)M_DEN * mm;       // adaptive preconditioner denominators (this CTA's rows)
  const bool adaptive = a.adaptive_precond != 0;

  auto store_to = [&](double* dst) {
    return [dst, m](int, int i, int j, double v) { dst[i * m + j] = v; };
  };

  int64_t iterations = 0;
  int n_hvp = 0, n_trial = 0, n_fallback = 0, n_step = 0;
  const int32_t* aux = reinterpret_cast<const int32_t*>(ws + (size_t)M_AUX * mm);   // the FP32 phase's counts
  if (status == SSN_INSTANCE_CONVERGED) {
    double* CrE = ws + (size_t)M_X2 * mm;       // approximate basis: sym(V^T (Cr/s) V)
    const bool approx = a.approx_basis != 0;
    // (the same bits for both CTAs of a cluster, so both take the same branch and barriers)
    const bool refine_basis = a.approx_basis && a.orthogonalize && !(a.sweeps && a.sweeps[inst] == 0);
    // A basis from no Jacobi sweep is a permutation (the identity in eigenvalue order), exact
    // in FP64: the basis changes of the set-up and the exit are then gathers, not products.
    const bool perm = a.sweeps && a.sweeps[inst] == 0;
    if (perm) {
      for (int r = threadIdx.x; r < m; r += kThreads) {
        int c = 0;
        for (int j = 0; j < m; ++j)
          if (V[(size_t)r * m + j] != 0.0) c = j;
        perm_row[r] = c;
        perm_col[c] = r;
      }
      __syncthreads();
    }
    if (a.phase == 2) {
      // the set-up of the phase-1 launch is in the workspace: Ce, Je, CrE (and Sr = CrE),
      // the refined basis in M_X1; omega, P = I, Q = 0 (omega since rewritten by the FP32 phase)
      if (refine_basis) V = ws + (size_t)M_X1 * mm;
      if (approx) {
        for (int i = threadIdx.x; i < m; i += kThreads) lam[i] = CrE[i * m + i];
        __syncthreads();
      }
    } else if (perm) {
      // V^T X V = X[c][c'] with c = perm_col: the same values the products give, gathered.
      // J(V)[r][b] = V[r + h][b] (r < h) or -V[r - h][b], so (V^T J(V))[a][b] = +-1 where
      // b = perm_row[perm_col[a] +- h].
      const int h = m / 2;
      const double* Crb = a.Cr + (size_t)inst * mm;
      auto jv = [&](int a0, int b0) -> double {
        const int r = perm_col[a0];
        return r < h ? (perm_row[r + h] == b0 ? 1.0 : 0.0) : (perm_row[r - h] == b0 ? -1.0 : 0.0);
      };
      SSN_FOR_IJ(team, m, {
        const int pa = perm_col[i];
        const int pb = perm_col[j];
        Ce[e] = (Ci[pa * m + pb] / s - Ci[pb * m + pa] / s) / 2;
        Je[e] = ((jv(i, j) - jv(j, i)) / 2) / s;
        if (approx) {
          const double c = (Crb[pa * m + pb] / s + Crb[pb * m + pa] / s) / 2;
          CrE[e] = c;
          Sr[e] = c;
        } else {
          Sr[e] = (i == j) ? lam[i] : 0.0;
        }
        Wm[e] = 0.0;
        Pm[e] = (i == j) ? 1.0 : 0.0;
        Qm[e] = 0.0;
      })
      team.sync();
      if (approx) {
        for (int i = threadIdx.x; i < m; i += kThreads) lam[i] = CrE[i * m + i];
        __syncthreads();
      }
    } else {
    // ---- eigenbasis set-up: Ce = skew(V^T (Ci/s) V), Je = skew(V^T J(V)) / s  (:106-111, :53-56)
    const int h = m / 2;
    if (refine_basis) {
      // V <- V (3I - V^T V) / 2 twice: vectors from FP32 rotations become orthogonal to FP64 rounding
      double* Vb[2] = {ws + (size_t)M_X2 * mm, ws + (size_t)M_X1 * mm};
      const double* Vin = V;
      for (int it = 0; it < 2; ++it) {
        {
          MatOp A[1] = {op_t(Vin, m)};
          MatOp B[1] = {op_n(Vin, m)};
          auto epi = store_to(T1);
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        team.sync();
        double* Vout = Vb[it];
        {
          MatOp A[1] = {op_n(Vin, m)};
          MatOp B[1] = {op_n(T1, m)};
          auto epi = [&](int, int i, int j, double v) {
            const int e = i * m + j;
            Vout[e] = 1.5 * Vin[e] - 0.5 * v;
          };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        team.sync();
        Vin = Vout;
      }
      V = Vin;                                  // == M_X1
    }
    each_ij<MB>(team, m, [&](int i, int j, int e) { return D2{Ci[e], V[(i < h ? i + h : i - h) * m + j]}; },
        [&](int i, int, int e, const D2& v) {
          T1[e] = v.x / s;
          T3[e] = i < h ? v.y : -v.y;
        });
    team.sync();
    if (a.approx_basis) {
      double* Kt = ws + (size_t)M_X0 * mm;
      const double* Crb = a.Cr + (size_t)inst * mm;
      {
        MatOp A[1] = {op_t(V, m)};
        MatOp B[2] = {op_n(T1, m), op_n(Crb, m)};
        auto epi = [&](int o, int i, int j, double v) {
          if (o == 0) T2[i * m + j] = v;
          else Kt[i * m + j] = v / s;
        };
        eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
      }
      __syncthreads();
      {
        MatOp A[1] = {op_t(V, m)};
        MatOp B[1] = {op_n(T3, m)};
        auto epi = store_to(Dl);
        eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
      }
      team.sync();
      {
        MatOp A[2] = {op_n(T2, m), op_n(Kt, m)};
        MatOp B[1] = {op_n(V, m)};
        auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T3)[i * m + j] = v; };
        eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
      }
      team.sync();
      SSN_FOR_IJ(team, m, {
        const int et = j * m + i;
        const double c = (T3[e] + T3[et]) / 2;
        CrE[e] = c;
        Sr[e] = c;
      })
      team.sync();
      for (int i = threadIdx.x; i < m; i += kThreads) lam[i] = CrE[i * m + i];
    } else {
      {
        MatOp A[1] = {op_t(V, m)};
        MatOp B[2] = {op_n(T1, m), op_n(T3, m)};
        auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T2 : Dl)[i * m + j] = v; };
        eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
      }
      team.sync();
      {
        MatOp A[1] = {op_n(T2, m)};
        MatOp B[1] = {op_n(V, m)};
        auto epi = store_to(T1);
        eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
      }
      team.sync();
    }
    // Skew parts are exactly antisymmetric ((x - y)/2 vs (y - x)/2), which every
    // later pass relies on: precondition(r) = r / den and skew(w + t d) = w + t d
    // hold bit for bit for exactly skew r, w, d.
    each_ij<MB>(team, m,
        [&](int i, int j, int e) {
          const int et = j * m + i;
          return D4{T1[e], T1[et], Dl[e], Dl[et]};
        },
        [&](int i, int j, int e, const D4& v) {
          Ce[e] = (v.x - v.y) / 2;
          Je[e] = ((v.z - v.w) / 2) / s;
          Wm[e] = 0.0;
          Pm[e] = (i == j) ? 1.0 : 0.0;
          Qm[e] = 0.0;
          if (!approx) Sr[e] = (i == j) ? lam[i] : 0.0;
        });
    team.sync();
    }
    if (a.phase == 1) {
      if constexpr (CL == 2) cg::this_cluster().sync();   // no CTA leaves while its peer may read it
      return;
    }

    // ---- warm start from the FP32 phase: P = (I + omega^2)^-1 in FP64 with the
    // positive-definiteness test, then the iteration continues at a general step
    int warm = 0, step0 = 0;
    if (a.phase == 2 && aux[0] > 0) {
      warm = aux[0];
      double* Ks = smem;
      const int mp16 = round_up(m, 16), kld = frag_ld(mp16);
      bool valid;
      if constexpr (CL == 1) {
        {
          MatOp A[1] = {op_n(Wm, m)};
          MatOp B[1] = {op_n(Wm, m)};
          auto epi = [&](int, int i, int j, double v) { Ks[i * kld + j] = __dadd_rn(i == j ? 1.0 : 0.0, v); };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {   // identity padding up to mp16
          const int i = e / mp16, j = e - i * mp16;
          if (i >= m || j >= m) Ks[i * kld + j] = (i == j) ? 1.0 : 0.0;
        }
        __syncthreads();
        valid = spd_inverse_blocked(Ks, mp16, kld, Ks + mp16 * kld, flag);
        if (valid) {
          SSN_FOR_IJ(team, m, { Pm[e] = Ks[i * kld + j]; })
        }
        __syncthreads();
      } else {
        {
          MatOp A[1] = {op_n(Wm, m)};
          MatOp B[1] = {op_n(Wm, m)};
          auto epi = [&](int, int i, int j, double v) { Kg[i * m + j] = __dadd_rn(i == j ? 1.0 : 0.0, v); };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        team.sync();
        if (rank == 0) {
          for (int i = (int)(threadIdx.x >> 5); i < m; i += kWarps)
            for (int j = (int)(threadIdx.x & 31); j < m; j += 32) Ks[i * kld + j] = Kg[i * m + j];
          for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {
            const int i = e / mp16, j = e - i * mp16;
            if (i >= m || j >= m) Ks[i * kld + j] = (i == j) ? 1.0 : 0.0;
          }
          __syncthreads();
          const bool ok = spd_inverse_blocked(Ks, mp16, kld, Ks + mp16 * kld, flag);
          if (threadIdx.x == 0) {
            vflag[0] = ok ? 1 : 0;
            vflag_peer[0] = ok ? 1 : 0;
          }
          if (ok)
            for (int i = (int)(threadIdx.x >> 5); i < m; i += kWarps)
              for (int j = (int)(threadIdx.x & 31); j < m; j += 32) Pm[i * m + j] = Ks[i * kld + j];
        }
        team.sync();
        valid = *reinterpret_cast<volatile int*>(vflag) != 0;
      }
      if (valid) {
        step0 = 1;
      } else {
        // not positive definite in FP64: start over from omega = 0 (P = I, Q = 0 from the set-up)
        SSN_FOR_IJ(team, m, { Wm[e] = 0.0; })
        team.sync();
      }
      iterations = warm;
    }

    const double sqrt_m = sqrt(static_cast<double>(m));
    const double* SiCur = Ce;  // Si = Ci in the eigenbasis at step 0 (:121-122)
    bool done = false;
    // Newton steps left for this launch: the cap counts the FP32 phase's updates too
    for (int step = step0, left = a.max_newton - warm; left > 0 && !done && status == SSN_INSTANCE_CONVERGED;
         ++step, --left) {
      ++n_step;
      if (step > 0) {
        // Q = -omega P (:124)
        {
          MatOp A[1] = {op_n(Wm, m)};
          MatOp B[1] = {op_n(Pm, m)};
          auto epi = [&](int, int i, int j, double v) { Qm[i * m + j] = -v; };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        team.sync();
        // sandwich (:67-71): Yr = P diag(l) - Q Ce, Yi = P Ce + Q diag(l)
        if (approx) {
          // full rotated Gram: Yr + i Yi = (P + iQ)(CrE + i Ce)
          MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
          MatOp B[2] = {op_n(CrE, m), op_n(Ce, m)};
          auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
          eng.template mul<2, 2, 2, C_SANDF>(A, B, epi);
        } else {
          MatOp A[2] = {op_n(Qm, m), op_n(Pm, m)};
          MatOp B[1] = {op_n(Ce, m)};
          auto epi = [&](int o, int i, int j, double v) {
            const int e = i * m + j;
            if (o == 0) T1[e] = __dsub_rn(__dmul_rn(Pm[e], lam[j]), v);
            else T2[e] = __dadd_rn(v, __dmul_rn(Qm[e], lam[j]));
          };
          eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
        }
        // Sr' = Yr P^T + Yi Q^T, Si' = Yi P^T - Yr Q^T (recover_block on m x m).  Its A
        // operands are this CTA's own rows of Yr, Yi; its B operands P, Q are complete.
        __syncthreads();
        {
          MatOp A[2] = {op_n(T1, m), op_n(T2, m)};
          MatOp B[2] = {op_t(Pm, m), op_t(Qm, m)};
          auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T3 : Dl)[i * m + j] = v; };
          eng.template mul<2, 2, 2, C_CPLX>(A, B, epi);
        }
        team.sync();
        SiCur = Si;
      }
      // Sr = sym, Si = skew, gradient = Je - Si and its norm (:126-128)
      double gn2 = 0.0;
      if (step > 0) {
        each_ij<MB>(team, m,
            [&](int i, int j, int e) {
              const int et = j * m + i;
              return D5{T3[e], T3[et], Dl[e], Dl[et], Je[e]};
            },
            [&](int, int, int e, const D5& v) {
              Sr[e] = (v.x + v.y) / 2;
              const double x = (v.z - v.w) / 2;
              Si[e] = x;
              const double gij = v.u - x;
              G[e] = gij;
              gn2 += gij * gij;
            });
      } else {
        each_ij<MB>(team, m, [&](int, int, int e) { return D2{Je[e], Ce[e]}; },
            [&](int, int, int e, const D2& v) {
              const double gij = v.x - v.y;
              G[e] = gij;
              gn2 += gij * gij;
            });
      }
      const double gnorm = sqrt(team.sum(gn2));
      const double residual = gnorm * s / sqrt_m;
      if (!(residual >= a.feas_tol / 2)) {
        if (!isfinite(residual)) status = SSN_INSTANCE_NONFINITE;
        done = true;
        break;
      }
      ++iterations;

      // ---- search direction.  g is exactly skew, so precondition(-g) = -g / den.
      double slope;
      if (step == 0) {
        // one preconditioner application solves H(E) = E L + L E exactly (:138-140)
        double sl = 0.0;
        each_ij<MB>(team, m, [&](int, int, int e) { return G[e]; },
            [&](int i, int j, int e, double gv) {
              const double z = __ddiv_rn(-gv, lam[i] + lam[j]);
              Dd[e] = z;
              sl += gv * z;
            });
        slope = team.sum(sl);
      } else {
        // PCG (:142-161)
        if (adaptive) {
          // diagonals of P and Sr (all rows of Sr are visible after the residual's cluster sum)
          for (int i = threadIdx.x; i < m; i += kThreads) {
            pdg[i] = Pm[i * m + i];
            sdg[i] = Sr[i * m + i];
          }
          __syncthreads();
          // Both (i, j) and (j, i) evaluate the same expression on the upper-triangle entries
          // (a, b) = (min, max), so the denominators are exactly symmetric and r / den stays
          // exactly antisymmetric: the CG directions, trials and omega keep exact skewness.
          each_ij<MB>(team, m,
              [&](int i, int j, int) {
                const int eu = imin(i, j) * m + imax(i, j);
                return D4{Pm[eu], Sr[eu], Qm[eu], Si[eu]};
              },
              [&](int i, int j, int e, const D4& v) {
                const int a0 = imin(i, j), b0 = imax(i, j);
                double dn = pdg[a0] * sdg[b0] + pdg[b0] * sdg[a0] - 2.0 * v.x * v.y + 2.0 * v.z * v.w;
                if (!(dn > 0.0)) dn = lam[a0] + lam[b0];   // only off-diagonal entries matter; keep them positive
                Dn[e] = i == j ? 1.0 : dn;
              });
        }
        auto den = [&](int i, int j, int e) { return adaptive ? Dn[e] : lam[i] + lam[j]; };
        double rz = 0.0;
        each_ij<MB>(team, m, [&](int i, int j, int e) { return D2{G[e], den(i, j, e)}; },
            [&](int, int, int e, const D2& v) {
              const double r = -v.x;
              const double z = __ddiv_rn(r, v.y);
              Rr[e] = r;
              Dd[e] = 0.0;
              Pp[e] = z;
              rz += r * z;
            });
        rz = team.sum(rz);
        const double tol = fmin(fmax(sqrt(residual), 1e-8), 0.1) * gnorm;
        for (int it = 0; it < a.max_cg; ++it) {
          // H(p) = Z - Z^T with Z = P (p Sr) - Q (p Si) (:74-76); Z rows stay in shared memory
          {
            MatOp A[1] = {op_n(Pp, m)};
            MatOp B[2] = {op_n(Sr, m), op_n(Si, m)};
            auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
            eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
          }
          team.sync();
          {
            MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
            MatOp B[2] = {op_n(T1, m), op_n(T2, m)};
            const int zr0 = team.r0;
            auto epi = [&](int, int i, int j, double v) { Zs[(i - zr0) * zld + j] = v; };
            eng.template mul<2, 2, 1, C_DIFF>(A, B, epi);
          }
          team.sync();
          ++n_hvp;
          double curv = 0.0;
          each_ij<MB>(team, m, [&](int i, int j, int e) { return D3{Pp[e], zval(i, j), zval(j, i)}; },
              [&](int, int, int, const D3& v) { curv += v.x * (v.y - v.z); });
          curv = team.sum(curv);
          if (!(curv > 0.0)) break;  // cg_active &= curvature > 0 (:152)
          const double alpha = rz / curv;
          double rn2 = 0.0, rz_next = 0.0;
          each_ij<MB>(team, m,
              [&](int i, int j, int e) { return D6{zval(i, j), zval(j, i), Dd[e], Pp[e], Rr[e], den(i, j, e)}; },
              [&](int, int, int e, const D6& v) {
                const double hp = v.x - v.y;
                Dd[e] = __dadd_rn(v.z, __dmul_rn(alpha, v.w));
                const double r = __dsub_rn(v.u, __dmul_rn(alpha, hp));
                Rr[e] = r;
                rn2 += r * r;
                rz_next += r * __ddiv_rn(r, v.d);
              });
          team.sum2(rn2, rz_next);
          const double rnorm = sqrt(rn2);
          if (!(rnorm > tol)) break;  // (:155-157)
          const double beta = rz_next / rz;
          each_ij<MB>(team, m, [&](int i, int j, int e) { return D3{Rr[e], den(i, j, e), Pp[e]}; },
              [&](int, int, int e, const D3& v) { Pp[e] = __dadd_rn(__ddiv_rn(v.x, v.y), __dmul_rn(beta, v.z)); });
          __syncthreads();   // the next HVP reads only this CTA's rows of p (its A operand)
          rz = rz_next;
        }
        double sl = 0.0;
        each_ij<MB>(team, m, [&](int, int, int e) { return D2{G[e], Dd[e]}; },
            [&](int, int, int, const D2& v) { sl += v.x * v.y; });
        slope = team.sum(sl);
        // non-descent fallback to the preconditioned gradient (:163-164)
        if (slope >= 0.0) {
          ++n_fallback;
          double s2 = 0.0;
          each_ij<MB>(team, m, [&](int i, int j, int e) { return D2{G[e], den(i, j, e)}; },
              [&](int, int, int e, const D2& v) {
                const double z = __ddiv_rn(-v.x, v.y);
                Dd[e] = z;
                s2 += v.x * z;
              });
          slope = team.sum(s2);
        }
      }

      // ---- Armijo backtracking with the exact objective change (:166-190)
      double t = 1.0;
      bool accepted = false;
      for (int bt = 0; bt < a.max_backtrack; ++bt) {
        ++n_trial;
        double first = 0.0;
        each_ij<MB>(team, m, [&](int, int, int e) { return D3{Dd[e], G[e], Wm[e]}; },
            [&](int, int, int e, const D3& v) {
              const double dl = __dmul_rn(t, v.x);
              Dl[e] = dl;
              first += v.y * dl;
              Wt[e] = __dadd_rn(v.z, dl);      // == skew(omega + delta) for exactly skew omega, delta
            });
        first = team.sum(first);
        // K = I + trial trial, positive-definiteness test + inverse in shared memory
        double* Ks = smem;
        const int mp16 = round_up(m, 16), kld = frag_ld(mp16);
        if constexpr (CL == 1) {
          {
            MatOp A[1] = {op_n(Wt, m)};
            MatOp B[1] = {op_n(Wt, m)};
            auto epi = [&](int, int i, int j, double v) {
              Ks[i * kld + j] = __dadd_rn(i == j ? 1.0 : 0.0, v);
            };
            eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
          }
          for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {   // identity padding up to mp16
            const int i = e / mp16, j = e - i * mp16;
            if (i >= m || j >= m) Ks[i * kld + j] = (i == j) ? 1.0 : 0.0;
          }
          __syncthreads();
          const bool valid = spd_inverse_blocked(Ks, mp16, kld, Ks + mp16 * kld, flag);
          if (valid) {
            SSN_FOR_IJ(team, m, { Pt[e] = Ks[i * kld + j]; })
          }
          __syncthreads();
          if (valid) {
            // V = P_trial delta; dSr = delta Sr, dSi = delta Si (:177-178)
            {
              MatOp A[1] = {op_n(Pt, m)};
              MatOp B[1] = {op_n(Dl, m)};
              auto epi = store_to(T1);
              eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
            }
            __syncthreads();
            {
              MatOp A[1] = {op_n(Dl, m)};
              MatOp B[2] = {op_n(Sr, m), op_n(SiCur, m)};
              auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T2 : T3)[i * m + j] = v; };
              eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
            }
            __syncthreads();
            // tail = <V, dSr + trial dSi> (line_change, hvp_fused.cu:259-371)
            double tail = 0.0;
            {
              MatOp A[1] = {op_n(Wt, m)};
              MatOp B[1] = {op_n(T3, m)};
              auto epi = [&](int, int i, int j, double v) {
                const int e = i * m + j;
                tail += __dmul_rn(T1[e], __dadd_rn(T2[e], v));
              };
              eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
            }
            tail = team.sum(tail);
            const double change = __dadd_rn(first, tail);
            if (change <= 1e-4 * t * slope) {
              double* tmp = Wm;
              Wm = Wt;
              Wt = tmp;
              tmp = Pm;
              Pm = Pt;
              Pt = tmp;
              accepted = true;
              break;
            }
          }
        } else {
          // Cluster: each CTA forms its rows of K in L2.  Then CTA 0 alone inverts K
          // while CTA 1 forms, for all rows, the trial's products that do not need the
          // inverse: U = delta Sr + trial (delta Si) (line_change's dSr + trial dSi).
          // Every cluster barrier below is reached by both CTAs on every trial.
          {
            MatOp A[1] = {op_n(Wt, m)};
            MatOp B[1] = {op_n(Wt, m)};
            auto epi = [&](int, int i, int j, double v) { Kg[i * m + j] = __dadd_rn(i == j ? 1.0 : 0.0, v); };
            eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
          }
          team.sync();
          if (rank == 0) {
            for (int i = (int)(threadIdx.x >> 5); i < m; i += kWarps)
              for (int j = (int)(threadIdx.x & 31); j < m; j += 32) Ks[i * kld + j] = Kg[i * m + j];
            for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {   // identity padding up to mp16
              const int i = e / mp16, j = e - i * mp16;
              if (i >= m || j >= m) Ks[i * kld + j] = (i == j) ? 1.0 : 0.0;
            }
            __syncthreads();
            const bool ok = spd_inverse_blocked(Ks, mp16, kld, Ks + mp16 * kld, flag);
            if (threadIdx.x == 0) {
              vflag[0] = ok ? 1 : 0;
              vflag_peer[0] = ok ? 1 : 0;
            }
            if (ok)
              for (int i = (int)(threadIdx.x >> 5); i < m; i += kWarps)
                for (int j = (int)(threadIdx.x & 31); j < m; j += 32) Pt[i * m + j] = Ks[i * kld + j];
          } else {
            {
              MatOp A[1] = {op_n(Dl, m)};
              MatOp B[2] = {op_n(Sr, m), op_n(SiCur, m)};
              auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T2 : T3)[i * m + j] = v; };
              eng.template mul_all<1, 2, 2, C_SHARED_A>(A, B, epi);
            }
            __syncthreads();
            {
              MatOp A[1] = {op_n(Wt, m)};
              MatOp B[1] = {op_n(T3, m)};
              auto epi = [&](int, int i, int j, double v) {
                const int e = i * m + j;
                T2[e] = __dadd_rn(T2[e], v);
              };
              eng.template mul_all<1, 1, 1, C_ONE>(A, B, epi);
            }
          }
          team.sync();
          const bool valid = *reinterpret_cast<volatile int*>(vflag) != 0;
          if (valid) {
            // tail = <P_trial delta, U> over this CTA's rows (line_change, hvp_fused.cu:259-371)
            double tail = 0.0;
            {
              MatOp A[1] = {op_n(Pt, m)};
              MatOp B[1] = {op_n(Dl, m)};
              auto epi = [&](int, int i, int j, double v) { tail += __dmul_rn(v, T2[i * m + j]); };
              eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
            }
            tail = team.sum(tail);
            const double change = __dadd_rn(first, tail);
            if (change <= 1e-4 * t * slope) {
              double* tmp = Wm;
              Wm = Wt;
              Wt = tmp;
              tmp = Pm;
              Pm = Pt;
              Pt = tmp;
              accepted = true;
              break;
            }
          }
        }
        t = t / 2;
      }
      if (!accepted) status = SSN_INSTANCE_LINE_SEARCH;
    }
    if (status == SSN_INSTANCE_CONVERGED && !done) status = SSN_INSTANCE_NEWTON_CAP;

    // ---- back to the original basis (:58-64): omega = skew(V w V^T), P = V P V^T, Q = V Q V^T
    double* Wout = a.omega + (size_t)inst * mm;
    double* Pout = a.P + (size_t)inst * mm;
    double* Qout = a.Q + (size_t)inst * mm;
    team.sync();
    if (perm) {
      // permutation basis: (V X V^T)[r][q] = X[perm_row[r]][perm_row[q]]
      SSN_FOR_IJ(team, m, {
        const int oi = perm_row[i];
        const int oj = perm_row[j];
        Wout[e] = (Wm[oi * m + oj] - Wm[oj * m + oi]) / 2;
        Pout[e] = Pm[oi * m + oj];
        Qout[e] = Qm[oi * m + oj];
      })
    } else {
    {
      MatOp A[1] = {op_n(V, m)};
      MatOp B[2] = {op_n(Wm, m), op_n(Pm, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T3)[i * m + j] = v; };
      eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
    }
    __syncthreads();
    {
      MatOp A[1] = {op_n(V, m)};
      MatOp B[1] = {op_n(Qm, m)};
      auto epi = store_to(T2);
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    __syncthreads();
    {
      MatOp A[2] = {op_n(T1, m), op_n(T3, m)};
      MatOp B[1] = {op_t(V, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Dl : Pout)[i * m + j] = v; };
      eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
    }
    __syncthreads();
    {
      MatOp A[1] = {op_n(T2, m)};
      MatOp B[1] = {op_t(V, m)};
      auto epi = store_to(Qout);
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    team.sync();
    SSN_FOR_IJ(team, m, { Wout[e] = (Dl[e] - Dl[j * m + i]) / 2; })
    }
  }
  if (threadIdx.x == 0 && rank == 0) {
    a.iterations[inst] = iterations;
    a.status[inst] = status;
    if (a.counters) {
      a.counters[inst * 8 + 0] = n_step;
      a.counters[inst * 8 + 1] = n_hvp;
      a.counters[inst * 8 + 2] = n_trial;
      a.counters[inst * 8 + 3] = n_fallback;
      const bool f32 = a.phase == 2;
      for (int c = 0; c < 4; ++c) a.counters[inst * 8 + 4 + c] = f32 ? aux[1 + c] : 0;
    }
  }
  if constexpr (CL == 2) cg::this_cluster().sync();   // no CTA leaves while its peer may read its shared memory
}

static size_t dual_smem_bytes(int MB, int CL) {
  const int region = dual_region_doubles(MB, CL);
  return sizeof(double) * ((size_t)region + 2 * kWarps + 3 * kMaxM + 8) + 16 + sizeof(int) * 2 * kMaxM;
}

static int sm_count() { return current_device_sm_count(); }

template <int MB, int CL>
static cudaError_t launch_dual_mb(const DualArgs& args, int batch, cudaStream_t stream) {
  const size_t smem = dual_smem_bytes(MB, CL);
  cudaError_t err = cudaFuncSetAttribute(dual_kernel<MB, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(batch * CL);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, dual_kernel<MB, CL>, args);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// Two CTAs per instance when the batch leaves half the SMs idle and m is large
// enough for the row split to pay; one otherwise.
int dual_cluster_size(int batch, int m) {
  const ssn_tuning* tune = active_tuning();
  if (tune && tune->cluster > 0) return (tune->cluster == 2 && m > 32) ? 2 : 1;   // autotuned
  return (m >= 48 && 2 * batch <= sm_count()) ? 2 : 1;
}

static cudaError_t launch_dual_phase(const DualArgs& args, int batch, bool two, cudaStream_t stream) {
  switch (bucket_of(args.m)) {
    case 1: return launch_dual_mb<1, 1>(args, batch, stream);
    case 2: return two ? launch_dual_mb<2, 2>(args, batch, stream) : launch_dual_mb<2, 1>(args, batch, stream);
    case 3: return two ? launch_dual_mb<3, 2>(args, batch, stream) : launch_dual_mb<3, 1>(args, batch, stream);
    default: return two ? launch_dual_mb<4, 2>(args, batch, stream) : launch_dual_mb<4, 1>(args, batch, stream);
  }
}

// FP32 residual below which the split form's FP32 phase hands over to the FP64
// iteration: FP32 resolves these residuals to about 1e-7, and from 1e-5 one FP64
// Newton step (quadratic convergence) usually reaches the stopping tolerance.
constexpr double kFp32SwitchTol = 1e-5;

// Events recorded around the Newton launches of the calling host thread (a measurement
// hook, ssn_set_newton_events): before the set-up, before the FP32 phase, before the FP64
// iteration, after it.
static thread_local cudaEvent_t t_newton_events[4] = {};
static thread_local bool t_newton_events_set = false;

void set_newton_events(void* const* events) {
  t_newton_events_set = events != nullptr;
  for (int i = 0; i < 4; ++i) t_newton_events[i] = events ? static_cast<cudaEvent_t>(events[i]) : nullptr;
}

static cudaError_t mark(int i, cudaStream_t stream) {
  return t_newton_events_set ? cudaEventRecord(t_newton_events[i], stream) : cudaSuccess;
}

cudaError_t launch_dual(const DualArgs& args, int batch, cudaStream_t stream, cudaEvent_t side_fork) {
  int cl = dual_cluster_size(imax(batch, args.concurrent), args.m);
  // The split form's FP32 phase holds m in (64, 96] on a 2-CTA cluster only.  Unless the
  // autotune table fixes the cluster, take it there even where the rule above gives one
  // CTA (more instances than half the SMs, as in large or ragged batches): a few FP32
  // steps and one FP64 step on two SMs cost less SM time than every step in FP64 on one.
  const ssn_tuning* tune = active_tuning();
  if (args.fp32_newton && args.approx_basis && !(tune && tune->cluster > 0) && !dual32_supported(args.m, cl) &&
      dual32_supported(args.m, 2))
    cl = 2;
  const bool two = cl == 2;
  cudaError_t e = mark(0, stream);
  if (e != cudaSuccess) return e;
  if (!(args.fp32_newton && args.approx_basis && dual32_supported(args.m, cl))) {
    DualArgs a = args;
    a.phase = 0;
    if ((e = mark(1, stream)) != cudaSuccess || (e = mark(2, stream)) != cudaSuccess) return e;
    if (side_fork && (e = cudaEventRecord(side_fork, stream)) != cudaSuccess) return e;
    e = launch_dual_phase(a, batch, two, stream);
    return e == cudaSuccess ? mark(3, stream) : e;
  }
  // split form: basis set-up (FP64), early Newton steps (FP32), last steps and exit (FP64)
  DualArgs a = args;
  a.phase = 1;
  e = launch_dual_phase(a, batch, two, stream);
  if (e == cudaSuccess) e = mark(1, stream);
  if (e == cudaSuccess && side_fork) e = cudaEventRecord(side_fork, stream);
  if (e != cudaSuccess) return e;
  Dual32Args b{};
  b.m = args.m;
  b.max_newton = args.max_newton;
  b.max_cg = args.max_cg;
  b.max_backtrack = args.max_backtrack;
  b.switch_tol = kFp32SwitchTol;
  b.work = args.work;
  b.scale = args.scale;
  b.eig_status = args.eig_status;
  b.adaptive = args.adaptive_precond;
  e = launch_dual32(b, batch, cl, stream);
  if (e == cudaSuccess) e = mark(2, stream);
  if (e != cudaSuccess) return e;
  a.phase = 2;
  e = launch_dual_phase(a, batch, two, stream);
  return e == cudaSuccess ? mark(3, stream) : e;
}

// ---------------------------------------------------------------- adjoint (implicit gradient)
// Per instance, in the original basis, with K = (I + i omega)^-1 = P + iQ,
// C = Cr + i Ci = b^H b and M = Mr + i Mi = g^H b (b = A + iD, g = Ga + iGd):
//   S = K C K,  Gamma = -skew(Im(K M K)) + skew(G_omega),
//   H mu = Gamma by preconditioned CG, H(E) = Z - Z^T with Z = P E Sr - Q E Si
//   (the reference's Hessian-vector product, hvp_fused.py:22-53, which is
//   minus the Jacobian of Im(S) - J_m in omega),
//   N = 2i K mu K,
// and writes P, Q and Pn = Nr^T, Qn = -Ni^T, so that two recovery products give
//   dL/dT = [Re; Im] (g K + b N)  (recover(G, P, Q) + recover(T, Pn, Qn)).
// The CG's preconditioner is the diagonal of H in this basis,
//   P_ii Sr_jj + P_jj Sr_ii - 2 P_ij Sr_ij + 2 Q_ij Si_ij.
// One CTA per instance; every branch follows CTA-wide reductions, so all
// threads take the same path.
enum AdjMat { A_SR = 0, A_SI, A_DN, A_MU, A_R, A_PP, A_T1, A_T2, A_Y1, A_Y2 };
static_assert(A_Y2 + 1 <= kAdjointMats, "adjoint workspace matrix count");

template <int MB, int CL>
__global__ void __launch_bounds__(kThreads, 1) adjoint_kernel(AdjointArgs a) {
  extern __shared__ __align__(16) double smem[];
  const int m = a.m, mm = m * m;
  const int rank = CL == 1 ? 0 : (int)cg::this_cluster().block_rank();
  const int inst = blockIdx.x / CL;
  constexpr int region = dual_region_doubles(MB, CL);
  double* red = smem + region;                // 2*kWarps doubles
  double* xch = red + 2 * kWarps;             // 8 doubles: cluster exchange slots
  int* flag = reinterpret_cast<int*>(xch + 8);
  double* pdg = xch + 16;                     // kMaxM doubles: diag(P)
  double* sdg = pdg + kMaxM;                  // kMaxM doubles: diag(Sr)
  double* Zs = smem;                          // this CTA's rows of the HVP outer product
  const int zld = m + 1;
  const int half = round_up(cdiv(m, CL), 8);
  Team<CL> team;
  team.rank = rank;
  team.r0 = imin(m, rank * half);
  team.r1 = imin(m, (rank + 1) * half);
  team.red = red;
  team.xch = xch;
  team.xch_peer = xch;
  team.parity = 0;
  const double* Zpeer = Zs;
  int peer_r0 = 0;
  if constexpr (CL == 2) {
    team.xch_peer = cg::this_cluster().map_shared_rank(xch, rank ^ 1);
    Zpeer = cg::this_cluster().map_shared_rank(Zs, rank ^ 1);
    peer_r0 = imin(m, (rank ^ 1) * half);
  }
  auto zval = [&](int j, int i) -> double {
    if (CL == 1 || (j >= team.r0 && j < team.r1)) return Zs[(j - team.r0) * zld + i];
    return Zpeer[(j - peer_r0) * zld + i];
  };
  Dual<MB, CL> eng{m, smem, team.r0, team.r1 - team.r0};

  double* ws = a.work + (size_t)inst * kAdjointMats * mm;
  double* Sr = ws + (size_t)A_SR * mm;
  double* Si = ws + (size_t)A_SI * mm;
  double* Dn = ws + (size_t)A_DN * mm;
  double* Mu = ws + (size_t)A_MU * mm;
  double* Rr = ws + (size_t)A_R * mm;
  double* Pp = ws + (size_t)A_PP * mm;
  double* T1 = ws + (size_t)A_T1 * mm;
  double* T2 = ws + (size_t)A_T2 * mm;
  double* Y1 = ws + (size_t)A_Y1 * mm;
  double* Y2 = ws + (size_t)A_Y2 * mm;
  const double* W = a.omega + (size_t)inst * mm;
  const double* Cr = a.Cr + (size_t)inst * mm;
  const double* Ci = a.Ci + (size_t)inst * mm;
  const double* Mr = a.Mr + (size_t)inst * mm;
  const double* Mi = a.Mi + (size_t)inst * mm;
  const double* Gw = a.Gw ? a.Gw + (size_t)inst * mm : nullptr;
  double* Pm = a.P + (size_t)inst * mm;
  double* Qm = a.Q + (size_t)inst * mm;
  double* Pn = a.Pn + (size_t)inst * mm;
  double* Qn = a.Qn + (size_t)inst * mm;
  int status = SSN_INSTANCE_CONVERGED;
  int iters = 0;

  // P = (I + omega omega)^-1 with the positive-definiteness test, Q = -omega P.  In a cluster
  // each CTA forms its rows of K in L2 (Y1 as scratch) and both invert the full K, so both
  // take the same decision.
  {
    double* Ks = smem;
    const int mp16 = round_up(m, 16), kld = frag_ld(mp16);
    MatOp A[1] = {op_n(W, m)};
    MatOp B[1] = {op_n(W, m)};
    if constexpr (CL == 1) {
      auto epi = [&](int, int i, int j, double v) { Ks[i * kld + j] = (i == j ? 1.0 : 0.0) + v; };
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    } else {
      auto epi = [&](int, int i, int j, double v) { Y1[i * m + j] = (i == j ? 1.0 : 0.0) + v; };
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
      team.sync();
      for (int i = (int)(threadIdx.x >> 5); i < m; i += kWarps)
        for (int j = (int)(threadIdx.x & 31); j < m; j += 32) Ks[i * kld + j] = Y1[i * m + j];
    }
    for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {
      const int i = e / mp16, j = e - i * mp16;
      if (i >= m || j >= m) Ks[i * kld + j] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    const bool valid = spd_inverse_blocked(Ks, mp16, kld, Ks + mp16 * kld, flag);
    if (valid) {
      SSN_FOR_IJ(team, m, { Pm[e] = Ks[i * kld + j]; })
    } else {
      status = SSN_INSTANCE_NONFINITE;
    }
    team.sync();
  }
  if (status == SSN_INSTANCE_CONVERGED) {
    {
      MatOp A[1] = {op_n(W, m)};
      MatOp B[1] = {op_n(Pm, m)};
      auto epi = [&](int, int i, int j, double v) { Qm[i * m + j] = -v; };
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    team.sync();
    // Y = K C (this CTA's rows), then S = Y K; symmetric / antisymmetric parts need all rows
    {
      MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
      MatOp B[2] = {op_n(Cr, m), op_n(Ci, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Y1 : Y2)[i * m + j] = v; };
      eng.template mul<2, 2, 2, C_SANDF>(A, B, epi);
    }
    __syncthreads();
    {
      MatOp A[2] = {op_n(Y1, m), op_n(Y2, m)};
      MatOp B[2] = {op_n(Pm, m), op_n(Qm, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
      eng.template mul<2, 2, 2, C_SANDF>(A, B, epi);
    }
    team.sync();
    each_ij<MB>(team, m,
        [&](int i, int j, int e) {
          const int et = j * m + i;
          return D4{T1[e], T1[et], T2[e], T2[et]};
        },
        [&](int, int, int e, const D4& v) {
          Sr[e] = (v.x + v.y) / 2;
          Si[e] = (v.z - v.w) / 2;
        });
    team.sync();
    // Y = K M, then Im(Y K) = Y1 Q + Y2 P (this CTA's rows)
    {
      MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
      MatOp B[2] = {op_n(Mr, m), op_n(Mi, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Y1 : Y2)[i * m + j] = v; };
      eng.template mul<2, 2, 2, C_SANDF>(A, B, epi);
    }
    __syncthreads();
    {
      MatOp A[2] = {op_n(Y1, m), op_n(Y2, m)};
      MatOp B[2] = {op_n(Qm, m), op_n(Pm, m)};
      auto epi = [&](int, int i, int j, double v) { T2[i * m + j] = v; };
      eng.template mul<2, 2, 1, C_SHARED_SUM>(A, B, epi);
    }
    team.sync();
    // Gamma = -skew(Im(K M K)) + skew(G_omega) (exactly antisymmetric), preconditioner,
    // CG start: mu = 0, r = Gamma, p = r / den
    for (int i = threadIdx.x; i < m; i += kThreads) {
      pdg[i] = Pm[i * m + i];
      sdg[i] = Sr[i * m + i];
    }
    __syncthreads();
    double gn2 = 0.0, rz = 0.0;
    each_ij<MB>(team, m,
        [&](int i, int j, int e) {
          const int et = j * m + i;
          // the denominator from the upper-triangle entries: exactly symmetric, so mu stays skew
          const int eu = imin(i, j) * m + imax(i, j);
          return D6{T2[e], T2[et], Gw ? Gw[e] : 0.0, Gw ? Gw[et] : 0.0, Pm[eu] * Sr[eu], Qm[eu] * Si[eu]};
        },
        [&](int i, int j, int e, const D6& v) {
          const double g = ((v.y - v.x) + (v.z - v.w)) / 2;
          const int a0 = imin(i, j), b0 = imax(i, j);
          double dn = pdg[a0] * sdg[b0] + pdg[b0] * sdg[a0] - 2.0 * v.u + 2.0 * v.d;
          if (!(dn > 0.0)) dn = 1.0;
          if (i == j) dn = 1.0;
          Dn[e] = dn;
          Rr[e] = g;
          Mu[e] = 0.0;
          const double z = g / dn;
          Pp[e] = z;
          gn2 += g * g;
          rz += g * z;
        });
    team.sum2(gn2, rz);
    const double gnorm = sqrt(gn2);
    if (!isfinite(gnorm) || !isfinite(rz)) status = SSN_INSTANCE_NONFINITE;
    double rnorm = gnorm;
    const double stop = a.tol * gnorm;
    while (status == SSN_INSTANCE_CONVERGED && rnorm > stop) {
      if (iters >= a.max_cg) {
        status = SSN_INSTANCE_NEWTON_CAP;
        break;
      }
      ++iters;
      {
        MatOp A[1] = {op_n(Pp, m)};
        MatOp B[2] = {op_n(Sr, m), op_n(Si, m)};
        auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
        eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
      }
      team.sync();
      {
        MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
        MatOp B[2] = {op_n(T1, m), op_n(T2, m)};
        const int zr0 = team.r0;
        auto epi = [&](int, int i, int j, double v) { Zs[(i - zr0) * zld + j] = v; };
        eng.template mul<2, 2, 1, C_DIFF>(A, B, epi);
      }
      team.sync();
      double curv = 0.0;
      each_ij<MB>(team, m, [&](int i, int j, int e) { return D3{Pp[e], zval(i, j), zval(j, i)}; },
          [&](int, int, int, const D3& v) { curv += v.x * (v.y - v.z); });
      curv = team.sum(curv);
      if (!(curv > 0.0)) {            // H is positive definite at a strict dual optimum
        status = isfinite(curv) ? SSN_INSTANCE_NEWTON_CAP : SSN_INSTANCE_NONFINITE;
        break;
      }
      const double alpha = rz / curv;
      double rn2 = 0.0, rz_next = 0.0;
      each_ij<MB>(team, m,
          [&](int i, int j, int e) { return D6{zval(i, j), zval(j, i), Mu[e], Pp[e], Rr[e], Dn[e]}; },
          [&](int, int, int e, const D6& v) {
            Mu[e] = v.z + alpha * v.w;
            const double r = v.u - alpha * (v.x - v.y);
            Rr[e] = r;
            rn2 += r * r;
            rz_next += r * (r / v.d);
          });
      team.sum2(rn2, rz_next);
      rnorm = sqrt(rn2);
      const double beta = rz_next / rz;
      rz = rz_next;
      each_ij<MB>(team, m, [&](int, int, int e) { return D3{Rr[e], Dn[e], Pp[e]}; },
          [&](int, int, int e, const D3& v) { Pp[e] = v.x / v.y + beta * v.z; });
      __syncthreads();       // the next HVP reads only this CTA's rows of p; mu was published by sum2
    }
    // N = 2i K mu K: U = [P mu, Q mu]; K mu K = (U1 P - U2 Q) + i (U1 Q + U2 P)
    // (only for a converged solve: a failed one writes NaN below, row by row)
    if (status == SSN_INSTANCE_CONVERGED) {
      {
        MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
        MatOp B[1] = {op_n(Mu, m)};
        auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Y1 : Y2)[i * m + j] = v; };
        eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
      }
      __syncthreads();
      {
        MatOp A[2] = {op_n(Y1, m), op_n(Y2, m)};
        MatOp B[2] = {op_n(Pm, m), op_n(Qm, m)};
        // Nr = -2 Im(K mu K), Ni = 2 Re(K mu K); Pn = Nr^T, Qn = -Ni^T
        auto epi = [&](int o, int i, int j, double v) {
          if (o == 0) Qn[j * m + i] = -2.0 * v;
          else Pn[j * m + i] = -2.0 * v;
        };
        eng.template mul<2, 2, 2, C_SANDF>(A, B, epi);
      }
    }
  }
  if (status != SSN_INSTANCE_CONVERGED) {
    __syncthreads();
    SSN_FOR_IJ(team, m, {
      Pn[e] = NAN;
      Qn[e] = NAN;
    })
  }
  if (threadIdx.x == 0 && rank == 0) {
    a.status[inst] = status;
    if (a.cg_iters) a.cg_iters[inst] = iters;
  }
  if constexpr (CL == 2) cg::this_cluster().sync();   // no CTA leaves while its peer may read its shared memory
}

size_t adjoint_smem_bytes(int MB, int CL) {
  return sizeof(double) * ((size_t)dual_region_doubles(MB, CL) + 2 * kWarps + 16 + 2 * kMaxM) + 16;
}

template <int MB, int CL>
static cudaError_t launch_adjoint_mb(const AdjointArgs& args, int batch, cudaStream_t stream) {
  const size_t smem = adjoint_smem_bytes(MB, CL);
  cudaError_t err = cudaFuncSetAttribute(adjoint_kernel<MB, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(batch * CL);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  err = cudaLaunchKernelEx(&cfg, adjoint_kernel<MB, CL>, args);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// One CTA per instance, or a 2-CTA cluster when the batch leaves SMs idle (the rule of
// the Newton kernel).
cudaError_t launch_adjoint(const AdjointArgs& args, int batch, cudaStream_t stream) {
  const bool two = dual_cluster_size(batch, args.m) == 2;
  switch (bucket_of(args.m)) {
    case 1: return launch_adjoint_mb<1, 1>(args, batch, stream);
    case 2: return two ? launch_adjoint_mb<2, 2>(args, batch, stream) : launch_adjoint_mb<2, 1>(args, batch, stream);
    case 3: return two ? launch_adjoint_mb<3, 2>(args, batch, stream) : launch_adjoint_mb<3, 1>(args, batch, stream);
    default: return two ? launch_adjoint_mb<4, 2>(args, batch, stream) : launch_adjoint_mb<4, 1>(args, batch, stream);
  }
}

// ---------------------------------------------------------------- SPD inverse component
__global__ void __launch_bounds__(kThreads, 1)
    spd_inverse_kernel(const double* K, double* P, int32_t* info, int m) {
  extern __shared__ __align__(16) double smem[];
  const int inst = blockIdx.x, mm = m * m;
  const int mp16 = round_up(m, 16), ld = frag_ld(mp16);
  int* flag = reinterpret_cast<int*>(smem + spd_region_doubles(m));
  const double* Kin = K + (size_t)inst * mm;
  for (int e = threadIdx.x; e < mp16 * mp16; e += kThreads) {
    const int i = e / mp16, j = e - i * mp16;
    smem[i * ld + j] = (i < m && j < m) ? Kin[i * m + j] : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  const bool ok = spd_inverse_blocked(smem, mp16, ld, smem + mp16 * ld, flag);
  double* Pout = P + (size_t)inst * mm;
  for (int e = threadIdx.x; e < mm; e += kThreads) {
    const int i = e / m, j = e - i * m;
    Pout[e] = ok ? smem[i * ld + j] : NAN;
  }
  if (threadIdx.x == 0) info[inst] = ok ? 0 : 1;
}

cudaError_t launch_spd_inverse(const double* K, double* P, int32_t* info, int batch, int m,
                               cudaStream_t stream) {
  const size_t smem = sizeof(double) * (size_t)spd_region_doubles(m) + 16;
  cudaError_t err = cudaFuncSetAttribute(spd_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  spd_inverse_kernel<<<batch, kThreads, smem, stream>>>(K, P, info, m);
  return cudaGetLastError();
}

}  // namespace ssn
