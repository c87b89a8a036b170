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

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

enum Mat {
  M_CE = 0, M_JE, M_W, M_WT, M_P, M_PT, M_Q, M_SR, M_SI, M_G, M_D, M_R, M_PP, M_HP, M_DL,
  M_T1, M_T2, M_T3, M_X0, M_X1, M_X2
};
static_assert(M_X2 + 1 == kDualMats, "workspace matrix count");

constexpr uint32_t C_ONE = coef_bit(0, 0, 0, 1);
constexpr uint32_t C_SHARED_B = coef_bit(0, 0, 0, 1) | coef_bit(1, 1, 0, 1);
constexpr uint32_t C_SHARED_A = coef_bit(0, 0, 0, 1) | coef_bit(1, 0, 1, 1);
constexpr uint32_t C_DIFF = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 2);
constexpr uint32_t C_CPLX = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1) | coef_bit(1, 1, 0, 1) |
                            coef_bit(1, 0, 1, 2);

// In-place Gauss-Jordan inversion of an SPD matrix held in shared memory
// (ld = m + 1).  Pivot k uses the current Schur complement diagonal, which is
// positive for every k exactly when the matrix is positive definite -- the
// same test torch.linalg.cholesky_ex applies.  Returns false (uniformly) on a
// non-positive or non-finite pivot.  vec: 4*m doubles of scratch.  One CTA
// barrier per pivot: the next pivot row/column are written to a second buffer.
__device__ bool spd_inverse_smem(double* K, int m, double* vec) {
  const int ld = m + 1;
  double* rowv[2] = {vec, vec + m};
  double* colv[2] = {vec + 2 * m, vec + 3 * m};
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    rowv[0][j] = K[j];
    colv[0][j] = K[j * ld];
  }
  __syncthreads();
  const int mm = m * m;
  for (int k = 0; k < m; ++k) {
    const int cur = k & 1, nxt = cur ^ 1;
    const double piv = rowv[cur][k];
    if (!(piv > 0.0) || !isfinite(piv)) return false;
    const double inv = 1.0 / piv;
    const double* rk = rowv[cur];
    const double* ck = colv[cur];
    for (int e = threadIdx.x; e < mm; e += blockDim.x) {
      const int i = e / m, j = e - i * m;
      double v;
      if (i == k) {
        v = (j == k) ? inv : rk[j] * inv;
      } else if (j == k) {
        v = -ck[i] * inv;
      } else {
        v = K[i * ld + j] - ck[i] * (rk[j] * inv);
      }
      K[i * ld + j] = v;
      if (i == k + 1) rowv[nxt][j] = v;
      if (j == k + 1) colv[nxt][i] = v;
    }
    __syncthreads();
  }
  return true;
}

template <int MB>
struct Dual {
  int m, mm;
  double* smem;
  int slot;

  template <int NA, int NB, int NOUT, uint32_t COEF, class Epi>
  __device__ __forceinline__ void mul(const MatOp (&A)[NA], const MatOp (&B)[NB], Epi& epi) const {
    using TL = Tile<MB, NOUT>;
    ssn::tile_product<TL::WR, TL::WC, NA, NB, NOUT, COEF>(A, B, m, m, m, smem, slot, epi);
  }
};

template <int MB>
__global__ void __launch_bounds__(kThreads, 1) dual_kernel(DualArgs a) {
  extern __shared__ __align__(16) double smem[];
  const int inst = blockIdx.x;
  const int m = a.m, mm = m * m, tid = threadIdx.x;
  const int slot = slot_doubles(MB);
  double* red = smem + 8 * slot;              // 2*kWarps doubles
  double* lam = red + 2 * kWarps;             // m doubles
  Dual<MB> eng{m, mm, smem, slot};

  double* ws = a.work + (size_t)inst * kDualMats * mm;
  double* buf[kDualMats];
#pragma unroll
  for (int k = 0; k < kDualMats; ++k) buf[k] = ws + (size_t)k * mm;
  const double* Ci = a.Ci + (size_t)inst * mm;
  const double* V = a.vectors + (size_t)inst * mm;
  const double s = a.scale[inst];
  int status = a.eig_status ? a.eig_status[inst] : SSN_INSTANCE_CONVERGED;
  for (int i = tid; i < m; i += kThreads) lam[i] = a.values[(size_t)inst * m + i];
  __syncthreads();

  double *Ce = buf[M_CE], *Je = buf[M_JE], *Wm = buf[M_W], *Wt = buf[M_WT];
  double *Pm = buf[M_P], *Pt = buf[M_PT], *Qm = buf[M_Q], *Sr = buf[M_SR], *Si = buf[M_SI];
  double *G = buf[M_G], *Dd = buf[M_D], *Rr = buf[M_R], *Pp = buf[M_PP], *Hp = buf[M_HP];
  double *Dl = buf[M_DL], *T1 = buf[M_T1], *T2 = buf[M_T2], *T3 = buf[M_T3];

  auto store_to = [&](double* dst) {
    return [dst, m](int, int i, int j, double v) { dst[i * m + j] = v; };
  };
  auto precond = [&](const double* R, int i, int j) -> double {
    const double x = __ddiv_rn(R[i * m + j], lam[i] + lam[j]);
    const double y = __ddiv_rn(R[j * m + i], lam[j] + lam[i]);
    return __dmul_rn(__dsub_rn(x, y), 0.5);
  };

  int64_t iterations = 0;
  int n_hvp = 0, n_trial = 0, n_fallback = 0, n_step = 0;
  if (status == SSN_INSTANCE_CONVERGED) {
    // ---- eigenbasis set-up: Ce = skew(V^T (Ci/s) V), Je = skew(V^T J(V)) / s  (:106-111, :53-56)
    for (int e = tid; e < mm; e += kThreads) T1[e] = Ci[e] / s;
    for (int e = tid; e < mm; e += kThreads) {
      const int i = e / m, j = e - i * m, h = m / 2;
      T3[e] = i < h ? V[(i + h) * m + j] : -V[(i - h) * m + j];
    }
    __syncthreads();
    {
      MatOp A[1] = {op_t(V, m)};
      MatOp B[2] = {op_n(T1, m), op_n(T3, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T2 : Dl)[i * m + j] = v; };
      eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
    }
    {
      MatOp A[1] = {op_n(T2, m)};
      MatOp B[1] = {op_n(V, m)};
      auto epi = store_to(T1);
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    for (int e = tid; e < mm; e += kThreads) {
      const int i = e / m, j = e - i * m;
      Ce[e] = (T1[e] - T1[j * m + i]) / 2;
      Je[e] = ((Dl[e] - Dl[j * m + i]) / 2) / s;
      Wm[e] = 0.0;
      Pm[e] = (i == j) ? 1.0 : 0.0;
      Qm[e] = 0.0;
      Sr[e] = (i == j) ? lam[i] : 0.0;
    }
    __syncthreads();

    const double sqrt_m = sqrt(static_cast<double>(m));
    const double* SiCur = Ce;  // Si = Ci in the eigenbasis at step 0 (:121-122)
    bool done = false;
    for (int step = 0; step < a.max_newton && !done && status == SSN_INSTANCE_CONVERGED; ++step) {
      ++n_step;
      if (step > 0) {
        // Q = -omega P (:124)
        {
          MatOp A[1] = {op_n(Wm, m)};
          MatOp B[1] = {op_n(Pm, m)};
          auto epi = [&](int, int i, int j, double v) { Qm[i * m + j] = -v; };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        // sandwich (:67-71): Yr = P diag(l) - Q Ce, Yi = P Ce + Q diag(l)
        {
          MatOp A[2] = {op_n(Qm, m), op_n(Pm, m)};
          MatOp B[1] = {op_n(Ce, m)};
          auto epi = [&](int o, int i, int j, double v) {
            const int e = i * m + j;
            if (o == 0) T1[e] = __dsub_rn(__dmul_rn(Pm[e], lam[j]), v);
            else T2[e] = __dadd_rn(v, __dmul_rn(Qm[e], lam[j]));
          };
          eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
        }
        // Sr' = Yr P^T + Yi Q^T, Si' = Yi P^T - Yr Q^T (recover_block on m x m)
        {
          MatOp A[2] = {op_n(T1, m), op_n(T2, m)};
          MatOp B[2] = {op_t(Pm, m), op_t(Qm, m)};
          auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Sr : Si)[i * m + j] = v; };
          eng.template mul<2, 2, 2, C_CPLX>(A, B, epi);
        }
        SiCur = Si;
      }
      // Sr = sym, Si = skew, gradient = Je - Si and its norm (:126-128)
      double gn2 = 0.0;
      for (int e = tid; e < mm; e += kThreads) {
        const int i = e / m, j = e - i * m;
        if (i > j) continue;
        const int et = j * m + i;
        double sij, sji;
        if (step > 0) {
          const double r = (Sr[e] + Sr[et]) / 2;
          Sr[e] = r;
          Sr[et] = r;
          const double x = (Si[e] - Si[et]) / 2;
          const double y = (Si[et] - Si[e]) / 2;
          Si[e] = x;
          Si[et] = y;
          sij = x;
          sji = y;
        } else {
          sij = Ce[e];
          sji = Ce[et];
        }
        const double gij = Je[e] - sij;
        G[e] = gij;
        gn2 += gij * gij;
        if (i != j) {
          const double gji = Je[et] - sji;
          G[et] = gji;
          gn2 += gji * gji;
        }
      }
      const double gnorm = sqrt(block_sum(gn2, red));
      const double residual = gnorm * s / sqrt_m;
      if (!(residual >= a.feas_tol / 2)) {
        if (!isfinite(residual)) status = SSN_INSTANCE_NONFINITE;
        done = true;
        break;
      }
      ++iterations;

      // ---- search direction
      double slope;
      if (step == 0) {
        // one preconditioner application solves H(E) = E L + L E exactly (:138-140)
        double sl = 0.0;
        for (int e = tid; e < mm; e += kThreads) {
          const int i = e / m, j = e - i * m;
          const double x = __ddiv_rn(-G[e], lam[i] + lam[j]);
          const double y = __ddiv_rn(-G[j * m + i], lam[j] + lam[i]);
          const double z = __dmul_rn(__dsub_rn(x, y), 0.5);
          Dd[e] = z;
          sl += G[e] * z;
        }
        slope = block_sum(sl, red);
      } else {
        // PCG (:142-161)
        for (int e = tid; e < mm; e += kThreads) {
          Rr[e] = -G[e];
          Dd[e] = 0.0;
        }
        __syncthreads();
        double rz = 0.0;
        for (int e = tid; e < mm; e += kThreads) {
          const int i = e / m, j = e - i * m;
          const double z = precond(Rr, i, j);
          Pp[e] = z;
          rz += Rr[e] * z;
        }
        rz = block_sum(rz, red);
        const double tol = fmin(fmax(sqrt(residual), 1e-8), 0.1) * gnorm;
        for (int it = 0; it < a.max_cg; ++it) {
          // Hp = H(p): U = p Sr, V = p Si; Z = P U - Q V; Hp = Z - Z^T (:74-76)
          {
            MatOp A[1] = {op_n(Pp, m)};
            MatOp B[2] = {op_n(Sr, m), op_n(Si, m)};
            auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
            eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
          }
          {
            MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
            MatOp B[2] = {op_n(T1, m), op_n(T2, m)};
            auto epi = store_to(T3);
            eng.template mul<2, 2, 1, C_DIFF>(A, B, epi);
          }
          ++n_hvp;
          double curv = 0.0;
          for (int e = tid; e < mm; e += kThreads) {
            const int i = e / m, j = e - i * m;
            const double h = T3[e] - T3[j * m + i];
            Hp[e] = h;
            curv += Pp[e] * h;
          }
          curv = block_sum(curv, red);
          if (!(curv > 0.0)) break;  // cg_active &= curvature > 0 (:152)
          const double alpha = rz / curv;
          double rn2 = 0.0;
          for (int e = tid; e < mm; e += kThreads) {
            Dd[e] = __dadd_rn(Dd[e], __dmul_rn(alpha, Pp[e]));
            const double r = __dsub_rn(Rr[e], __dmul_rn(alpha, Hp[e]));
            Rr[e] = r;
            rn2 += r * r;
          }
          const double rnorm = sqrt(block_sum(rn2, red));
          if (!(rnorm > tol)) break;  // (:155-157)
          double rz_next = 0.0;
          for (int e = tid; e < mm; e += kThreads) {
            const int i = e / m, j = e - i * m;
            rz_next += Rr[e] * precond(Rr, i, j);
          }
          rz_next = block_sum(rz_next, red);
          const double beta = rz_next / rz;
          for (int e = tid; e < mm; e += kThreads) {
            const int i = e / m, j = e - i * m;
            Pp[e] = __dadd_rn(precond(Rr, i, j), __dmul_rn(beta, Pp[e]));
          }
          __syncthreads();
          rz = rz_next;
        }
        double sl = 0.0;
        for (int e = tid; e < mm; e += kThreads) sl += G[e] * Dd[e];
        slope = block_sum(sl, red);
        // non-descent fallback to the preconditioned gradient (:163-164)
        if (slope >= 0.0) {
          ++n_fallback;
          double s2 = 0.0;
          for (int e = tid; e < mm; e += kThreads) {
            const int i = e / m, j = e - i * m;
            const double x = __ddiv_rn(-G[e], lam[i] + lam[j]);
            const double y = __ddiv_rn(-G[j * m + i], lam[j] + lam[i]);
            const double z = __dmul_rn(__dsub_rn(x, y), 0.5);
            Dd[e] = z;
            s2 += G[e] * z;
          }
          slope = block_sum(s2, red);
        }
      }

      // ---- Armijo backtracking with the exact objective change (:166-190)
      double t = 1.0;
      bool accepted = false;
      for (int bt = 0; bt < a.max_backtrack; ++bt) {
        ++n_trial;
        double first = 0.0;
        for (int e = tid; e < mm; e += kThreads) {
          const int i = e / m, j = e - i * m, et = j * m + i;
          const double dl = __dmul_rn(t, Dd[e]);
          Dl[e] = dl;
          first += G[e] * dl;
          const double x = __dadd_rn(Wm[e], dl);
          const double y = __dadd_rn(Wm[et], __dmul_rn(t, Dd[et]));
          Wt[e] = (x - y) / 2;
        }
        first = block_sum(first, red);
        // K = I + trial trial, factor test + inverse in shared memory
        double* Ks = smem;
        const int kld = m + 1;
        {
          MatOp A[1] = {op_n(Wt, m)};
          MatOp B[1] = {op_n(Wt, m)};
          auto epi = [&](int, int i, int j, double v) {
            Ks[i * kld + j] = __dadd_rn(i == j ? 1.0 : 0.0, v);
          };
          eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
        }
        const bool valid = spd_inverse_smem(Ks, m, smem + m * kld);
        if (valid) {
          for (int e = tid; e < mm; e += kThreads) {
            const int i = e / m, j = e - i * m;
            Pt[e] = Ks[i * kld + j];
          }
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
          {
            MatOp A[1] = {op_n(Dl, m)};
            MatOp B[2] = {op_n(Sr, m), op_n(SiCur, m)};
            auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T2 : T3)[i * m + j] = v; };
            eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
          }
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
          tail = block_sum(tail, red);
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
        t = t / 2;
      }
      if (!accepted) status = SSN_INSTANCE_LINE_SEARCH;
    }
    if (status == SSN_INSTANCE_CONVERGED && !done) status = SSN_INSTANCE_NEWTON_CAP;

    // ---- back to the original basis (:58-64): omega = skew(V w V^T), P = V P V^T, Q = V Q V^T
    double* Wout = a.omega + (size_t)inst * mm;
    double* Pout = a.P + (size_t)inst * mm;
    double* Qout = a.Q + (size_t)inst * mm;
    {
      MatOp A[1] = {op_n(V, m)};
      MatOp B[1] = {op_n(Wm, m)};
      auto epi = store_to(T1);
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    {
      MatOp A[1] = {op_n(T1, m)};
      MatOp B[1] = {op_t(V, m)};
      auto epi = store_to(T2);
      eng.template mul<1, 1, 1, C_ONE>(A, B, epi);
    }
    for (int e = tid; e < mm; e += kThreads) {
      const int i = e / m, j = e - i * m;
      Wout[e] = (T2[e] - T2[j * m + i]) / 2;
    }
    {
      MatOp A[1] = {op_n(V, m)};
      MatOp B[2] = {op_n(Pm, m), op_n(Qm, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T3)[i * m + j] = v; };
      eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
    }
    {
      MatOp A[2] = {op_n(T1, m), op_n(T3, m)};
      MatOp B[1] = {op_t(V, m)};
      auto epi = [&](int o, int i, int j, double v) { (o == 0 ? Pout : Qout)[i * m + j] = v; };
      eng.template mul<2, 1, 2, C_SHARED_B>(A, B, epi);
    }
  }
  if (tid == 0) {
    a.iterations[inst] = iterations;
    a.status[inst] = status;
    if (a.counters) {
      a.counters[inst * 4 + 0] = n_step;
      a.counters[inst * 4 + 1] = n_hvp;
      a.counters[inst * 4 + 2] = n_trial;
      a.counters[inst * 4 + 3] = n_fallback;
    }
  }
}

static size_t dual_smem_bytes(int MB) {
  return sizeof(double) * (8 * (size_t)slot_doubles(MB) + 2 * kWarps + kMaxM);
}

template <int MB>
static cudaError_t launch_dual_mb(const DualArgs& args, int batch, cudaStream_t stream) {
  const size_t smem = dual_smem_bytes(MB);
  cudaError_t err = cudaFuncSetAttribute(dual_kernel<MB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  dual_kernel<MB><<<batch, kThreads, smem, stream>>>(args);
  return cudaGetLastError();
}

cudaError_t launch_dual(const DualArgs& args, int batch, cudaStream_t stream) {
  switch (bucket_of(args.m)) {
    case 1: return launch_dual_mb<1>(args, batch, stream);
    case 2: return launch_dual_mb<2>(args, batch, stream);
    case 3: return launch_dual_mb<3>(args, batch, stream);
    default: return launch_dual_mb<4>(args, batch, stream);
  }
}

// ---------------------------------------------------------------- SPD inverse component
__global__ void __launch_bounds__(kThreads, 1)
    spd_inverse_kernel(const double* K, double* P, int32_t* info, int m) {
  extern __shared__ __align__(16) double smem[];
  const int inst = blockIdx.x, mm = m * m, ld = m + 1;
  const double* Kin = K + (size_t)inst * mm;
  for (int e = threadIdx.x; e < mm; e += kThreads) {
    const int i = e / m, j = e - i * m;
    smem[i * ld + j] = Kin[e];
  }
  __syncthreads();
  const bool ok = spd_inverse_smem(smem, m, smem + m * ld);
  double* Pout = P + (size_t)inst * mm;
  for (int e = threadIdx.x; e < mm; e += kThreads) {
    const int i = e / m, j = e - i * m;
    Pout[e] = ok ? smem[i * ld + j] : NAN;
  }
  if (threadIdx.x == 0) info[inst] = ok ? 0 : 1;
}

cudaError_t launch_spd_inverse(const double* K, double* P, int32_t* info, int batch, int m,
                               cudaStream_t stream) {
  const size_t smem = sizeof(double) * ((size_t)m * (m + 1) + 4 * m);
  cudaError_t err = cudaFuncSetAttribute(spd_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  spd_inverse_kernel<<<batch, kThreads, smem, stream>>>(K, P, info, m);
  return cudaGetLastError();
}

}  // namespace ssn
