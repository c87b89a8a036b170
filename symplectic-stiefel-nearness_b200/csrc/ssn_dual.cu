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

// Element loops without integer division: warp w owns rows w, w+16, ..., lane l
// owns columns l, l+32, ...; consecutive lanes touch consecutive addresses.
#define SSN_FOR_IJ(m_, BODY)                                                          \
  for (int i = (int)(threadIdx.x >> 5); i < (m_); i += kWarps)                        \
    for (int j = (int)(threadIdx.x & 31); j < (m_); j += 32) {                        \
      const int e = i * (m_) + j;                                                     \
      (void)e;                                                                        \
      BODY                                                                            \
    }

template <int MB>
__global__ void __launch_bounds__(kThreads, 1) dual_kernel(DualArgs a) {
  extern __shared__ __align__(16) double smem[];
  const int inst = blockIdx.x;
  const int m = a.m, mm = m * m;
  const int slot = slot_doubles(MB);
  const int region = imax(8 * slot, spd_region_doubles(m));
  double* red = smem + region;                // 2*kWarps doubles
  double* lam = red + 2 * kWarps;             // m doubles
  int* flag = reinterpret_cast<int*>(lam + kMaxM);
  double* Zs = smem;                          // m x (m+1): HVP outer product, after the engine
  const int zld = m + 1;
  Dual<MB> eng{m, mm, smem, slot};

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

  auto store_to = [&](double* dst) {
    return [dst, m](int, int i, int j, double v) { dst[i * m + j] = v; };
  };

  int64_t iterations = 0;
  int n_hvp = 0, n_trial = 0, n_fallback = 0, n_step = 0;
  if (status == SSN_INSTANCE_CONVERGED) {
    // ---- eigenbasis set-up: Ce = skew(V^T (Ci/s) V), Je = skew(V^T J(V)) / s  (:106-111, :53-56)
    const int h = m / 2;
    SSN_FOR_IJ(m, {
      T1[e] = Ci[e] / s;
      T3[e] = i < h ? V[(i + h) * m + j] : -V[(i - h) * m + j];
    })
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
    // Skew parts are exactly antisymmetric ((x - y)/2 vs (y - x)/2), which every
    // later pass relies on: precondition(r) = r / den and skew(w + t d) = w + t d
    // hold bit for bit for exactly skew r, w, d.
    SSN_FOR_IJ(m, {
      const int et = j * m + i;
      Ce[e] = (T1[e] - T1[et]) / 2;
      Je[e] = ((Dl[e] - Dl[et]) / 2) / s;
      Wm[e] = 0.0;
      Pm[e] = (i == j) ? 1.0 : 0.0;
      Qm[e] = 0.0;
      Sr[e] = (i == j) ? lam[i] : 0.0;
    })
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
          auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T3 : Dl)[i * m + j] = v; };
          eng.template mul<2, 2, 2, C_CPLX>(A, B, epi);
        }
        SiCur = Si;
      }
      // Sr = sym, Si = skew, gradient = Je - Si and its norm (:126-128)
      double gn2 = 0.0;
      if (step > 0) {
        SSN_FOR_IJ(m, {
          const int et = j * m + i;
          Sr[e] = (T3[e] + T3[et]) / 2;
          const double x = (Dl[e] - Dl[et]) / 2;
          Si[e] = x;
          const double gij = Je[e] - x;
          G[e] = gij;
          gn2 += gij * gij;
        })
      } else {
        SSN_FOR_IJ(m, {
          const double gij = Je[e] - Ce[e];
          G[e] = gij;
          gn2 += gij * gij;
        })
      }
      const double gnorm = sqrt(block_sum(gn2, red));
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
        SSN_FOR_IJ(m, {
          const double z = __ddiv_rn(-G[e], lam[i] + lam[j]);
          Dd[e] = z;
          sl += G[e] * z;
        })
        slope = block_sum(sl, red);
      } else {
        // PCG (:142-161)
        double rz = 0.0;
        SSN_FOR_IJ(m, {
          const double r = -G[e];
          const double z = __ddiv_rn(r, lam[i] + lam[j]);
          Rr[e] = r;
          Dd[e] = 0.0;
          Pp[e] = z;
          rz += r * z;
        })
        rz = block_sum(rz, red);
        const double tol = fmin(fmax(sqrt(residual), 1e-8), 0.1) * gnorm;
        for (int it = 0; it < a.max_cg; ++it) {
          // H(p) = Z - Z^T with Z = P (p Sr) - Q (p Si) (:74-76); Z stays in shared memory
          {
            MatOp A[1] = {op_n(Pp, m)};
            MatOp B[2] = {op_n(Sr, m), op_n(Si, m)};
            auto epi = [&](int o, int i, int j, double v) { (o == 0 ? T1 : T2)[i * m + j] = v; };
            eng.template mul<1, 2, 2, C_SHARED_A>(A, B, epi);
          }
          {
            MatOp A[2] = {op_n(Pm, m), op_n(Qm, m)};
            MatOp B[2] = {op_n(T1, m), op_n(T2, m)};
            auto epi = [&](int, int i, int j, double v) { Zs[i * zld + j] = v; };
            eng.template mul<2, 2, 1, C_DIFF>(A, B, epi);
          }
          ++n_hvp;
          double curv = 0.0;
          SSN_FOR_IJ(m, { curv += Pp[e] * (Zs[i * zld + j] - Zs[j * zld + i]); })
          curv = block_sum(curv, red);
          if (!(curv > 0.0)) break;  // cg_active &= curvature > 0 (:152)
          const double alpha = rz / curv;
          double rn2 = 0.0, rz_next = 0.0;
          SSN_FOR_IJ(m, {
            const double hp = Zs[i * zld + j] - Zs[j * zld + i];
            Dd[e] = __dadd_rn(Dd[e], __dmul_rn(alpha, Pp[e]));
            const double r = __dsub_rn(Rr[e], __dmul_rn(alpha, hp));
            Rr[e] = r;
            rn2 += r * r;
            rz_next += r * __ddiv_rn(r, lam[i] + lam[j]);
          })
          block_sum2(rn2, rz_next, red);
          const double rnorm = sqrt(rn2);
          if (!(rnorm > tol)) break;  // (:155-157)
          const double beta = rz_next / rz;
          SSN_FOR_IJ(m, {
            Pp[e] = __dadd_rn(__ddiv_rn(Rr[e], lam[i] + lam[j]), __dmul_rn(beta, Pp[e]));
          })
          __syncthreads();
          rz = rz_next;
        }
        double sl = 0.0;
        SSN_FOR_IJ(m, { sl += G[e] * Dd[e]; })
        slope = block_sum(sl, red);
        // non-descent fallback to the preconditioned gradient (:163-164)
        if (slope >= 0.0) {
          ++n_fallback;
          double s2 = 0.0;
          SSN_FOR_IJ(m, {
            const double z = __ddiv_rn(-G[e], lam[i] + lam[j]);
            Dd[e] = z;
            s2 += G[e] * z;
          })
          slope = block_sum(s2, red);
        }
      }

      // ---- Armijo backtracking with the exact objective change (:166-190)
      double t = 1.0;
      bool accepted = false;
      for (int bt = 0; bt < a.max_backtrack; ++bt) {
        ++n_trial;
        double first = 0.0;
        SSN_FOR_IJ(m, {
          const double dl = __dmul_rn(t, Dd[e]);
          Dl[e] = dl;
          first += G[e] * dl;
          Wt[e] = __dadd_rn(Wm[e], dl);      // == skew(omega + delta) for exactly skew omega, delta
        })
        first = block_sum(first, red);
        // K = I + trial trial, positive-definiteness test + inverse in shared memory
        double* Ks = smem;
        const int mp16 = round_up(m, 16), kld = frag_ld(mp16);
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
          SSN_FOR_IJ(m, { Pt[e] = Ks[i * kld + j]; })
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
    SSN_FOR_IJ(m, { Wout[e] = (T2[e] - T2[j * m + i]) / 2; })
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
  if (threadIdx.x == 0) {
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
  const int region = imax(8 * slot_doubles(MB), spd_region_doubles(32 * MB));
  return sizeof(double) * ((size_t)region + 2 * kWarps + kMaxM) + 16;
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
