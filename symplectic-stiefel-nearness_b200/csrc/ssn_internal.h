// ssn_internal.h -- host-side launch helpers shared by the translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ssn.h"

namespace ssn {

// Number of m x m FP64 matrices of per-instance dual workspace (the last one holds
// small per-instance data: the FP32 phase's Newton updates and counters).
constexpr int kDualMats = 23;

// SM count of the current device, cached per device index (148 on B200; 148 if
// the query fails).  Safe to call from several host threads.
int current_device_sm_count();

// The autotuned launch parameters that apply to the launches the calling host thread
// is enqueueing (set by ssn_solve for its problem class), or null: the built-in rules.
const ssn_tuning* active_tuning();
// The first installed entry matching (precision, n, m, batch), or null.
const ssn_tuning* find_tuning(int precision, int n, int m, int batch);
// Makes `t` the calling thread's active tuning for the scope's lifetime.
struct TuningScope {
  const ssn_tuning* prev;
  explicit TuningScope(const ssn_tuning* t);
  ~TuningScope();
  TuningScope(const TuningScope&) = delete;
  TuningScope& operator=(const TuningScope&) = delete;
};

struct DualArgs {
  int m;
  int max_newton, max_cg, max_backtrack;
  double feas_tol;
  const double* Cr;        // [B,m,m] (unscaled)
  const double* Ci;        // [B,m,m]
  const double* values;    // [B,m]   eigenvalues of Cr/s
  const double* vectors;   // [B,m,m] eigenvectors
  const double* scale;     // [B]
  const int32_t* eig_status;  // [B]
  const int32_t* sweeps;      // [B] Jacobi sweeps of the basis, or null: 0 means the identity
                              // basis (a permutation), which needs no re-orthogonalisation
  double* work;            // [B, kDualMats, m, m]
  double* omega;           // [B,m,m] out, original basis
  double* P;               // [B,m,m] out
  double* Q;               // [B,m,m] out
  int64_t* iterations;     // [B] out
  int32_t* status;         // [B] out
  int32_t* counters;       // [B,8] out (may be null): newton steps, hvps, trials, fallbacks of the
                           // FP64 iteration, then of the FP32 phase (zero when it does not run)
  // Full rotated Gram: the kernel works with V^T (Cr/s) V in the sandwich
  // instead of assuming it is exactly diag(lambda), and takes lambda from its
  // diagonal.  Needed when the vectors only roughly diagonalise Cr/s (split
  // form), and used with the adaptive preconditioner, where the iteration can
  // pass near-singular I + i omega whose inverse would amplify the eigenbasis'
  // rounding residual.  orthogonalize: first make V orthogonal to FP64 rounding
  // with two Newton-Schulz steps V <- V (3I - V^T V) / 2.
  int approx_basis;
  int orthogonalize;
  // Preconditioner of the CG (and of the fallback direction): 0 the reference's
  // skew(R / (lambda_i + lambda_j)), exact for omega = 0; 1 the diagonal of the
  // Hessian at the current omega in the working basis,
  //   P_ii Sr_jj + P_jj Sr_ii - 2 P_ij Sr_ij + 2 Q_ij Si_ij,
  // which equals lambda_i + lambda_j at omega = 0 and keeps CG short where
  // omega is large (ill-conditioned targets).
  int adaptive_precond;
  // Instances whose Newton kernels share the GPU at the same time (0: this batch
  // alone).  A 2-CTA cluster per instance pays only while SMs would otherwise idle.
  int concurrent;
  // Split form: run the early Newton steps in FP32 (dual32_kernel) where the FP32
  // state fits on chip, then the FP64 iteration warm-started from its omega.
  int fp32_newton;
  // dual_kernel phase: 0 the whole solve; 1 the basis set-up only (rotated Gram into
  // the workspace); 2 the Newton iteration and exit after a phase-1 launch, started
  // from the FP32 phase's omega when it took at least one Newton update.
  int phase;
};

// The FP32 early Newton phase of the split form (ssn_dual32.cu).
struct Dual32Args {
  int m;
  int max_newton, max_cg, max_backtrack;
  double switch_tol;       // hand over to the FP64 iteration once the FP32 residual is below this
  double* work;            // [B, kDualMats, m, m]: the phase-1 set-up in, omega and counters out
  const double* scale;     // [B]
  const int32_t* eig_status;  // [B] (may be null)
  int adaptive;            // the Hessian-diagonal preconditioner for the CG steps
};
bool dual32_supported(int m, int cluster);
cudaError_t launch_dual32(const Dual32Args& args, int batch, int cluster, cudaStream_t stream);
int dual_cluster_size(int batch, int m);

// Adjoint of the solve (implicit gradient), one CTA per instance.
constexpr int kAdjointMats = 10;
struct AdjointArgs {
  int m, max_cg;
  double tol;              // CG stops at ||r|| <= tol ||Gamma||
  const double* Cr;        // [B,m,m] b^H b, real and imaginary parts
  const double* Ci;
  const double* Mr;        // [B,m,m] g^H b
  const double* Mi;
  const double* omega;     // [B,m,m] the solve's multiplier (original basis)
  const double* Gw;        // [B,m,m] dL/d omega, or null
  double* work;            // [B, kAdjointMats, m, m]
  double* P;               // [B,m,m] out: K = P + iQ
  double* Q;
  double* Pn;              // [B,m,m] out: recovery operands of b N
  double* Qn;
  int32_t* status;         // [B] out
  int32_t* cg_iters;       // [B] out (may be null)
};
cudaError_t launch_adjoint(const AdjointArgs& args, int batch, cudaStream_t stream);
// Mr = Ga^T A + Gd^T D, Mi = Ga^T D - Gd^T A (row-split partials summed in a fixed order).
cudaError_t launch_cross_gram(const double* Ga, const double* Gd, int64_t g_stride, const double* A,
                              const double* D, int64_t ab_stride, double* Mr, double* Mi, int batch, int rows,
                              int m, double* partial, cudaStream_t stream);

size_t eigh_smem_bytes(int m);
size_t eigh_workspace_bytes(int batch, int m);
cudaError_t launch_eigh(const double* Cr, double* values, double* vectors, double* scale,
                        int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                        cudaStream_t stream);
// Jacobi capped at max_sweeps (no convergence requirement), FP32 or FP64 rotations:
// the rough eigenbasis of the split-precision form.  skip_corr > 0: an instance whose
// largest off-diagonal correlation |c_pq| / sqrt(c_pp c_qq) is below skip_corr gets no
// sweep (identity basis).
cudaError_t launch_eigh_approx(const double* Cr, double* values, double* vectors, double* scale,
                               int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                               int max_sweeps, bool fp32, float skip_corr, cudaStream_t stream);
// side_fork (may be null) is recorded on the stream where the Newton steps start (before
// the FP32 phase, else before the FP64 iteration): work that waits on it overlaps them.
cudaError_t launch_dual(const DualArgs& args, int batch, cudaStream_t stream, cudaEvent_t side_fork = nullptr);
// Measurement hook behind ssn_set_newton_events (per host thread; null clears).
void set_newton_events(void* const* events);
// The whole uniform-batch solve (the body of ssn_solve) on one stream; `concurrent` as in DualArgs.
int solve_batch(const double* T, double* X, double* omega, int64_t* iterations, int32_t* status, int batch,
                int n, int m, void* workspace, const ssn_options* opt, cudaStream_t stream, int concurrent);
size_t solve_workspace_bytes(int batch, int n, int m);
bool solve_options_ok(const ssn_options* opt);
cudaError_t launch_probe_fp64_mma(double* sink, int iters, double* flops, cudaStream_t stream);
cudaError_t launch_probe_s8_mma(const int8_t* A, const int8_t* B, int32_t* C, int n, int k, int* stall,
                                cudaStream_t stream);

size_t gram_partial_doubles(int batch, int rows, int m);
// number of row splits launch_gram uses for this shape when capped at max_splits
int gram_splits(int batch, int rows, int max_splits);
cudaError_t launch_gram(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                        int batch, int rows, int m, double* partial, cudaStream_t stream,
                        int max_splits = 1 << 30);
// Fixed-order sum of row-split partials [B][splits][2][m][m] (Cr part, G part) into Cr and Ci = G - G^T.
cudaError_t launch_gram_finalize(const double* partial, double* Cr, double* Ci, int batch, int m, int splits,
                                 cudaStream_t stream);
// Split-precision (INT8 Ozaki, tcgen05) Gram.  Workspace: ozaki_gram_workspace_bytes.
size_t ozaki_gram_workspace_bytes(int batch, int rows, int m);
cudaError_t launch_gram_ozaki(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                              int batch, int rows, int m, void* workspace, int32_t* row_exp, int* stall,
                              cudaStream_t stream);
// Split-precision (INT8 Ozaki, tcgen05) recovery Ur = A P^T + D Q^T, Ui = D P^T - A Q^T in two parts:
// the digits of W = [A | D] (independent of P, Q, so they can run early on another stream),
// then the products.  Both use the same workspace (ozaki_recover_workspace_bytes).
size_t ozaki_recover_workspace_bytes(int batch, int rows, int m);
cudaError_t launch_recover_wdigits(const double* A, const double* D, int64_t ab_stride, int batch, int rows, int m,
                                   void* workspace, cudaStream_t stream);
cudaError_t launch_recover_products(const double* P, const double* Q, double* Ur, double* Ui, int64_t u_stride,
                                    int batch, int rows, int m, void* workspace, cudaStream_t stream);
cudaError_t launch_recover_ozaki(const double* A, const double* D, int64_t ab_stride, const double* P,
                                 const double* Q, double* Ur, double* Ui, int64_t u_stride, int batch, int rows,
                                 int m, void* workspace, cudaStream_t stream);
cudaError_t launch_recover(const double* A, const double* D, int64_t ab_stride, const double* P,
                           const double* Q, double* Ur, double* Ui, int64_t u_stride, int batch,
                           int rows, int m, cudaStream_t stream);

// component kernels (mirrors of the reference wrappers)
cudaError_t launch_inner_products(const double* E, const double* Sr, const double* Si, double* U,
                                  double* V, int batch, int m, cudaStream_t stream);
cudaError_t launch_outer_skew(const double* P, const double* Q, const double* U, const double* V,
                              double* H, int batch, int m, double* scratch, cudaStream_t stream);
cudaError_t launch_sandwich_front(const double* values, const double* Ci, const double* P,
                                  const double* Q, double* Yr, double* Yi, int batch, int m,
                                  cudaStream_t stream);
cudaError_t launch_line_change(const double* g, const double* delta, const double* V,
                               const double* dSr, const double* trial, const double* dSi,
                               double* change, int batch, int m, cudaStream_t stream);
cudaError_t launch_precondition(const double* R, const double* den, double* out, int batch, int m,
                                cudaStream_t stream);
cudaError_t launch_cg_update(const double* d, const double* r, const double* p, const double* Hp,
                             const double* alpha, double* nd, double* nr, int batch, int m,
                             cudaStream_t stream);
cudaError_t launch_cg_next(const double* z, const double* p, const double* beta,
                           const uint8_t* active, double* out, int batch, int m,
                           cudaStream_t stream);
cudaError_t launch_spd_inverse(const double* K, double* P, int32_t* info, int batch, int m,
                               cudaStream_t stream);
cudaError_t launch_inverse_from_cholesky(const double* L, double* P, int batch, int m,
                                         cudaStream_t stream);
cudaError_t launch_cholesky_k(const double* omega, double* L, int32_t* info, int batch, int m,
                              cudaStream_t stream);

}  // namespace ssn
