/*
 * ssn.h -- C ABI of the B200 (sm_100a) batched dual Newton-CG solver for the
 * nearest real symplectic Stiefel matrix:
 *
 *     minimise ||X - T||_F^2   subject to   X^T J_2n X = J_2k,
 *     J_2r = [[0, I_r], [-I_r, 0]],   T, X in R^{2n x 2k},  m = 2k.
 *
 * All arithmetic is IEEE FP64.  Every pointer argument is a DEVICE pointer to
 * row-major, densely packed data unless stated otherwise; every call is
 * asynchronous on the given stream (0 = legacy default stream) and returns an
 * ssn_status.  No entry point allocates device memory: scratch comes from the
 * caller-owned workspace (ssn_workspace_bytes), so the caller (PyTorch in the
 * Python package) owns all memory, as in the reference where torch owns every
 * tensor and kernels receive raw pointers (src/symplectic_projection/
 * cuda_kernels.py:17-20).
 *
 * Limits: 1 <= k <= 64 (m <= 128), n >= k, batch >= 1.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root, yulinxie20/symplectic-stiefel-nearness).
 */
#ifndef SSN_H_
#define SSN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* ssn_stream_t; /* == cudaStream_t */

typedef enum {
  SSN_OK = 0,
  SSN_ERR_INVALID_ARGUMENT = 1, /* shape, pointer or option out of range      */
  SSN_ERR_CUDA = 2,             /* a CUDA runtime call or launch failed          */
  SSN_ERR_NEWTON_CAP = 3,       /* Newton cap reached (dual_recommended_hvp.py:191) */
  SSN_ERR_LINE_SEARCH = 4,      /* no descent step in MAX_BACKTRACK halvings (:190) */
  SSN_ERR_NONFINITE = 5,        /* NaN/Inf met in the input or the iteration      */
  SSN_ERR_EIGH = 6,             /* Jacobi sweeps did not converge                  */
  SSN_ERR_WORKSPACE = 7,        /* workspace missing or too small                  */
  SSN_ERR_SCRATCH_LIMIT = 8     /* problem larger than the fixed no-allocation scratch */
} ssn_status;

/* Per-instance status words written by ssn_solve / ssn_dual (int32 per target). */
enum {
  SSN_INSTANCE_CONVERGED = 0,
  SSN_INSTANCE_NEWTON_CAP = 3,
  SSN_INSTANCE_LINE_SEARCH = 4,
  SSN_INSTANCE_NONFINITE = 5,
  SSN_INSTANCE_EIGH = 6
};

/* Arithmetic of a solve (ssn_options.precision). */
enum {
  /* Plain FP64 throughout: the reference's algorithm step for step (same
   * iterates up to rounding), with a fully converged FP64 Jacobi eigenbasis. */
  SSN_PRECISION_FP64 = 0,
  /* Split precision: the Gram and the recovery are INT8 Ozaki products on the
   * tensor cores; the eigenbasis of the scaled Gram comes from a few FP32
   * Jacobi sweeps (ssn_options.eig_sweeps), is re-orthogonalised in FP64, and
   * the Newton iteration uses the full rotated Gram, so the solution is the
   * same dual optimum.  The early Newton steps run in FP32
   * (ssn_options.fp32_newton); the last Newton step(s), their line search and
   * positive-definiteness test, and the residual that declares convergence
   * are FP64.  Inputs and outputs are FP64 and every result is held to the
   * same acceptance bounds as the FP64 form. */
  SSN_PRECISION_SPLIT = 1
};

/* Solver constants; defaults follow dual_recommended_hvp.py:13-16. */
typedef struct {
  int max_newton;    /* 100 */
  int max_cg;        /* 150 */
  int max_backtrack; /* 40  */
  double feas_tol;   /* 1e-8: an instance is done when residual < feas_tol / 2 */
  int precision;     /* SSN_PRECISION_FP64 (default) or SSN_PRECISION_SPLIT */
  int eig_sweeps;    /* split form: Jacobi sweeps of the rough eigenbasis (max 24); 0 = default:
                        no sweep when every off-diagonal correlation of the scaled Gram is
                        below 0.1 (identity basis), else 1 */
  int preconditioner; /* SSN_PRECOND_EIGENBASIS (default) or SSN_PRECOND_ADAPTIVE */
  int fp32_newton;   /* split form: 0 (default) or 1 run the early Newton steps in FP32 where
                        their state fits on chip (m <= 64, or m <= 96 with two CTAs per
                        instance), until the FP32 residual is below 1e-5; -1 keeps every
                        Newton step in FP64.  Ignored by the FP64 form. */
  int reserved[4];
} ssn_options;

/* CG preconditioner (ssn_options.preconditioner). */
enum {
  /* skew(R / (lambda_i + lambda_j)) in the eigenbasis of the scaled Gram: the
   * reference's (dual_recommended_hvp.py:113-114), exact at omega = 0.  The
   * default, in both precision forms. */
  SSN_PRECOND_EIGENBASIS = 0,
  /* the diagonal of the Hessian at the current omega in the working basis,
   * P_ii Sr_jj + P_jj Sr_ii - 2 P_ij Sr_ij + 2 Q_ij Si_ij (lambda_i + lambda_j at
   * omega = 0), with the full rotated Gram in the sandwich and the basis
   * refined to FP64 orthogonality.  No counterpart in the reference: it keeps
   * CG short on ill-conditioned targets, where the reference's preconditioner
   * lets CG saturate and the Newton cap is reached.  It reaches the same dual
   * optimum along another path, so on targets whose dual is very flat the
   * result agrees with the reference's only to that flatness. */
  SSN_PRECOND_ADAPTIVE = 1
};

/*
 * Launch parameters chosen by an autotuner for one problem class.  ssn_solve
 * and ssn_solve_ragged (per shape group) look the table up by (precision, m,
 * n, batch); the first matching entry wins, and a field of 0 keeps the
 * library's built-in rule for that parameter.  No counterpart in the
 * reference, which hard-codes its chunking and tiles (dual_recommended_hvp.py:13,
 * gram_triangle_reflect.py:32-36).  The parameters change only the schedule:
 * results agree with the built-in schedule's to the products' rounding.
 */
typedef struct {
  int precision;      /* SSN_PRECISION_FP64 or SSN_PRECISION_SPLIT */
  int m;              /* 2k */
  int n_min, n_max;   /* inclusive range of n */
  int batch_min, batch_max; /* inclusive range of the batch (or shape group) size */
  int gram_splits;    /* FP64 Gram: row splits per instance, 1..64 */
  int gram_chunks;    /* split-form Gram: row chunks per instance, 1..32 */
  int recover_parts;  /* split-form recovery: parts of each (instance, column group)'s row tiles, 1..1024 */
  int cluster;        /* Newton kernels: CTAs per instance, 1 or 2 (2 needs m > 32) */
} ssn_tuning;

/* Install `count` entries (copied; at most 1024; count 0 clears the table).
 * Returns SSN_ERR_INVALID_ARGUMENT, leaving the table unchanged, if any entry
 * is out of range.  Not to be called while another host thread is inside a
 * solve.  ssn_get_tuning copies up to `capacity` entries out and returns how
 * many are installed. */
int ssn_set_tuning(const ssn_tuning* entries, int count);
int ssn_get_tuning(ssn_tuning* entries, int capacity);

/* Library version as 10000*major + 100*minor + patch. */
int ssn_version(void);
/* Static string naming a status code. */
const char* ssn_status_string(int status);
/* Fill *opt with the reference defaults. */
void ssn_default_options(ssn_options* opt);

/* Bytes of device workspace ssn_solve needs for this problem size. */
size_t ssn_workspace_bytes(int batch, int n, int m);

/*
 * Full solve: T [batch, 2n, m] -> X [batch, 2n, m], omega [batch, m, m],
 * iterations int64 [batch] (Newton updates per instance), status int32 [batch].
 * opt->precision selects the plain FP64 form or the split-precision form.
 * Replaces symplectic_projection.solve (dual_recommended_hvp.py:231-242),
 * i.e. gram_chunks (:79-96) + dual_batch (:99-191) + recover_matmul (:194-228),
 * with device-resident input and output (no chunked PCIe staging).
 * Returns SSN_OK when the work was enqueued; per-instance outcomes are in
 * `status` once the stream reaches them (the reference raises RuntimeError
 * for the whole batch when any instance hits a cap; the Python layer does).
 */
int ssn_solve(const double* T, double* X, double* omega, int64_t* iterations,
              int32_t* status, int batch, int n, int m,
              void* workspace, size_t workspace_bytes,
              const ssn_options* opt, ssn_stream_t stream);

/*
 * Ragged batch: `count` targets of different shapes in one call.  Instance i is
 * T_i [2 n[i], m[i]] row-major at T + t_offset[i] (offsets in doubles, even),
 * its X_i at X + t_offset[i] and its omega_i [m[i], m[i]] at omega +
 * w_offset[i]; iterations[i] and status[i] as in ssn_solve.  n, m, t_offset and
 * w_offset are HOST arrays.  The instances are grouped by shape; every group is
 * gathered into a contiguous batch, solved by the ssn_solve pipeline and
 * scattered back, with the groups running concurrently on streams forked from
 * (and joined back into) `stream`.  The plan goes to the device with one copy
 * from pageable host memory, which waits for the work already on `stream`.
 * Replaces a loop of symplectic_projection.solve calls, one per shape
 * (dual_recommended_hvp.py:231-242).
 */
size_t ssn_ragged_workspace_bytes(int count, const int* n, const int* m);
int ssn_solve_ragged(const double* T, double* X, double* omega, int64_t* iterations,
                     int32_t* status, int count, const int* n, const int* m,
                     const int64_t* t_offset, const int64_t* w_offset,
                     void* workspace, size_t workspace_bytes,
                     const ssn_options* opt, ssn_stream_t stream);

/*
 * Gradient through the solve (the adjoint): given T [batch, 2n, m], the solve's
 * omega [batch, m, m] and the loss gradients G = dL/dX [batch, 2n, m] and Gw =
 * dL/d omega [batch, m, m] (either may be NULL), writes dT = dL/dT [batch, 2n, m].
 * Implicit differentiation of the dual optimality condition at omega: one
 * preconditioned CG solve with the solver's Hessian-vector product per instance
 * (tolerance 1e-12 relative, at most max(opt->max_cg, 10 m) steps) and FP64
 * tall-skinny products.  status[b]: 0 ok, 3 CG cap, 5 non-finite or I + omega^2
 * not positive definite (dT of that instance is NaN); cg_iterations may be NULL.
 * No counterpart in the reference, which solves under torch.no_grad
 * (dual_recommended_hvp.py:231); its operators are the reference's HVP
 * (hvp_fused.py:22-53), sandwich (dual_recommended_hvp.py:67-71) and recovery
 * (recovery_fused.py:19-30).
 */
size_t ssn_adjoint_workspace_bytes(int batch, int n, int m);
int ssn_adjoint(const double* T, const double* omega, const double* G, const double* Gw,
                double* dT, int32_t* status, int32_t* cg_iterations, int batch, int n, int m,
                void* workspace, size_t workspace_bytes, const ssn_options* opt,
                ssn_stream_t stream);

/*
 * Gram products of T = [A; D]:  Cr = A^T A + D^T D,  Ci = A^T D - D^T A
 * (overwritten, not accumulated).  A, D are [batch, rows, m] with batch
 * strides ab_stride (elements, >= rows*m).  Replaces gram_add_
 * (gram_triangle_reflect.py:19-36; kernels gram_offdiag / gram_diagonal,
 * gram_triangle_reflect.cu:51-104).  Needs ssn_gram_workspace_bytes bytes.
 * opt NULL or SSN_PRECISION_FP64: FP64 tensor-core (DMMA) products.
 * SSN_PRECISION_SPLIT: INT8 Ozaki products on the tcgen05 tensor cores (six
 * balanced 8-bit digits per value with per-(row chunk, column) power-of-two
 * scales, exact INT32 accumulation, FP64 recombination): relative error about
 * 1e-12 of max|T|^2 per entry for Gaussian T.
 */
size_t ssn_gram_workspace_bytes(int batch, int rows, int m);
int ssn_gram(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
             int batch, int rows, int m, void* workspace, size_t workspace_bytes,
             const ssn_options* opt, ssn_stream_t stream);

/*
 * ssn_gram without a workspace argument, for callers that cannot allocate
 * device memory at the call (a host framework whose pooling allocator owns the
 * device, or a caller that must never reach cudaMalloc).  No counterpart in the
 * reference.  Its scratch is one fixed array of ssn_gram_noalloc_scratch_bytes()
 * (16 MiB) in the library's device memory, held by every GPU that loads the
 * library until exit.  A call needs batch * 2 * m^2 doubles of it (more row
 * splits are used when they fit); larger calls return SSN_ERR_SCRATCH_LIMIT
 * without launching.  Every call shares the array: calls that overlap on the
 * GPU race and must be serialised by the caller.  The first call on a device
 * resolves the array's address (cudaGetSymbolAddress) and should come before
 * any stream capture.  No call allocates.
 */
size_t ssn_gram_noalloc_scratch_bytes(void);
int ssn_gram_noalloc(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                     int batch, int rows, int m, ssn_stream_t stream);

/*
 * Cross Gram of two tall-skinny pairs G = [Ga; Gd] and T = [A; D]:
 *   Mr = Ga^T A + Gd^T D,   Mi = Ga^T D - Gd^T A   (M = G^H b style product of
 * the complex views g = Ga + i Gd, b = A + i D: M = conj(g)^T b).
 * Ga, Gd are [batch, rows, m] with batch stride g_stride; A, D with ab_stride;
 * Mr, Mi are [batch, m, m] contiguous (overwritten).  FP64 tensor-core (DMMA)
 * products, row-split with a fixed-order sum of the split partials.  The
 * reference computes these contractions with torch matmuls in its acceptance
 * test (experiment.py:105-137: the tangent projection (J X)^T E of
 * baselines/geometry.py:22-40) and in the adjoint's right-hand side.  Needs
 * ssn_cross_gram_workspace_bytes bytes.
 */
size_t ssn_cross_gram_workspace_bytes(int batch, int rows, int m);
int ssn_cross_gram(const double* Ga, const double* Gd, int64_t g_stride, const double* A,
                   const double* D, int64_t ab_stride, double* Mr, double* Mi, int batch, int rows,
                   int m, void* workspace, size_t workspace_bytes, ssn_stream_t stream);

/*
 * Recovery products:  Ur = A P^T + D Q^T,  Ui = D P^T - A Q^T.
 * A, D, Ur, Ui are [batch, rows, m] with batch strides ab_stride / u_stride;
 * P, Q are [batch, m, m] contiguous.  Replaces recover_block
 * (recovery_fused.py:19-30; kernel recover_fused, recovery_fused.cu:2-41).
 * opt NULL or SSN_PRECISION_FP64: FP64 tensor-core (DMMA) products, no
 * workspace (workspace may be NULL).  SSN_PRECISION_SPLIT: INT8 Ozaki
 * products on the tcgen05 tensor cores (six balanced digits of every row of
 * [A D] and of [P Q], [-Q P], exact INT32 accumulation, FP64 recombination;
 * each entry within about 2^-45 K of its largest row contributions; Ur and Ui
 * 16-byte aligned); needs
 * ssn_recover_workspace_bytes of workspace.
 */
size_t ssn_recover_workspace_bytes(int batch, int rows, int m);
int ssn_recover(const double* A, const double* D, int64_t ab_stride,
                const double* P, const double* Q, double* Ur, double* Ui, int64_t u_stride,
                int batch, int rows, int m, void* workspace, size_t workspace_bytes,
                const ssn_options* opt, ssn_stream_t stream);

/*
 * Symmetric eigendecomposition of the scaled Gram matrix, Cr / s = V diag(w) V^T
 * with s = max(1, trace(Cr)/m) (dual_recommended_hvp.py:106-108, where the
 * reference calls torch.linalg.eigh).  Cyclic two-sided Jacobi; eigenvalues
 * ascending.  opt NULL or opt->precision == SSN_PRECISION_FP64: FP64 rotations
 * until convergence.  SSN_PRECISION_SPLIT: opt->eig_sweeps FP32 sweeps, a rough
 * basis for ssn_newton's split form (V only approximately orthogonal).
 * scale and sweeps (Jacobi sweeps per instance) may be NULL.  The workspace
 * (ssn_eigh_workspace_bytes) holds the rotation log.
 */
size_t ssn_eigh_workspace_bytes(int batch, int m);
int ssn_eigh(const double* Cr, double* values, double* vectors, double* scale,
             int32_t* sweeps, int batch, int m, void* workspace, size_t workspace_bytes,
             const ssn_options* opt, ssn_stream_t stream);

/*
 * Dual Newton-CG on given Gram matrices: (Cr, Ci) -> omega, and the final
 * inverse parts P + iQ = (I + i omega)^-1, all in the original basis, plus
 * iterations and status (either precision form, opt->precision).  Replaces dual_batch (dual_recommended_hvp.py:99-191)
 * with the `final` cache (:131-134).  Needs ssn_dual_workspace_bytes.
 */
size_t ssn_dual_workspace_bytes(int batch, int m);
int ssn_dual(const double* Cr, const double* Ci, double* omega, double* P, double* Q,
             int64_t* iterations, int32_t* status, int batch, int m,
             void* workspace, size_t workspace_bytes, const ssn_options* opt,
             ssn_stream_t stream);

/*
 * The Newton-CG part of ssn_dual alone, given the eigendecomposition from
 * ssn_eigh (values, vectors, scale, and its per-instance status eig_status,
 * which may be NULL).  counters (may be NULL) receives int32 [batch, 8]:
 * Newton steps run, Hessian-vector products, line-search trials and fallbacks
 * of the FP64 iteration, then the same four of the split form's FP32 phase
 * (zeros when it does not run).
 * Cr (the unscaled Gram) is read only with the full rotated Gram (the split
 * form, or the adaptive preconditioner), where it is required; it may be NULL
 * otherwise.
 * Replaces dual_batch (dual_recommended_hvp.py:109-191) after the eigh call.
 * Needs ssn_newton_workspace_bytes.
 */
size_t ssn_newton_workspace_bytes(int batch, int m);
int ssn_newton(const double* Cr, const double* Ci, const double* values, const double* vectors,
               const double* scale, const int32_t* eig_status, double* omega, double* P, double* Q,
               int64_t* iterations, int32_t* status, int32_t* counters, int batch, int m,
               void* workspace, size_t workspace_bytes, const ssn_options* opt,
               ssn_stream_t stream);

/*
 * Measurement helper with no counterpart in the reference.  While set, every
 * Newton-CG run started from the calling host thread (ssn_newton, ssn_dual,
 * ssn_solve) records events[0..3] on its stream: before the basis set-up,
 * before the split form's FP32 Newton phase, before the FP64 iteration, and
 * after it (events[1] and [2] coincide when no FP32 phase runs).  events: four
 * cudaEvent_t handles owned by the caller; NULL stops the recording.
 */
int ssn_set_newton_events(void* const* events);

/*
 * Measurement helper with no counterpart in the reference: launches a
 * dependent-chain-free FP64 DMMA loop on every SM so a caller can time the
 * FP64 tensor-pipe peak with its own events (the roofline denominator of the
 * FP64 kernels).  sink: device buffer of >= 8192 doubles.  *flops receives the
 * FP64 flops the launch performs.
 */
int ssn_probe_fp64_mma(double* sink, int iters, double* flops, ssn_stream_t stream);

/*
 * Check of the INT8 tensor-core path with no counterpart in the reference:
 * one CTA computes C[128 x n] = A[128 x k] * B[n x k]^T (row-major int8 in,
 * int32 out) with tcgen05.mma kind::i8 from no-swizzle K-major shared-memory
 * operands into a TMEM accumulator.  The split-precision Gram and recovery
 * kernels are built from the same descriptors.  16 <= n <= 256, n % 16 == 0,
 * 32 <= k <= 256, k % 32 == 0, A and B 16-byte aligned.  *stall (device) is
 * set to 1 if the MMA completion was not observed within the wait bound.
 */
int ssn_probe_s8_mma(const int8_t* A, const int8_t* B, int32_t* C, int n, int k, int* stall,
                     ssn_stream_t stream);

/* ---- component operations (mirrors of the reference kernel wrappers) ----
 * All matrices [batch, m, m] contiguous FP64; vectors [batch] or [batch, m]. */

/* U = E Sr, V = E Si.  Replaces inner_products (hvp_fused.py:22-34, hvp_inner, hvp_fused.cu:2-38). */
int ssn_inner_products(const double* E, const double* Sr, const double* Si,
                       double* U, double* V, int batch, int m, ssn_stream_t stream);
/* H = Z - Z^T with Z = P U - Q V.  Replaces outer_skew (hvp_fused.py:37-53, hvp_outer*, hvp_fused.cu:83-238). */
int ssn_outer_skew(const double* P, const double* Q, const double* U, const double* V,
                   double* H, int batch, int m, ssn_stream_t stream);
/* Yr = P diag(values) - Q Ci, Yi = P Ci + Q diag(values).
 * Replaces sandwich_front (hvp_fused.py:56-69, hvp_sandwich_front, hvp_fused.cu:41-80). */
int ssn_sandwich_front(const double* values, const double* Ci, const double* P, const double* Q,
                       double* Yr, double* Yi, int batch, int m, ssn_stream_t stream);
/* change[b] = <gradient, delta> + <V, delta_Sr + trial delta_Si>.
 * Replaces line_change (hvp_fused.py:72-87, hvp_line_partial/finish, hvp_fused.cu:259-371). */
int ssn_line_change(const double* gradient, const double* delta, const double* V,
                    const double* delta_Sr, const double* trial, const double* delta_Si,
                    double* change, int batch, int m, ssn_stream_t stream);
/* out = 0.5 (R/den - (R/den)^T).  Replaces fused_precondition (hvp_fused.py:110-117, hvp_fused.cu:374-387). */
int ssn_precondition(const double* R, const double* denominator, double* out,
                     int batch, int m, ssn_stream_t stream);
/* new_direction = direction + alpha p, new_r = r - alpha Hp (separately rounded).
 * Replaces cg_update (hvp_fused.py:120-130, hvp_fused.cu:389-405). */
int ssn_cg_update(const double* direction, const double* r, const double* p, const double* Hp,
                  const double* alpha, double* new_direction, double* new_r,
                  int batch, int m, ssn_stream_t stream);
/* out = active ? z + beta p : 0.  Replaces cg_next (hvp_fused.py:133-143, hvp_fused.cu:407-420). */
int ssn_cg_next(const double* z, const double* p, const double* beta, const uint8_t* active,
                double* out, int batch, int m, ssn_stream_t stream);
/* P = (L L^T)^-1 from a lower Cholesky factor, any m <= 128.  Replaces
 * inverse_from_cholesky (cholesky_inverse_kernel.py:27-39, m = 128 only there). */
int ssn_inverse_from_cholesky(const double* L, double* P, int batch, int m, ssn_stream_t stream);
/* P = K^-1 for SPD K with a positive-definiteness flag (info[b] = 0 when every
 * pivot is positive, else the 1-based failing pivot), the device equivalent of
 * torch.linalg.cholesky_ex + construct_inverse (dual_recommended_hvp.py:173-176). */
int ssn_spd_inverse(const double* K, double* P, int32_t* info, int batch, int m, ssn_stream_t stream);
/* L = chol(I + omega omega), lower triangular, for skew omega [batch, m, m]
 * (dual_recommended_hvp.py:63 and :173, torch.linalg.cholesky(I + omega @ omega);
 * dual_batch returns this L).  info[b] = 0, or the 1-based order of the first
 * leading minor that is not positive definite (L's columns from there are 0). */
int ssn_cholesky_k(const double* omega, double* L, int32_t* info, int batch, int m, ssn_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SSN_H_ */
