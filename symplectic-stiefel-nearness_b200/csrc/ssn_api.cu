// ssn_api.cu -- the extern "C" entry points declared in include/ssn.h:
// argument validation, workspace layout and the solve pipeline
//   Gram (split-K + finalize) -> Jacobi eigh -> persistent dual Newton-CG -> recovery,
// all enqueued on the caller's stream, with no host synchronisation.
#include <stdint.h>
#include <string.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace {

using namespace ssn;

constexpr int kVersion = 100;  // 0.1.0

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

bool shape_ok(int batch, int m) { return batch >= 1 && m >= 2 && m <= kMaxM && (m % 2) == 0; }

int cuda_status(cudaError_t e) { return e == cudaSuccess ? SSN_OK : SSN_ERR_CUDA; }

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Workspace layout of ssn_solve (byte offsets, 256-byte aligned sections).
struct SolveLayout {
  size_t cr, ci, values, vectors, scale, pfin, qfin, work, eig_status, sweeps, eig_ws, rec, stall, total;
};

SolveLayout solve_layout(int batch, int n, int m) {
  const size_t mm = (size_t)m * m;
  SolveLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align_up(off + bytes, 256);
    return at;
  };
  L.cr = take(sizeof(double) * batch * mm);
  L.ci = take(sizeof(double) * batch * mm);
  L.values = take(sizeof(double) * batch * m);
  L.vectors = take(sizeof(double) * batch * mm);
  L.scale = take(sizeof(double) * batch);
  L.pfin = take(sizeof(double) * batch * mm);
  L.qfin = take(sizeof(double) * batch * mm);
  // the Gram partial sums share the Newton workspace (they are dead before it is used)
  const size_t work = sizeof(double) * (size_t)batch * kDualMats * mm;
  // each form's Gram plan under that form's tuning entry, as solve_batch will run it
  size_t partial, oz;
  {
    TuningScope scope(find_tuning(SSN_PRECISION_FP64, n, m, batch));
    partial = sizeof(double) * gram_partial_doubles(batch, n, m);
  }
  {
    TuningScope scope(find_tuning(SSN_PRECISION_SPLIT, n, m, batch));
    oz = ozaki_gram_workspace_bytes(batch, n, m);
  }
  if (oz > partial) partial = oz;
  L.work = take(work > partial ? work : partial);
  L.eig_status = take(sizeof(int32_t) * batch);
  L.sweeps = take(sizeof(int32_t) * batch);
  L.eig_ws = take(eigh_workspace_bytes(batch, m));
  // split form: the recovery's digits of [A | D] (made early, alongside the Newton phase)
  L.rec = take(ozaki_recover_workspace_bytes(batch, n, m));
  L.stall = take(sizeof(int32_t) * 4);                        // split form: tensor-core wait-limit flag
  L.total = off;
  return L;
}

struct DualLayout {
  size_t values, vectors, scale, work, eig_status, eig_ws, total;
};

DualLayout dual_layout(int batch, int m) {
  const size_t mm = (size_t)m * m;
  DualLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align_up(off + bytes, 256);
    return at;
  };
  L.values = take(sizeof(double) * batch * m);
  L.vectors = take(sizeof(double) * batch * mm);
  L.scale = take(sizeof(double) * batch);
  L.work = take(sizeof(double) * (size_t)batch * kDualMats * mm);
  L.eig_status = take(sizeof(int32_t) * batch);
  L.eig_ws = take(eigh_workspace_bytes(batch, m));
  L.total = off;
  return L;
}

// One FP32 sweep: on Gaussian targets it also takes the fewest CG steps (1 sweep: 15.3
// HVPs per target at 64 x 8192 x 96; 2: 17.5; 3 and 5: 17.7), since the full rotated
// Gram in the sandwich carries what the rough basis leaves off the diagonal.
constexpr int kDefaultEigSweeps = 1;
// With the default sweep count, a Gram whose off-diagonal correlations are all below
// this keeps the identity basis: on Gaussian targets (largest correlation about
// 4 / sqrt(2n)) that takes fewer Newton and CG steps than a sweep (64 x 8192 x 96:
// 450 Newton steps and 772 HVPs, against 512 and 978), and the full rotated Gram in
// the sandwich carries the off-diagonal part.  Ill-conditioned Grams keep the sweep.
constexpr float kRoughBasisSkip = 0.1f;

// The split form's two streams.  The recovery's W digits depend only on T, so a
// side stream of the LOWEST priority makes them while the Newton kernels run, and
// the solve itself runs on a stream of the HIGHER priority: the block scheduler
// hands freed SMs to pending CTAs of the higher-priority stream first, so the
// digit kernel's short CTAs (2048 at 64 x 8192 x 96) fill what the Newton kernels
// leave over instead of delaying them.  (At equal priority they delayed the eigen
// and Newton launches by about 0.23 ms there, nearly the digit kernel's whole run.)
// Streams and events are created once per host thread and kept, and every fork and
// join is an event, so a call can be captured into a CUDA graph (they become edges).
constexpr int kMaxDevices = 64;

// The side stream of the calling thread on the current device.  Calls from one
// thread share it; the events order each call's side work correctly.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t forked = nullptr, done = nullptr;   // `forked`: recorded by launch_dual
  cudaError_t open() {
    struct Pool {
      cudaStream_t stream = nullptr;
      cudaEvent_t forked = nullptr, done = nullptr;
    };
    thread_local Pool pool[kMaxDevices];
    int dev = 0, least = 0, greatest = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    Pool& p = pool[dev];
    if (!p.stream) {
      e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
      if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&p.stream, cudaStreamNonBlocking, least);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.forked, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    stream = p.stream;
    forked = p.forked;
    done = p.done;
    return cudaSuccess;
  }
  cudaError_t wait_forked() { return cudaStreamWaitEvent(stream, forked, 0); }
  cudaError_t record() { return cudaEventRecord(done, stream); }
  cudaError_t join(cudaStream_t parent) { return cudaStreamWaitEvent(parent, done, 0); }
};

// The stream the split solve runs on: the caller's own when its priority is above
// the lowest, else a highest-priority stream forked from it (one per caller stream,
// thread and device, up to kMainSlots of them; past that the caller's stream).
struct MainStream {
  static constexpr int kMainSlots = 32;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaError_t fork(cudaStream_t parent) {
    struct Slot {
      int dev = -1;
      cudaStream_t parent = nullptr, stream = nullptr;
      cudaEvent_t forked = nullptr, done = nullptr;
    };
    thread_local Slot slots[kMainSlots];
    stream = parent;
    done = nullptr;
    int dev = 0, least = 0, greatest = 0, pr = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamGetPriority(parent, &pr);
    if (e != cudaSuccess) return e;
    if (greatest >= least || pr < least) return cudaSuccess;
    Slot* s = nullptr;
    for (Slot& c : slots) {
      if (c.dev == dev && c.parent == parent) {
        s = &c;
        break;
      }
      if (!s && c.dev < 0) s = &c;
    }
    if (!s) return cudaSuccess;                  // every slot taken: stay on the caller's stream
    if (s->dev < 0) {
      // no stream is created while the caller's stream is being captured
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if ((e = cudaStreamIsCapturing(parent, &cs)) != cudaSuccess) return e;
      if (cs != cudaStreamCaptureStatusNone) return cudaSuccess;
      e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, greatest);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->forked, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
      s->dev = dev;
      s->parent = parent;
    }
    e = cudaEventRecord(s->forked, parent);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, s->forked, 0);
    if (e != cudaSuccess) return e;
    stream = s->stream;
    done = s->done;
    return cudaSuccess;
  }
  cudaError_t join(cudaStream_t parent) {
    if (!done) return cudaSuccess;
    cudaError_t e = cudaEventRecord(done, stream);
    return e == cudaSuccess ? cudaStreamWaitEvent(parent, done, 0) : e;
  }
};

void fill_options(const ssn_options* opt, DualArgs& a) {
  ssn_options d;
  ssn_default_options(&d);
  if (!opt) opt = &d;
  a.max_newton = opt->max_newton;
  a.max_cg = opt->max_cg;
  a.max_backtrack = opt->max_backtrack;
  a.feas_tol = opt->feas_tol;
  const bool split = opt->precision == SSN_PRECISION_SPLIT;
  a.adaptive_precond = opt->preconditioner == SSN_PRECOND_ADAPTIVE ? 1 : 0;
  a.approx_basis = (split || a.adaptive_precond) ? 1 : 0;    // full rotated Gram
  // refine V to FP64 orthogonality with the full Gram: needed for FP32 rotations, and worth
  // its four m x m products for FP64 ones too, whose ~1e-14 residue ill-conditioned targets
  // (an inverse of norm ~1e2 in P + iQ) amplify into the primal's stationarity
  a.orthogonalize = a.approx_basis;
  // split form: the early Newton steps in FP32 unless the caller keeps them FP64
  a.fp32_newton = (split && opt->fp32_newton >= 0) ? 1 : 0;
}

bool split_form(const ssn_options* opt) { return opt && opt->precision == SSN_PRECISION_SPLIT; }
int eig_sweeps(const ssn_options* opt) { return opt && opt->eig_sweeps > 0 ? opt->eig_sweeps : kDefaultEigSweeps; }

bool options_ok(const ssn_options* opt) {
  if (!opt) return true;
  return opt->max_newton >= 1 && opt->max_newton <= 100000 && opt->max_cg >= 1 &&
         opt->max_cg <= 100000 && opt->max_backtrack >= 1 && opt->max_backtrack <= 1074 &&
         opt->feas_tol > 0.0 &&
         (opt->precision == SSN_PRECISION_FP64 || opt->precision == SSN_PRECISION_SPLIT) &&
         opt->eig_sweeps >= 0 && opt->eig_sweeps <= 24 && opt->fp32_newton >= -1 && opt->fp32_newton <= 1 &&
         (opt->preconditioner == SSN_PRECOND_EIGENBASIS || opt->preconditioner == SSN_PRECOND_ADAPTIVE);
}

// Eigenbasis of the scaled Gram for either precision form.
cudaError_t eigenbasis(const ssn_options* opt, const double* Cr, double* values, double* vectors, double* scale,
                       int32_t* sweeps, int32_t* status, int batch, int m, void* ws, cudaStream_t stream) {
  if (split_form(opt))
    return launch_eigh_approx(Cr, values, vectors, scale, sweeps, status, batch, m, ws, eig_sweeps(opt), true,
                              (opt && opt->eig_sweeps > 0) ? 0.0f : kRoughBasisSkip, stream);
  return launch_eigh(Cr, values, vectors, scale, sweeps, status, batch, m, ws, stream);
}

// The solve pipeline on one stream (the split form's side work on the side stream).
int solve_on(const double* T, double* X, double* omega, int64_t* iterations, int32_t* status, int batch, int n,
             int m, void* workspace, const ssn_options* opt, cudaStream_t stream, int concurrent) {
  const SolveLayout L = solve_layout(batch, n, m);
  // the problem class's autotuned launch parameters, for every launch below
  TuningScope tuning(find_tuning(split_form(opt) ? SSN_PRECISION_SPLIT : SSN_PRECISION_FP64, n, m, batch));
  char* ws = static_cast<char*>(workspace);
  double* Cr = reinterpret_cast<double*>(ws + L.cr);
  double* Ci = reinterpret_cast<double*>(ws + L.ci);
  double* values = reinterpret_cast<double*>(ws + L.values);
  double* vectors = reinterpret_cast<double*>(ws + L.vectors);
  double* scale = reinterpret_cast<double*>(ws + L.scale);
  double* Pf = reinterpret_cast<double*>(ws + L.pfin);
  double* Qf = reinterpret_cast<double*>(ws + L.qfin);
  double* work = reinterpret_cast<double*>(ws + L.work);
  int32_t* eig_status = reinterpret_cast<int32_t*>(ws + L.eig_status);

  const int64_t stride = 2LL * n * m;
  const double* A = T;
  const double* D = T + (size_t)n * m;
  int* stall = reinterpret_cast<int*>(ws + L.stall);
  const bool split = split_form(opt);
  cudaError_t e = split ? launch_gram_ozaki(A, D, stride, Cr, Ci, batch, n, m, work, nullptr, stall, stream)
                        : launch_gram(A, D, stride, Cr, Ci, batch, n, m, work, stream);
  if (e != cudaSuccess) return SSN_ERR_CUDA;
  SideStream side;
  if (split && side.open() != cudaSuccess) return SSN_ERR_CUDA;
  int32_t* sweeps = reinterpret_cast<int32_t*>(ws + L.sweeps);
  e = eigenbasis(opt, Cr, values, vectors, scale, sweeps, eig_status, batch, m, ws + L.eig_ws, stream);
  if (e != cudaSuccess) return SSN_ERR_CUDA;
  DualArgs a{};
  a.m = m;
  fill_options(opt, a);
  a.Cr = Cr;
  a.Ci = Ci;
  a.values = values;
  a.vectors = vectors;
  a.scale = scale;
  a.eig_status = eig_status;
  a.sweeps = sweeps;
  a.work = work;
  a.omega = omega;
  a.P = Pf;
  a.Q = Qf;
  a.iterations = iterations;
  a.status = status;
  a.counters = nullptr;
  a.concurrent = concurrent;
  e = launch_dual(a, batch, stream, split ? side.forked : nullptr);
  if (e != cudaSuccess) return SSN_ERR_CUDA;
  if (split) {
    // the digits of [A | D] for the recovery do not depend on the dual solution: made on
    // the side stream from the start of the Newton steps (side.forked), beside them
    e = side.wait_forked();
    if (e == cudaSuccess) e = launch_recover_wdigits(A, D, stride, batch, n, m, ws + L.rec, side.stream);
    if (e == cudaSuccess) e = side.record();
    if (e == cudaSuccess) e = side.join(stream);
    if (e == cudaSuccess)
      e = launch_recover_products(Pf, Qf, X, X + (size_t)n * m, stride, batch, n, m, ws + L.rec, stream);
  } else {
    e = launch_recover(A, D, stride, Pf, Qf, X, X + (size_t)n * m, stride, batch, n, m, stream);
  }
  return cuda_status(e);
}

}  // namespace

namespace ssn {

size_t solve_workspace_bytes(int batch, int n, int m) { return solve_layout(batch, n, m).total; }
bool solve_options_ok(const ssn_options* opt) { return options_ok(opt); }

// Arguments checked by the caller (ssn_solve, ssn_solve_ragged).  The split form runs
// on a higher-priority stream than its side work (MainStream), joined back into `stream`
// also after an error, so nothing enqueued here outlives the caller's view of it.
int solve_batch(const double* T, double* X, double* omega, int64_t* iterations, int32_t* status, int batch,
                int n, int m, void* workspace, const ssn_options* opt, cudaStream_t stream, int concurrent) {
  if (!split_form(opt)) return solve_on(T, X, omega, iterations, status, batch, n, m, workspace, opt, stream, concurrent);
  MainStream main;
  if (main.fork(stream) != cudaSuccess) return SSN_ERR_CUDA;
  const int rc = solve_on(T, X, omega, iterations, status, batch, n, m, workspace, opt, main.stream, concurrent);
  const cudaError_t e = main.join(stream);
  return rc != SSN_OK ? rc : cuda_status(e);
}

}  // namespace ssn

extern "C" {

int ssn_version(void) { return kVersion; }

const char* ssn_status_string(int status) {
  switch (status) {
    case SSN_OK: return "ok";
    case SSN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SSN_ERR_CUDA: return "CUDA error";
    case SSN_ERR_NEWTON_CAP: return "batched Newton iteration cap reached";
    case SSN_ERR_LINE_SEARCH: return "batched line search found no descent step";
    case SSN_ERR_NONFINITE: return "non-finite value in the iteration";
    case SSN_ERR_EIGH: return "Jacobi eigensolver did not converge";
    case SSN_ERR_WORKSPACE: return "workspace missing or too small";
    case SSN_ERR_SCRATCH_LIMIT: return "problem exceeds the fixed scratch of the no-allocation entry point";
    default: return "unknown status";
  }
}

void ssn_default_options(ssn_options* opt) {
  if (!opt) return;
  memset(opt, 0, sizeof(*opt));
  opt->max_newton = 100;
  opt->max_cg = 150;
  opt->max_backtrack = 40;
  opt->feas_tol = 1e-8;
}

size_t ssn_workspace_bytes(int batch, int n, int m) {
  if (!shape_ok(batch, m) || n < m / 2) return 0;
  return solve_layout(batch, n, m).total;
}

int ssn_solve(const double* T, double* X, double* omega, int64_t* iterations, int32_t* status,
              int batch, int n, int m, void* workspace, size_t workspace_bytes,
              const ssn_options* opt, ssn_stream_t stream_) {
  if (!shape_ok(batch, m) || n < m / 2 || !T || !X || !omega || !iterations || !status ||
      !options_ok(opt))
    return SSN_ERR_INVALID_ARGUMENT;
  if (!aligned16(T) || !aligned16(X) || !aligned16(omega)) return SSN_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < solve_layout(batch, n, m).total || !aligned16(workspace))
    return SSN_ERR_WORKSPACE;
  return solve_batch(T, X, omega, iterations, status, batch, n, m, workspace, opt,
                     reinterpret_cast<cudaStream_t>(stream_), 0);
}

size_t gram_fp64_bytes(int batch, int rows, int m) { return sizeof(double) * gram_partial_doubles(batch, rows, m); }

size_t ssn_gram_workspace_bytes(int batch, int rows, int m) {
  if (!shape_ok(batch, m) || rows < 1) return 0;
  const size_t f = gram_fp64_bytes(batch, rows, m);
  const size_t z = align_up(ozaki_gram_workspace_bytes(batch, rows, m), 256) + 256;   // + stall flag
  return f > z ? f : z;
}

int ssn_gram(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci, int batch,
             int rows, int m, void* workspace, size_t workspace_bytes, const ssn_options* opt,
             ssn_stream_t stream) {
  if (!shape_ok(batch, m) || rows < 1 || !A || !D || !Cr || !Ci || ab_stride < (int64_t)rows * m ||
      (ab_stride % 2) != 0 || !aligned16(A) || !aligned16(D) || !options_ok(opt))
    return SSN_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < ssn_gram_workspace_bytes(batch, rows, m) || !aligned16(workspace))
    return SSN_ERR_WORKSPACE;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (split_form(opt)) {
    int* stall = reinterpret_cast<int*>(static_cast<char*>(workspace) +
                                        align_up(ozaki_gram_workspace_bytes(batch, rows, m), 256));
    return cuda_status(launch_gram_ozaki(A, D, ab_stride, Cr, Ci, batch, rows, m, workspace, nullptr, stall, st));
  }
  return cuda_status(launch_gram(A, D, ab_stride, Cr, Ci, batch, rows, m, static_cast<double*>(workspace), st));
}

size_t ssn_cross_gram_workspace_bytes(int batch, int rows, int m) {
  if (!shape_ok(batch, m) || rows < 1) return 0;
  return gram_fp64_bytes(batch, rows, m);
}

int ssn_cross_gram(const double* Ga, const double* Gd, int64_t g_stride, const double* A, const double* D,
                   int64_t ab_stride, double* Mr, double* Mi, int batch, int rows, int m, void* workspace,
                   size_t workspace_bytes, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || rows < 1 || !Ga || !Gd || !A || !D || !Mr || !Mi ||
      g_stride < (int64_t)rows * m || ab_stride < (int64_t)rows * m || (g_stride % 2) != 0 ||
      (ab_stride % 2) != 0 || !aligned16(Ga) || !aligned16(Gd) || !aligned16(A) || !aligned16(D))
    return SSN_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < ssn_cross_gram_workspace_bytes(batch, rows, m) || !aligned16(workspace))
    return SSN_ERR_WORKSPACE;
  return cuda_status(launch_cross_gram(Ga, Gd, g_stride, A, D, ab_stride, Mr, Mi, batch, rows, m,
                                       static_cast<double*>(workspace), reinterpret_cast<cudaStream_t>(stream)));
}

size_t ssn_recover_workspace_bytes(int batch, int rows, int m) {
  if (!shape_ok(batch, m) || rows < 1) return 0;
  return ozaki_recover_workspace_bytes(batch, rows, m);
}

int ssn_recover(const double* A, const double* D, int64_t ab_stride, const double* P, const double* Q,
                double* Ur, double* Ui, int64_t u_stride, int batch, int rows, int m, void* workspace,
                size_t workspace_bytes, const ssn_options* opt, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || rows < 1 || !A || !D || !P || !Q || !Ur || !Ui ||
      ab_stride < (int64_t)rows * m || u_stride < (int64_t)rows * m || (ab_stride % 2) != 0 ||
      (u_stride % 2) != 0 || !aligned16(A) || !aligned16(D) || !aligned16(P) || !aligned16(Q) ||
      !options_ok(opt))
    return SSN_ERR_INVALID_ARGUMENT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (split_form(opt)) {
    if (!aligned16(Ur) || !aligned16(Ui)) return SSN_ERR_INVALID_ARGUMENT;   // 16-byte row-segment stores
    if (!workspace || workspace_bytes < ozaki_recover_workspace_bytes(batch, rows, m) || !aligned16(workspace))
      return SSN_ERR_WORKSPACE;
    return cuda_status(launch_recover_ozaki(A, D, ab_stride, P, Q, Ur, Ui, u_stride, batch, rows, m,
                                            workspace, st));
  }
  return cuda_status(launch_recover(A, D, ab_stride, P, Q, Ur, Ui, u_stride, batch, rows, m, st));
}

size_t ssn_eigh_workspace_bytes(int batch, int m) {
  if (!shape_ok(batch, m)) return 0;
  return eigh_workspace_bytes(batch, m);
}

int ssn_eigh(const double* Cr, double* values, double* vectors, double* scale, int32_t* sweeps,
             int batch, int m, void* workspace, size_t workspace_bytes, const ssn_options* opt,
             ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !Cr || !values || !vectors || !options_ok(opt)) return SSN_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < eigh_workspace_bytes(batch, m) || !aligned16(workspace))
    return SSN_ERR_WORKSPACE;
  return cuda_status(eigenbasis(opt, Cr, values, vectors, scale, sweeps, nullptr, batch, m, workspace,
                                reinterpret_cast<cudaStream_t>(stream)));
}

size_t ssn_dual_workspace_bytes(int batch, int m) {
  if (!shape_ok(batch, m)) return 0;
  return dual_layout(batch, m).total;
}

int ssn_dual(const double* Cr, const double* Ci, double* omega, double* P, double* Q,
             int64_t* iterations, int32_t* status, int batch, int m, void* workspace,
             size_t workspace_bytes, const ssn_options* opt, ssn_stream_t stream_) {
  if (!shape_ok(batch, m) || !Cr || !Ci || !omega || !P || !Q || !iterations || !status ||
      !options_ok(opt) || !aligned16(Cr) || !aligned16(Ci))
    return SSN_ERR_INVALID_ARGUMENT;
  const DualLayout L = dual_layout(batch, m);
  if (!workspace || workspace_bytes < L.total || !aligned16(workspace)) return SSN_ERR_WORKSPACE;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  char* ws = static_cast<char*>(workspace);
  double* values = reinterpret_cast<double*>(ws + L.values);
  double* vectors = reinterpret_cast<double*>(ws + L.vectors);
  double* scale = reinterpret_cast<double*>(ws + L.scale);
  int32_t* eig_status = reinterpret_cast<int32_t*>(ws + L.eig_status);
  cudaError_t e = eigenbasis(opt, Cr, values, vectors, scale, nullptr, eig_status, batch, m,
                             ws + L.eig_ws, stream);
  if (e != cudaSuccess) return SSN_ERR_CUDA;
  DualArgs a{};
  a.m = m;
  fill_options(opt, a);
  a.Cr = Cr;
  a.Ci = Ci;
  a.values = values;
  a.vectors = vectors;
  a.scale = scale;
  a.eig_status = eig_status;
  a.work = reinterpret_cast<double*>(ws + L.work);
  a.omega = omega;
  a.P = P;
  a.Q = Q;
  a.iterations = iterations;
  a.status = status;
  a.counters = nullptr;
  return cuda_status(launch_dual(a, batch, stream));
}

size_t ssn_newton_workspace_bytes(int batch, int m) {
  if (!shape_ok(batch, m)) return 0;
  return sizeof(double) * (size_t)batch * kDualMats * m * m;
}

int ssn_newton(const double* Cr, const double* Ci, const double* values, const double* vectors,
               const double* scale, const int32_t* eig_status, double* omega, double* P, double* Q,
               int64_t* iterations, int32_t* status, int32_t* counters, int batch, int m, void* workspace,
               size_t workspace_bytes, const ssn_options* opt, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !Ci || !values || !vectors || !scale || !omega || !P || !Q ||
      !iterations || !status || !options_ok(opt) || !aligned16(Ci) || !aligned16(vectors))
    return SSN_ERR_INVALID_ARGUMENT;
  DualArgs chk{};
  chk.m = m;
  fill_options(opt, chk);
  if (chk.approx_basis && (!Cr || !aligned16(Cr))) return SSN_ERR_INVALID_ARGUMENT;   // full rotated Gram needs Cr
  if (!workspace || workspace_bytes < ssn_newton_workspace_bytes(batch, m) || !aligned16(workspace))
    return SSN_ERR_WORKSPACE;
  DualArgs a{};
  a.m = m;
  fill_options(opt, a);
  a.Cr = Cr;
  a.Ci = Ci;
  a.values = values;
  a.vectors = vectors;
  a.scale = scale;
  a.eig_status = eig_status;
  a.work = static_cast<double*>(workspace);
  a.omega = omega;
  a.P = P;
  a.Q = Q;
  a.iterations = iterations;
  a.status = status;
  a.counters = counters;
  return cuda_status(launch_dual(a, batch, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_set_newton_events(void* const* events) {
  set_newton_events(events);
  return SSN_OK;
}

int ssn_probe_fp64_mma(double* sink, int iters, double* flops, ssn_stream_t stream) {
  if (!sink || !flops || iters < 1 || iters > (1 << 24)) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_probe_fp64_mma(sink, iters, flops, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_probe_s8_mma(const int8_t* A, const int8_t* B, int32_t* C, int n, int k, int* stall,
                     ssn_stream_t stream) {
  if (!A || !B || !C || !stall || !aligned16(A) || !aligned16(B)) return SSN_ERR_INVALID_ARGUMENT;
  if (n < 16 || n > 256 || n % 16 != 0 || k < 32 || k > 256 || k % 32 != 0) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_probe_s8_mma(A, B, C, n, k, stall, reinterpret_cast<cudaStream_t>(stream)));
}

#define SSN_CHECK_MATS(...)                                                   \
  do {                                                                        \
    const void* ps_[] = {__VA_ARGS__};                                        \
    for (const void* p_ : ps_)                                                \
      if (!p_ || !aligned16(p_)) return SSN_ERR_INVALID_ARGUMENT;             \
  } while (0)

int ssn_inner_products(const double* E, const double* Sr, const double* Si, double* U, double* V,
                       int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m)) return SSN_ERR_INVALID_ARGUMENT;
  SSN_CHECK_MATS(E, Sr, Si, U, V);
  return cuda_status(launch_inner_products(E, Sr, Si, U, V, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_outer_skew(const double* P, const double* Q, const double* U, const double* V, double* H,
                   int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m)) return SSN_ERR_INVALID_ARGUMENT;
  SSN_CHECK_MATS(P, Q, U, V, H);
  return cuda_status(launch_outer_skew(P, Q, U, V, H, batch, m, nullptr, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_sandwich_front(const double* values, const double* Ci, const double* P, const double* Q,
                       double* Yr, double* Yi, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !values) return SSN_ERR_INVALID_ARGUMENT;
  SSN_CHECK_MATS(Ci, P, Q, Yr, Yi);
  return cuda_status(launch_sandwich_front(values, Ci, P, Q, Yr, Yi, batch, m,
                                           reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_line_change(const double* gradient, const double* delta, const double* V,
                    const double* delta_Sr, const double* trial, const double* delta_Si,
                    double* change, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !change) return SSN_ERR_INVALID_ARGUMENT;
  SSN_CHECK_MATS(gradient, delta, V, delta_Sr, trial, delta_Si);
  return cuda_status(launch_line_change(gradient, delta, V, delta_Sr, trial, delta_Si, change, batch, m,
                                        reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_precondition(const double* R, const double* denominator, double* out, int batch, int m,
                     ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !R || !denominator || !out) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_precondition(R, denominator, out, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_cg_update(const double* direction, const double* r, const double* p, const double* Hp,
                  const double* alpha, double* new_direction, double* new_r, int batch, int m,
                  ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !direction || !r || !p || !Hp || !alpha || !new_direction || !new_r)
    return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_cg_update(direction, r, p, Hp, alpha, new_direction, new_r, batch, m,
                                      reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_cg_next(const double* z, const double* p, const double* beta, const uint8_t* active,
                double* out, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !z || !p || !beta || !active || !out) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_cg_next(z, p, beta, active, out, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_inverse_from_cholesky(const double* L, double* P, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !L || !P) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_inverse_from_cholesky(L, P, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_spd_inverse(const double* K, double* P, int32_t* info, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !K || !P || !info) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_spd_inverse(K, P, info, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

int ssn_cholesky_k(const double* omega, double* L, int32_t* info, int batch, int m, ssn_stream_t stream) {
  if (!shape_ok(batch, m) || !omega || !L || !info) return SSN_ERR_INVALID_ARGUMENT;
  return cuda_status(launch_cholesky_k(omega, L, info, batch, m, reinterpret_cast<cudaStream_t>(stream)));
}

}  // extern "C"
