// ssn_adjoint.cu -- gradient of a loss through the solve: dL/dT from dL/dX and dL/d omega.
//
// The reference has no backward pass (its solver runs under torch.no_grad,
// dual_recommended_hvp.py:231).  This entry point differentiates the dual
// optimality condition Im(K C K) = J_m at the converged omega (implicit function
// theorem): one Hessian solve with the solver's own Hessian-vector product
// (hvp_fused.py:22-53) per instance, plus tall-skinny products around it.
// In complex form, b = A + iD, g = dL/dXa + i dL/dXd, K = (I + i omega)^-1:
//   M = g^H b                                   (cross Gram, 8 n m^2 flops)
//   Gamma = -skew(Im(K M K)) + skew(dL/d omega), H mu = Gamma   (adjoint kernel)
//   dL/db = g K + b N,  N = 2i K mu K           (two recovery products)
// and dL/dA = Re(dL/db), dL/dD = Im(dL/db).  X is not needed: the products
// with K recompute what the solve's recovery produced.
#include <cuda_runtime.h>

#include "ssn.h"
#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {
namespace {

size_t align_up_256(size_t v) { return (v + 255) / 256 * 256; }

struct AdjointLayout {
  size_t partial, cr, ci, mr, mi, p, q, pn, qn, work, tmp, oz, stall, total;
};

AdjointLayout adjoint_layout(int batch, int n, int m) {
  const size_t mm = (size_t)m * m;
  AdjointLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align_up_256(off + bytes);
    return at;
  };
  L.partial = take(sizeof(double) * gram_partial_doubles(batch, n, m));
  L.cr = take(sizeof(double) * batch * mm);
  L.ci = take(sizeof(double) * batch * mm);
  L.mr = take(sizeof(double) * batch * mm);
  L.mi = take(sizeof(double) * batch * mm);
  L.p = take(sizeof(double) * batch * mm);
  L.q = take(sizeof(double) * batch * mm);
  L.pn = take(sizeof(double) * batch * mm);
  L.qn = take(sizeof(double) * batch * mm);
  L.work = take(sizeof(double) * (size_t)batch * kAdjointMats * mm);
  L.tmp = take(sizeof(double) * (size_t)batch * 2 * n * m);
  // split form: the INT8 Ozaki Gram and recoveries (used one after the other)
  const size_t og = ozaki_gram_workspace_bytes(batch, n, m), orc = ozaki_recover_workspace_bytes(batch, n, m);
  L.oz = take(og > orc ? og : orc);
  L.stall = take(sizeof(int32_t) * 4);
  L.total = off;
  return L;
}

__global__ void add_into_kernel(double* __restrict__ dst, const double* __restrict__ src, int64_t n2) {
  double2* d = reinterpret_cast<double2*>(dst);
  const double2* s = reinterpret_cast<const double2*>(src);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.x * blockDim.x) {
    double2 a = d[e];
    const double2 b = s[e];
    a.x += b.x;
    a.y += b.y;
    d[e] = a;
  }
}

bool aligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace
}  // namespace ssn

using namespace ssn;

extern "C" {

size_t ssn_adjoint_workspace_bytes(int batch, int n, int m) {
  if (batch < 1 || m < 2 || m > kMaxM || (m % 2) != 0 || n < m / 2) return 0;
  return adjoint_layout(batch, n, m).total;
}

int ssn_adjoint(const double* T, const double* omega, const double* G, const double* Gw, double* dT,
                int32_t* status, int32_t* cg_iterations, int batch, int n, int m, void* workspace,
                size_t workspace_bytes, const ssn_options* opt, ssn_stream_t stream_) {
  if (batch < 1 || m < 2 || m > kMaxM || (m % 2) != 0 || n < m / 2 || !T || !omega || !dT || !status ||
      !solve_options_ok(opt))
    return SSN_ERR_INVALID_ARGUMENT;
  if (!aligned(T) || !aligned(omega) || !aligned(dT) || (G && !aligned(G)) || (Gw && !aligned(Gw)))
    return SSN_ERR_INVALID_ARGUMENT;
  const AdjointLayout L = adjoint_layout(batch, n, m);
  if (!workspace || workspace_bytes < L.total || !aligned(workspace)) return SSN_ERR_WORKSPACE;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  char* ws = static_cast<char*>(workspace);
  double* partial = reinterpret_cast<double*>(ws + L.partial);
  double* Cr = reinterpret_cast<double*>(ws + L.cr);
  double* Ci = reinterpret_cast<double*>(ws + L.ci);
  double* Mr = reinterpret_cast<double*>(ws + L.mr);
  double* Mi = reinterpret_cast<double*>(ws + L.mi);
  const int64_t stride = 2LL * n * m;
  const size_t mm = (size_t)m * m;

  // opt->precision == SSN_PRECISION_SPLIT: the Gram of T and the two recoveries run as INT8
  // Ozaki products on the tensor cores (the cross Gram stays FP64)
  const bool split = opt && opt->precision == SSN_PRECISION_SPLIT;
  void* oz = ws + L.oz;
  int* stall = reinterpret_cast<int*>(ws + L.stall);
  auto recover = [&](const double* A, const double* P, const double* Q, double* U) {
    return split ? launch_recover_ozaki(A, A + (size_t)n * m, stride, P, Q, U, U + (size_t)n * m, stride, batch, n,
                                        m, oz, stream)
                 : launch_recover(A, A + (size_t)n * m, stride, P, Q, U, U + (size_t)n * m, stride, batch, n, m,
                                  stream);
  };
  cudaError_t e = split ? launch_gram_ozaki(T, T + (size_t)n * m, stride, Cr, Ci, batch, n, m, oz, nullptr, stall,
                                            stream)
                        : launch_gram(T, T + (size_t)n * m, stride, Cr, Ci, batch, n, m, partial, stream);
  if (e == cudaSuccess) {
    if (G)
      e = launch_cross_gram(G, G + (size_t)n * m, stride, T, T + (size_t)n * m, stride, Mr, Mi, batch, n, m,
                            partial, stream);
    else {
      e = cudaMemsetAsync(Mr, 0, sizeof(double) * batch * mm, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(Mi, 0, sizeof(double) * batch * mm, stream);
    }
  }
  if (e != cudaSuccess) return SSN_ERR_CUDA;

  AdjointArgs a{};
  a.m = m;
  a.max_cg = opt ? (opt->max_cg > 10 * m ? opt->max_cg : 10 * m) : 10 * m;
  a.tol = 1e-12;
  a.Cr = Cr;
  a.Ci = Ci;
  a.Mr = Mr;
  a.Mi = Mi;
  a.omega = omega;
  a.Gw = Gw;
  a.work = reinterpret_cast<double*>(ws + L.work);
  a.P = reinterpret_cast<double*>(ws + L.p);
  a.Q = reinterpret_cast<double*>(ws + L.q);
  a.Pn = reinterpret_cast<double*>(ws + L.pn);
  a.Qn = reinterpret_cast<double*>(ws + L.qn);
  a.status = status;
  a.cg_iters = cg_iterations;
  e = launch_adjoint(a, batch, stream);
  if (e != cudaSuccess) return SSN_ERR_CUDA;

  if (G) {
    double* tmp = reinterpret_cast<double*>(ws + L.tmp);
    e = recover(G, a.P, a.Q, dT);
    if (e == cudaSuccess) e = recover(T, a.Pn, a.Qn, tmp);
    if (e == cudaSuccess) {
      const int64_t n2 = (int64_t)batch * stride / 2;
      add_into_kernel<<<4 * 148, 256, 0, stream>>>(dT, tmp, n2);
      e = cudaGetLastError();
    }
  } else {
    e = recover(T, a.Pn, a.Qn, dT);
  }
  return e == cudaSuccess ? SSN_OK : SSN_ERR_CUDA;
}

}  // extern "C"
