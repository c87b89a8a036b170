// ssn_components.cu -- stand-alone batched kernels for the individual
// operations of the Newton-CG, one per reference kernel wrapper
// (src/symplectic_projection/hvp_fused.py, cholesky_inverse_kernel.py).  The
// persistent solver fuses the same arithmetic; these entry points exist so
// each operation can be used and parity-checked on its own.
#include <math.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

namespace {
constexpr uint32_t kOne = coef_bit(0, 0, 0, 1);
constexpr uint32_t kSharedA = coef_bit(0, 0, 0, 1) | coef_bit(1, 0, 1, 1);
constexpr uint32_t kSharedB = coef_bit(0, 0, 0, 1) | coef_bit(1, 1, 0, 1);
constexpr uint32_t kDiff = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 2);

size_t engine_smem(int m) { return sizeof(double) * (8 * (size_t)slot_doubles(bucket_of(m)) + 2 * kWarps); }

template <class K>
cudaError_t prep(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
}
}  // namespace

// U = E Sr, V = E Si (hvp_inner, hvp_fused.cu:2-38)
template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    inner_products_kernel(const double* E, const double* Sr, const double* Si, double* U, double* V, int m) {
  extern __shared__ __align__(16) double smem[];
  const size_t off = (size_t)blockIdx.x * m * m;
  using TL = Tile<MB, 2>;
  MatOp A[1] = {op_n(E + off, m)};
  MatOp B[2] = {op_n(Sr + off, m), op_n(Si + off, m)};
  auto epi = [&](int o, int i, int j, double v) { (o == 0 ? U : V)[off + i * m + j] = v; };
  tile_product<TL::WR, TL::WC, 1, 2, 2, kSharedA>(A, B, m, m, m, smem, slot_doubles(MB), epi);
}

// H = Z - Z^T, Z = P U - Q V (hvp_outer*, hvp_fused.cu:83-238); Z kept in shared memory.
template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    outer_skew_kernel(const double* P, const double* Q, const double* U, const double* V, double* H, int m) {
  extern __shared__ __align__(16) double smem[];
  const size_t off = (size_t)blockIdx.x * m * m;
  using TL = Tile<MB, 1>;
  const int ld = m + 1;
  double* Z = smem;  // reused after the product's last barrier
  MatOp A[2] = {op_n(P + off, m), op_n(Q + off, m)};
  MatOp B[2] = {op_n(U + off, m), op_n(V + off, m)};
  auto epi = [&](int, int i, int j, double v) { Z[i * ld + j] = v; };
  tile_product<TL::WR, TL::WC, 2, 2, 1, kDiff>(A, B, m, m, m, smem, slot_doubles(MB), epi);
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    H[off + e] = Z[i * ld + j] - Z[j * ld + i];
  }
}

// Yr = P diag(values) - Q Ci, Yi = P Ci + Q diag(values) (hvp_sandwich_front, hvp_fused.cu:41-80)
template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    sandwich_front_kernel(const double* values, const double* Ci, const double* P, const double* Q,
                          double* Yr, double* Yi, int m) {
  extern __shared__ __align__(16) double smem[];
  const size_t off = (size_t)blockIdx.x * m * m;
  const double* lam = values + (size_t)blockIdx.x * m;
  using TL = Tile<MB, 2>;
  MatOp A[2] = {op_n(Q + off, m), op_n(P + off, m)};
  MatOp B[1] = {op_n(Ci + off, m)};
  auto epi = [&](int o, int i, int j, double v) {
    const size_t e = off + i * m + j;
    if (o == 0) Yr[e] = __dsub_rn(__dmul_rn(P[e], lam[j]), v);
    else Yi[e] = __dadd_rn(v, __dmul_rn(Q[e], lam[j]));
  };
  tile_product<TL::WR, TL::WC, 2, 1, 2, kSharedB>(A, B, m, m, m, smem, slot_doubles(MB), epi);
}

// change = <g, delta> + <V, dSr + trial dSi> (hvp_line_partial/finish, hvp_fused.cu:259-371)
template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    line_change_kernel(const double* g, const double* delta, const double* V, const double* dSr,
                       const double* trial, const double* dSi, double* change, int m) {
  extern __shared__ __align__(16) double smem[];
  const size_t off = (size_t)blockIdx.x * m * m;
  double* red = smem + 8 * slot_doubles(MB);
  using TL = Tile<MB, 1>;
  double tail = 0.0;
  MatOp A[1] = {op_n(trial + off, m)};
  MatOp B[1] = {op_n(dSi + off, m)};
  auto epi = [&](int, int i, int j, double v) {
    const size_t e = off + i * m + j;
    tail += __dmul_rn(V[e], __dadd_rn(dSr[e], v));
  };
  tile_product<TL::WR, TL::WC, 1, 1, 1, kOne>(A, B, m, m, m, smem, slot_doubles(MB), epi);
  double first = 0.0;
  for (int e = threadIdx.x; e < m * m; e += kThreads) first += __dmul_rn(g[off + e], delta[off + e]);
  block_sum2(first, tail, red);
  if (threadIdx.x == 0) change[blockIdx.x] = __dadd_rn(first, tail);
}

// elementwise PCG helpers (hvp_fused.cu:374-420)
__global__ void precondition_kernel(const double* R, const double* den, double* out, int m) {
  const size_t mm = (size_t)m * m, off = (size_t)blockIdx.y * mm;
  for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < mm; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / m, j = e - i * m, et = j * m + i;
    const double a = __ddiv_rn(R[off + e], den[off + e]);
    const double b = __ddiv_rn(R[off + et], den[off + et]);
    out[off + e] = __dmul_rn(__dsub_rn(a, b), 0.5);
  }
}

__global__ void cg_update_kernel(const double* d, const double* r, const double* p, const double* Hp,
                                 const double* alpha, double* nd, double* nr, int m) {
  const size_t mm = (size_t)m * m, off = (size_t)blockIdx.y * mm;
  const double a = alpha[blockIdx.y];
  for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < mm; e += (size_t)gridDim.x * blockDim.x) {
    nd[off + e] = __dadd_rn(d[off + e], __dmul_rn(a, p[off + e]));
    nr[off + e] = __dsub_rn(r[off + e], __dmul_rn(a, Hp[off + e]));
  }
}

__global__ void cg_next_kernel(const double* z, const double* p, const double* beta, const uint8_t* active,
                               double* out, int m) {
  const size_t mm = (size_t)m * m, off = (size_t)blockIdx.y * mm;
  const double bt = beta[blockIdx.y];
  const bool on = active[blockIdx.y] != 0;
  for (size_t e = blockIdx.x * blockDim.x + threadIdx.x; e < mm; e += (size_t)gridDim.x * blockDim.x) {
    const double nxt = __dadd_rn(z[off + e], __dmul_rn(bt, p[off + e]));
    out[off + e] = on ? nxt : 0.0;
  }
}

// P = (L L^T)^-1: in-place lower triangular inverse R = L^-1 (column sweep from
// the last column, each column one triangular matrix-vector product with the
// already inverted trailing block), then P = R^T R.
__global__ void __launch_bounds__(kThreads, 1)
    inverse_from_cholesky_kernel(const double* L, double* P, int m) {
  extern __shared__ __align__(16) double smem[];
  const int ld = m + 1;
  double* R = smem;
  double* x = smem + m * ld;
  const size_t off = (size_t)blockIdx.x * m * m;
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    R[i * ld + j] = (j <= i) ? L[off + e] : 0.0;
  }
  __syncthreads();
  for (int j = m - 1; j >= 0; --j) {
    const double rjj = 1.0 / R[j * ld + j];
    for (int i = j + 1 + threadIdx.x; i < m; i += kThreads) x[i] = R[i * ld + j];
    __syncthreads();
    // R[i][j] = -rjj * sum_{k=j+1..i} Rinv[i][k] * L[k][j]
    for (int i = j + 1 + threadIdx.x; i < m; i += kThreads) {
      double s = 0.0;
      for (int k = j + 1; k <= i; ++k) s += R[i * ld + k] * x[k];
      R[i * ld + j] = -rjj * s;
    }
    __syncthreads();
    if (threadIdx.x == 0) R[j * ld + j] = rjj;
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    const int k0 = i > j ? i : j;
    double s = 0.0;
    for (int k = k0; k < m; ++k) s += R[k * ld + i] * R[k * ld + j];
    P[off + e] = s;
  }
}

// L = chol(I + omega omega) for a skew omega (dual_recommended_hvp.py:63 and :173,
// torch.linalg.cholesky(I + omega @ omega)).  One CTA per instance: the lower
// triangle of K = I + omega omega is formed from omega staged in shared memory
// (through L's own storage, so one m x m array of shared memory suffices), then
// factored column by column (right-looking).  info = 0, or the order of the
// first leading minor that is not positive definite (L's columns from there
// are 0).
__global__ void __launch_bounds__(kThreads, 1)
    cholesky_k_kernel(const double* omega, double* L, int32_t* info, int m) {
  extern __shared__ __align__(16) double smem[];
  const int ld = m + 1;
  double* K = smem;
  __shared__ int bad;
  const size_t off = (size_t)blockIdx.x * m * m;
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    K[i * ld + j] = omega[off + e];
  }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    if (j > i) continue;
    double s = (i == j) ? 1.0 : 0.0;
    for (int k = 0; k < m; ++k) s = fma(K[i * ld + k], K[k * ld + j], s);
    L[off + e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    if (j <= i) K[i * ld + j] = L[off + e];
  }
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    const double d = K[j * ld + j];
    if (!(d > 0.0) || !isfinite(d)) {
      if (threadIdx.x == 0) bad = j + 1;
      break;
    }
    const double r = sqrt(d);
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < m; i += kThreads) K[i * ld + j] /= r;
    if (threadIdx.x == 0) K[j * ld + j] = r;
    __syncthreads();
    // trailing update of the lower triangle: K[i][l] -= L[i][j] L[l][j], j < l <= i
    const int t = m - j - 1;
    for (int e = threadIdx.x; e < t * t; e += kThreads) {
      const int i = j + 1 + e / t, l = j + 1 + e % t;
      if (l <= i) K[i * ld + l] = fma(-K[i * ld + j], K[l * ld + j], K[i * ld + l]);
    }
    __syncthreads();
  }
  __syncthreads();
  const int fail = bad;
  for (int e = threadIdx.x; e < m * m; e += kThreads) {
    const int i = e / m, j = e - i * m;
    L[off + e] = (j <= i && (fail == 0 || j < fail - 1)) ? K[i * ld + j] : 0.0;
  }
  if (threadIdx.x == 0) info[blockIdx.x] = fail;
}

#define SSN_MB_DISPATCH(KERNEL, SMEM, ...)                                              \
  do {                                                                                  \
    cudaError_t e_ = cudaSuccess;                                                       \
    switch (bucket_of(m)) {                                                             \
      case 1: e_ = prep(KERNEL<1>, SMEM); if (e_ == cudaSuccess) KERNEL<1><<<batch, kThreads, SMEM, stream>>>(__VA_ARGS__); break; \
      case 2: e_ = prep(KERNEL<2>, SMEM); if (e_ == cudaSuccess) KERNEL<2><<<batch, kThreads, SMEM, stream>>>(__VA_ARGS__); break; \
      case 3: e_ = prep(KERNEL<3>, SMEM); if (e_ == cudaSuccess) KERNEL<3><<<batch, kThreads, SMEM, stream>>>(__VA_ARGS__); break; \
      default: e_ = prep(KERNEL<4>, SMEM); if (e_ == cudaSuccess) KERNEL<4><<<batch, kThreads, SMEM, stream>>>(__VA_ARGS__); break; \
    }                                                                                   \
    if (e_ != cudaSuccess) return e_;                                                   \
  } while (0)

cudaError_t launch_inner_products(const double* E, const double* Sr, const double* Si, double* U,
                                  double* V, int batch, int m, cudaStream_t stream) {
  SSN_MB_DISPATCH(inner_products_kernel, engine_smem(m), E, Sr, Si, U, V, m);
  return cudaGetLastError();
}

cudaError_t launch_outer_skew(const double* P, const double* Q, const double* U, const double* V,
                              double* H, int batch, int m, double*, cudaStream_t stream) {
  SSN_MB_DISPATCH(outer_skew_kernel, engine_smem(m), P, Q, U, V, H, m);
  return cudaGetLastError();
}

cudaError_t launch_sandwich_front(const double* values, const double* Ci, const double* P,
                                  const double* Q, double* Yr, double* Yi, int batch, int m,
                                  cudaStream_t stream) {
  SSN_MB_DISPATCH(sandwich_front_kernel, engine_smem(m), values, Ci, P, Q, Yr, Yi, m);
  return cudaGetLastError();
}

cudaError_t launch_line_change(const double* g, const double* delta, const double* V,
                               const double* dSr, const double* trial, const double* dSi,
                               double* change, int batch, int m, cudaStream_t stream) {
  SSN_MB_DISPATCH(line_change_kernel, engine_smem(m), g, delta, V, dSr, trial, dSi, change, m);
  return cudaGetLastError();
}

static dim3 ew_grid(int batch, int m) { return dim3((unsigned)cdiv(m * m, 256), (unsigned)batch); }

cudaError_t launch_precondition(const double* R, const double* den, double* out, int batch, int m,
                                cudaStream_t stream) {
  precondition_kernel<<<ew_grid(batch, m), 256, 0, stream>>>(R, den, out, m);
  return cudaGetLastError();
}

cudaError_t launch_cg_update(const double* d, const double* r, const double* p, const double* Hp,
                             const double* alpha, double* nd, double* nr, int batch, int m,
                             cudaStream_t stream) {
  cg_update_kernel<<<ew_grid(batch, m), 256, 0, stream>>>(d, r, p, Hp, alpha, nd, nr, m);
  return cudaGetLastError();
}

cudaError_t launch_cg_next(const double* z, const double* p, const double* beta,
                           const uint8_t* active, double* out, int batch, int m,
                           cudaStream_t stream) {
  cg_next_kernel<<<ew_grid(batch, m), 256, 0, stream>>>(z, p, beta, active, out, m);
  return cudaGetLastError();
}

cudaError_t launch_inverse_from_cholesky(const double* L, double* P, int batch, int m,
                                         cudaStream_t stream) {
  const size_t smem = sizeof(double) * ((size_t)m * (m + 1) + m);
  cudaError_t err = prep(inverse_from_cholesky_kernel, smem);
  if (err != cudaSuccess) return err;
  inverse_from_cholesky_kernel<<<batch, kThreads, smem, stream>>>(L, P, m);
  return cudaGetLastError();
}

cudaError_t launch_cholesky_k(const double* omega, double* L, int32_t* info, int batch, int m,
                              cudaStream_t stream) {
  const size_t smem = sizeof(double) * (size_t)m * (m + 1);
  cudaError_t err = prep(cholesky_k_kernel, smem);
  if (err != cudaSuccess) return err;
  cholesky_k_kernel<<<batch, kThreads, smem, stream>>>(omega, L, info, m);
  return cudaGetLastError();
}

}  // namespace ssn
