// ssn_gemm.cu -- tall-skinny FP64 products over the 2n rows of T.
//
// Gram (replaces gram_add_, gram_triangle_reflect.py:19-36 and the gram_*
// kernels, gram_triangle_reflect.cu): Cr = A^T A + D^T D, Ci = A^T D - D^T A.
// Grid = (row splits, batch).  Each CTA streams 16-row K-panels of its rows of
// A and D into shared memory once (cp.async, double-buffered) and feeds both
// the A^T/D^T fragments and the A/D fragments from the same panels.  Partial
// m x m sums per split are reduced in a fixed order by a finalize kernel, which
// also mirrors Cr (upper triangle) and forms Ci = G - G^T exactly antisymmetric.
//
// Recovery (replaces recover_block, recovery_fused.py:19-30, and recover_fused,
// recovery_fused.cu:2-41): Ur = A P^T + D Q^T, Ui = D P^T - A Q^T, one CTA per
// (row block, instance), the four products sharing fragments.
#include <atomic>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

constexpr uint32_t C_GRAM = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1) | coef_bit(1, 0, 1, 1);
constexpr uint32_t C_CR = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1);
constexpr uint32_t C_G = coef_bit(0, 0, 1, 1);
constexpr uint32_t C_REC = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1) | coef_bit(1, 1, 0, 1) |
                           coef_bit(1, 0, 1, 2);

int current_device_sm_count() {
  constexpr int kMaxDevices = 64;
  static std::atomic<int> cache[kMaxDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  int sms = cache[dev].load(std::memory_order_relaxed);
  if (sms <= 0) {
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    cache[dev].store(sms, std::memory_order_relaxed);
  }
  return sms;
}

static int device_sm_count() { return current_device_sm_count(); }

struct GramSplit {
  int splits, chunk;
};

static GramSplit gram_split(int batch, int rows, int max_splits = 1 << 30) {
  const int sms = device_sm_count();
  int want = imin(cdiv(2 * sms, batch), 16);
  const ssn_tuning* tune = active_tuning();
  if (tune && tune->gram_splits > 0) want = tune->gram_splits;   // autotuned
  want = imax(1, imin(imin(want, cdiv(rows, 64)), max_splits));
  int chunk = round_up(cdiv(rows, want), kPanelK);
  int splits = cdiv(rows, chunk);
  return GramSplit{splits, chunk};
}

size_t gram_partial_doubles(int batch, int rows, int m) {
  const GramSplit gs = gram_split(batch, rows);
  return (size_t)batch * gs.splits * 2 * m * m;
}

template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    gram_kernel(const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride,
                double* __restrict__ partial, int rows, int m, int chunk, int splits) {
  extern __shared__ __align__(16) double smem[];
  const int s = blockIdx.x, b = blockIdx.y;
  const int mm = m * m;
  const int r0 = s * chunk;
  const int K = imin(rows, r0 + chunk) - r0;
  double* out = partial + ((size_t)b * splits + s) * 2 * mm;
  const double* Ab = A + (size_t)b * ab_stride + (size_t)r0 * m;
  const double* Db = D + (size_t)b * ab_stride + (size_t)r0 * m;
  const int slot = slot_doubles(MB);
  auto epi = [&](int o, int i, int j, double v) { out[(size_t)o * mm + i * m + j] = v; };
  if constexpr (MB < 4) {
    using TL = Tile<MB, 2>;
    MatOp Aop[2] = {op_t(Ab, m), op_t(Db, m)};
    MatOp Bop[2] = {MatOp{Ab, m, 0, 0}, MatOp{Db, m, 0, 1}};
    tile_product<TL::WR, TL::WC, 2, 2, 2, C_GRAM>(Aop, Bop, m, m, K, smem, slot, epi);
  } else {
    using TL = Tile<MB, 1>;
    MatOp Aop[2] = {op_t(Ab, m), op_t(Db, m)};
    MatOp Bop[2] = {MatOp{Ab, m, 0, 0}, MatOp{Db, m, 0, 1}};
    auto epi_cr = [&](int, int i, int j, double v) { out[i * m + j] = v; };
    auto epi_g = [&](int, int i, int j, double v) { out[(size_t)mm + i * m + j] = v; };
    tile_product<TL::WR, TL::WC, 2, 2, 1, C_CR>(Aop, Bop, m, m, K, smem, slot, epi_cr);
    tile_product<TL::WR, TL::WC, 2, 2, 1, C_G>(Aop, Bop, m, m, K, smem, slot, epi_g);
  }
}

// One thread per upper-triangle entry (i <= j) of every instance: sums the
// row-split partials in split order, mirrors Cr and forms Ci = G - G^T.
__global__ void gram_finalize_kernel(const double* __restrict__ partial, double* __restrict__ Cr,
                                     double* __restrict__ Ci, int m, int splits) {
  const int b = blockIdx.y, mm = m * m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= mm) return;
  const int i = e / m, j = e - i * m;
  if (i > j) return;
  const double* p = partial + (size_t)b * splits * 2 * mm;
  double sr = 0.0, gij = 0.0, gji = 0.0;
  for (int s = 0; s < splits; ++s) {
    const double* q = p + (size_t)s * 2 * mm;
    sr += q[e];
    gij += q[mm + e];
    gji += q[mm + j * m + i];
  }
  double* cr = Cr + (size_t)b * mm;
  double* ci = Ci + (size_t)b * mm;
  cr[e] = sr;
  cr[j * m + i] = sr;
  const double c = gij - gji;
  ci[e] = c;
  ci[j * m + i] = -c;
}

int gram_splits(int batch, int rows, int max_splits) { return gram_split(batch, rows, max_splits).splits; }

cudaError_t launch_gram_finalize(const double* partial, double* Cr, double* Ci, int batch, int m, int splits,
                                 cudaStream_t stream) {
  gram_finalize_kernel<<<dim3(cdiv(m * m, 128), batch), 128, 0, stream>>>(partial, Cr, Ci, m, splits);
  return cudaGetLastError();
}

cudaError_t launch_gram(const double* A, const double* D, int64_t ab_stride, double* Cr, double* Ci,
                        int batch, int rows, int m, double* partial, cudaStream_t stream, int max_splits) {
  const GramSplit gs = gram_split(batch, rows, max_splits);
  const int MB = bucket_of(m);
  const size_t smem = sizeof(double) * 8 * (size_t)slot_doubles(MB);
  dim3 grid(gs.splits, batch);
  cudaError_t err = cudaSuccess;
#define SSN_GRAM_CASE(MBV)                                                                        \
  case MBV:                                                                                       \
    err = cudaFuncSetAttribute(gram_kernel<MBV>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                               static_cast<int>(smem));                                          \
    if (err != cudaSuccess) return err;                                                           \
    gram_kernel<MBV><<<grid, kThreads, smem, stream>>>(A, D, ab_stride, partial, rows, m,         \
                                                       gs.chunk, gs.splits);                     \
    break;
  switch (MB) {
    SSN_GRAM_CASE(1)
    SSN_GRAM_CASE(2)
    SSN_GRAM_CASE(3)
    SSN_GRAM_CASE(4)
  }
#undef SSN_GRAM_CASE
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  gram_finalize_kernel<<<dim3(cdiv(m * m, 128), batch), 128, 0, stream>>>(partial, Cr, Ci, m, gs.splits);
  return cudaGetLastError();
}

// Cross Gram of two tall-skinny pairs (the adjoint's g^H b): Mr = Ga^T A + Gd^T D,
// Mi = Ga^T D - Gd^T A, row-split like the Gram; partials [B][splits][2][m][m].
constexpr uint32_t C_XMR = coef_bit(0, 0, 0, 1) | coef_bit(0, 1, 1, 1);
constexpr uint32_t C_XMI = coef_bit(0, 0, 1, 1) | coef_bit(0, 1, 0, 2);

template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    cross_gram_kernel(const double* __restrict__ Ga, const double* __restrict__ Gd, int64_t g_stride,
                      const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride,
                      double* __restrict__ partial, int rows, int m, int chunk, int splits) {
  extern __shared__ __align__(16) double smem[];
  const int s = blockIdx.x, b = blockIdx.y;
  const int mm = m * m;
  const int r0 = s * chunk;
  const int K = imin(rows, r0 + chunk) - r0;
  double* out = partial + ((size_t)b * splits + s) * 2 * mm;
  using TL = Tile<MB, 1>;
  MatOp Aop[2] = {op_t(Ga + (size_t)b * g_stride + (size_t)r0 * m, m),
                  op_t(Gd + (size_t)b * g_stride + (size_t)r0 * m, m)};
  MatOp Bop[2] = {op_n(A + (size_t)b * ab_stride + (size_t)r0 * m, m),
                  op_n(D + (size_t)b * ab_stride + (size_t)r0 * m, m)};
  auto epi_r = [&](int, int i, int j, double v) { out[i * m + j] = v; };
  auto epi_i = [&](int, int i, int j, double v) { out[(size_t)mm + i * m + j] = v; };
  tile_product<TL::WR, TL::WC, 2, 2, 1, C_XMR>(Aop, Bop, m, m, K, smem, slot_doubles(MB), epi_r);
  tile_product<TL::WR, TL::WC, 2, 2, 1, C_XMI>(Aop, Bop, m, m, K, smem, slot_doubles(MB), epi_i);
}

// Fixed-order sum of the cross Gram's split partials.
__global__ void cross_gram_finalize_kernel(const double* __restrict__ partial, double* __restrict__ Mr,
                                           double* __restrict__ Mi, int m, int splits) {
  const int b = blockIdx.y, mm = m * m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= mm) return;
  const double* p = partial + (size_t)b * splits * 2 * mm;
  double sr = 0.0, si = 0.0;
  for (int s = 0; s < splits; ++s) {
    sr += p[(size_t)s * 2 * mm + e];
    si += p[(size_t)s * 2 * mm + mm + e];
  }
  Mr[(size_t)b * mm + e] = sr;
  Mi[(size_t)b * mm + e] = si;
}

cudaError_t launch_cross_gram(const double* Ga, const double* Gd, int64_t g_stride, const double* A,
                              const double* D, int64_t ab_stride, double* Mr, double* Mi, int batch, int rows,
                              int m, double* partial, cudaStream_t stream) {
  const GramSplit gs = gram_split(batch, rows);
  const int MB = bucket_of(m);
  const size_t smem = sizeof(double) * 8 * (size_t)slot_doubles(MB);
  dim3 grid(gs.splits, batch);
  cudaError_t err = cudaSuccess;
#define SSN_XGRAM_CASE(MBV)                                                                          \
  case MBV:                                                                                          \
    err = cudaFuncSetAttribute(cross_gram_kernel<MBV>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                               static_cast<int>(smem));                                             \
    if (err != cudaSuccess) return err;                                                              \
    cross_gram_kernel<MBV><<<grid, kThreads, smem, stream>>>(Ga, Gd, g_stride, A, D, ab_stride,      \
                                                             partial, rows, m, gs.chunk, gs.splits); \
    break;
  switch (MB) {
    SSN_XGRAM_CASE(1)
    SSN_XGRAM_CASE(2)
    SSN_XGRAM_CASE(3)
    SSN_XGRAM_CASE(4)
  }
#undef SSN_XGRAM_CASE
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  cross_gram_finalize_kernel<<<dim3(cdiv(m * m, 128), batch), 128, 0, stream>>>(partial, Mr, Mi, m, gs.splits);
  return cudaGetLastError();
}

// rows per recovery CTA: WR limited so 2 outputs x WR x WC x 2 <= 36 doubles
template <int MB>
struct RecTile {
  static constexpr int WC = MB;
  static constexpr int WR = imin(4, 18 / (2 * MB));
  static constexpr int ROWS = 4 * WR * 8;
};

template <int MB>
__global__ void __launch_bounds__(kThreads, 1)
    recover_kernel(const double* __restrict__ A, const double* __restrict__ D, int64_t ab_stride,
                   const double* __restrict__ P, const double* __restrict__ Q, double* __restrict__ Ur,
                   double* __restrict__ Ui, int64_t u_stride, int rows, int m) {
  extern __shared__ __align__(16) double smem[];
  using TL = RecTile<MB>;
  const int r0 = blockIdx.x * TL::ROWS, b = blockIdx.y;
  const int R = imin(TL::ROWS, rows - r0);
  const int mm = m * m;
  MatOp Aop[2] = {op_n(A + (size_t)b * ab_stride + (size_t)r0 * m, m),
                  op_n(D + (size_t)b * ab_stride + (size_t)r0 * m, m)};
  MatOp Bop[2] = {op_t(P + (size_t)b * mm, m), op_t(Q + (size_t)b * mm, m)};
  double* ur = Ur + (size_t)b * u_stride + (size_t)r0 * m;
  double* ui = Ui + (size_t)b * u_stride + (size_t)r0 * m;
  auto epi = [&](int o, int i, int j, double v) { (o == 0 ? ur : ui)[(size_t)i * m + j] = v; };
  tile_product<TL::WR, TL::WC, 2, 2, 2, C_REC>(Aop, Bop, R, m, m, smem, slot_doubles_rows(TL::ROWS, MB), epi);
}

cudaError_t launch_recover(const double* A, const double* D, int64_t ab_stride, const double* P,
                           const double* Q, double* Ur, double* Ui, int64_t u_stride, int batch,
                           int rows, int m, cudaStream_t stream) {
  const int MB = bucket_of(m);
  cudaError_t err = cudaSuccess;
#define SSN_REC_CASE(MBV)                                                                         \
  case MBV: {                                                                                     \
    const size_t smem = sizeof(double) * 8 * (size_t)slot_doubles_rows(RecTile<MBV>::ROWS, MBV); \
    err = cudaFuncSetAttribute(recover_kernel<MBV>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                               static_cast<int>(smem));                                          \
    if (err != cudaSuccess) return err;                                                           \
    dim3 grid(cdiv(rows, RecTile<MBV>::ROWS), batch);                                             \
    recover_kernel<MBV><<<grid, kThreads, smem, stream>>>(A, D, ab_stride, P, Q, Ur, Ui,          \
                                                          u_stride, rows, m);                     \
    break;                                                                                        \
  }
  switch (MB) {
    SSN_REC_CASE(1)
    SSN_REC_CASE(2)
    SSN_REC_CASE(3)
    SSN_REC_CASE(4)
  }
#undef SSN_REC_CASE
  (void)err;
  return cudaGetLastError();
}

}  // namespace ssn
