// ssn_eigh.cu -- batched FP64 symmetric eigendecomposition (m <= 128) for the
// eigenbasis of the scaled Gram matrix, replacing the torch.linalg.eigh call of
// src/symplectic_projection/dual_recommended_hvp.py:106-108.
//
// Method: cyclic two-sided Jacobi with round-robin (circle) pair ordering; each
// step applies m/2 disjoint rotations.  Skip rule (Demmel-Veselic): rotate only
// if |a_pq| > eps * sqrt(|a_pp a_qq|); a sweep without rotations ends it.
//
// Two kernels:
//  * values (one CTA per instance, A in shared memory), two phases per step:
//    m/2 threads compute the step's rotations and its pair table; then every
//    2 x 2 block (pair a rows) x (pair b columns) is updated independently as
//    A' = J_a^T A J_b.  Each applied step's (c, s) is appended to a rotation
//    log in the workspace.
//  * vectors (one warp per row of V): rows of V = J_1 J_2 ... are independent
//    under column rotations, so each warp replays the log on its own row with
//    warp-level synchronisation only, spread over all SMs.
#include <float.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {

constexpr int kJacobiThreads = 512;
constexpr int kMaxSweeps = 24;

// index held by `slot` at step st (circle method: slot 0 fixed, the rest rotate); m1 = m - 1
__device__ __forceinline__ int rr_index(int slot, int st, int m1) {
  if (slot == 0) return 0;
  int v = slot - 1 + st;
  if (v >= m1) v -= m1;
  return 1 + v;
}

// Rotation zeroing a_pq of the 2 x 2 block [[app, apq], [apq, aqq]]:
// t = sgn(h) g / (|h| + hypot(h, g)) with h = aqq - app, g = 2 a_pq (the
// smaller root of t^2 + 2 (h/g) t - 1 = 0), c = 1/sqrt(1 + t^2), s = t c.
// Skipped (identity) when a_pq^2 <= eps^2 |a_pp a_qq|.
__device__ __forceinline__ bool make_rotation(double app, double aqq, double apq, double& c, double& s,
                                              double& t) {
  c = 1.0;
  s = 0.0;
  t = 0.0;
  if (!(apq * apq > (DBL_EPSILON * DBL_EPSILON) * fabs(app * aqq))) return false;
  const double h = aqq - app, g = 2.0 * apq;
  const double r = sqrt(h * h + g * g);
  t = (h >= 0.0 ? g : -g) / (fabs(h) + r);
  c = rsqrt(1.0 + t * t);
  s = t * c;
  return true;
}

size_t eigh_log_doubles(int batch, int m) {
  const int M = m / 2;
  return (size_t)batch * kMaxSweeps * (m - 1) * M * 2;
}

__global__ void __launch_bounds__(kJacobiThreads, 1)
    jacobi_values_kernel(const double* __restrict__ Cr, double* __restrict__ values,
                         double* __restrict__ scale_out, int32_t* __restrict__ sweeps_out,
                         int32_t* __restrict__ status_out, double* __restrict__ rlog,
                         int32_t* __restrict__ nsteps_out, int32_t* __restrict__ order_out, int m) {
  extern __shared__ __align__(16) double sm[];
  const int inst = blockIdx.x, tid = threadIdx.x;
  const int ld = m + 1, M = m / 2, m1 = m - 1;
  double* A = sm;                                                    // m x ld
  double2* cs = reinterpret_cast<double2*>(A + ((m * ld + 1) & ~1)); // [64]: (c, s) of the current step
  double* tt = reinterpret_cast<double*>(cs + 64);                   // [64]: tan of the current step
  int2* pq = reinterpret_cast<int2*>(tt + 64);                       // [64]: (p, q) of the current step, p < q
  double* red = reinterpret_cast<double*>(pq + 64);                  // kJacobiThreads/32
  int* ctl = reinterpret_cast<int*>(red + kJacobiThreads / 32);      // [0..1]: rotated in sweep (parity), [2]: last step+1
  short2* blk = reinterpret_cast<short2*>(ctl + 4);                  // off-diagonal blocks a < b
  const int nblk = M * (M - 1) / 2;

  const double* C = Cr + (size_t)inst * m * m;
  double* L = rlog + (size_t)inst * kMaxSweeps * m1 * M * 2;
  double tr = 0.0;
  for (int i = tid; i < m; i += kJacobiThreads) tr += C[(size_t)i * m + i];
  tr = block_sum<kJacobiThreads>(tr, red);
  const double scale = fmax(tr / m, 1.0);
  for (int e = tid; e < m * m; e += kJacobiThreads) {
    const int i = e / m, j = e - i * m;
    A[i * ld + j] = C[e] / scale;
  }
  for (int k = tid; k < nblk; k += kJacobiThreads) {
    int a = 0, r = k;   // row-major strict upper triangle: row a holds M - 1 - a blocks
    while (r >= M - 1 - a) { r -= M - 1 - a; ++a; }
    blk[k] = make_short2((short)a, (short)(a + 1 + r));
  }
  if (tid == 0) { ctl[0] = 0; ctl[1] = 0; ctl[2] = 0; ctl[3] = 0; }
  __syncthreads();

  int g = 0, st = 0, sweep = 0;
  bool converged = false;
  const int max_steps = kMaxSweeps * m1;
  while (g < max_steps) {
    // phase 1: rotations of this step (M threads), logged for the vectors kernel
    if (tid < M) {
      int p = rr_index(tid, st, m1), q = rr_index(m - 1 - tid, st, m1);
      if (p > q) { const int x = p; p = q; q = x; }
      double c, s, t;
      const bool rot = make_rotation(A[p * ld + p], A[q * ld + q], A[p * ld + q], c, s, t);
      cs[tid] = make_double2(c, s);
      tt[tid] = t;
      pq[tid] = make_int2(p, q);
      L[((size_t)g * M + tid) * 2 + 0] = c;
      L[((size_t)g * M + tid) * 2 + 1] = s;
      if (rot) { ctl[sweep & 1] = 1; ctl[2] = g + 1; }
    }
    __syncthreads();
    // phase 2: A <- J^T A J, every 2 x 2 block (pair a rows) x (pair b columns) independently
    for (int k = tid; k < nblk + M; k += kJacobiThreads) {
      if (k >= nblk) {                 // diagonal block of pair a
        const int a = k - nblk;
        const double2 r = cs[a];
        if (r.y == 0.0) continue;
        const int2 ia = pq[a];
        const double t = tt[a], apq = A[ia.x * ld + ia.y];
        A[ia.x * ld + ia.x] -= t * apq;
        A[ia.y * ld + ia.y] += t * apq;
        A[ia.x * ld + ia.y] = 0.0;
        A[ia.y * ld + ia.x] = 0.0;
        continue;
      }
      const short2 ab = blk[k];
      const double2 ra = cs[ab.x], rb = cs[ab.y];
      if (ra.y == 0.0 && rb.y == 0.0) continue;
      const int2 ia = pq[ab.x], ib = pq[ab.y];
      const double x = A[ia.x * ld + ib.x], y = A[ia.x * ld + ib.y];
      const double z = A[ia.y * ld + ib.x], w = A[ia.y * ld + ib.y];
      const double u0 = ra.x * x - ra.y * z, u1 = ra.x * y - ra.y * w;   // rows of J_a^T M
      const double v0 = ra.y * x + ra.x * z, v1 = ra.y * y + ra.x * w;
      const double n00 = u0 * rb.x - u1 * rb.y, n01 = u0 * rb.y + u1 * rb.x;
      const double n10 = v0 * rb.x - v1 * rb.y, n11 = v0 * rb.y + v1 * rb.x;
      A[ia.x * ld + ib.x] = n00;
      A[ib.x * ld + ia.x] = n00;
      A[ia.x * ld + ib.y] = n01;
      A[ib.y * ld + ia.x] = n01;
      A[ia.y * ld + ib.x] = n10;
      A[ib.x * ld + ia.y] = n10;
      A[ia.y * ld + ib.y] = n11;
      A[ib.y * ld + ia.y] = n11;
    }
    __syncthreads();
    ++g;
    if (++st == m1) {  // a sweep ended: stop after a sweep without rotations
      st = 0;
      // flags of this sweep's parity were last written before the barrier above;
      // the next writer of this slot is two sweeps away, behind many barriers
      const bool any = ctl[sweep & 1] != 0;
      __syncthreads();
      if (tid == 0) ctl[sweep & 1] = 0;
      ++sweep;
      if (!any) {
        converged = true;
        break;
      }
    }
  }

  // eigenvalues in ascending order; ties by index
  for (int i = tid; i < m; i += kJacobiThreads) {
    const double li = A[i * ld + i];
    int r = 0;
    for (int j = 0; j < m; ++j) {
      const double lj = A[j * ld + j];
      r += (lj < li || (lj == li && j < i)) ? 1 : 0;
    }
    values[(size_t)inst * m + r] = li;
    order_out[(size_t)inst * m + i] = r;
  }
  if (tid == 0) {
    if (scale_out) scale_out[inst] = scale;
    if (sweeps_out) sweeps_out[inst] = sweep;
    nsteps_out[inst] = ctl[2] < g ? ctl[2] : g;   // steps to replay: up to the last rotation
    bool finite = true;
    for (int i = 0; i < m; ++i) finite = finite && isfinite(A[i * ld + i]);
    if (status_out)
      status_out[inst] = !finite ? SSN_INSTANCE_NONFINITE : (converged ? SSN_INSTANCE_CONVERGED : SSN_INSTANCE_EIGH);
  }
}

constexpr int kVecWarps = 8;
constexpr int kVecChunk = 32;   // log steps staged in shared memory at a time

// V = J_1 J_2 ... J_n applied to the identity, one warp per row of V; the CTA
// stages the rotation log through shared memory in chunks of kVecChunk steps.
// Columns are written in ascending eigenvalue order.
__global__ void __launch_bounds__(kVecWarps * 32)
    jacobi_vectors_kernel(const double* __restrict__ rlog, const int32_t* __restrict__ nsteps,
                          const int32_t* __restrict__ order, double* __restrict__ vectors, int m) {
  extern __shared__ __align__(16) double sv[];
  const int inst = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * kVecWarps + warp;
  const int M = m / 2, m1 = m - 1, ld = m + 1;
  double2* chunk = reinterpret_cast<double2*>(sv);                    // [kVecChunk][M]
  double* v = sv + 2 * kVecChunk * M + warp * ld;
  const bool active = row < m;
  if (active)
    for (int c = lane; c < m; c += 32) v[c] = (c == row) ? 1.0 : 0.0;
  const double2* L = reinterpret_cast<const double2*>(rlog + (size_t)inst * kMaxSweeps * m1 * M * 2);
  const int n = nsteps[inst];
  int st = 0;
  for (int g0 = 0; g0 < n; g0 += kVecChunk) {
    const int cnt = imin(kVecChunk, n - g0);
    __syncthreads();                                                   // previous chunk consumed
    for (int e = threadIdx.x; e < cnt * M; e += kVecWarps * 32) chunk[e] = L[(size_t)g0 * M + e];
    __syncthreads();
    if (active) {
      for (int gg = 0; gg < cnt; ++gg) {
        for (int a = lane; a < M; a += 32) {
          const double2 r = chunk[gg * M + a];
          if (r.y == 0.0) continue;
          int p = rr_index(a, st, m1), q = rr_index(m - 1 - a, st, m1);
          if (p > q) { const int x = p; p = q; q = x; }
          const double vp = v[p], vq = v[q];
          v[p] = r.x * vp - r.y * vq;
          v[q] = r.y * vp + r.x * vq;
        }
        __syncwarp();
        st = (st + 1 == m1) ? 0 : st + 1;
      }
    } else {
      st = (st + cnt) % m1;
    }
  }
  if (!active) return;
  double* out = vectors + (size_t)inst * m * m + (size_t)row * m;
  const int32_t* ord = order + (size_t)inst * m;
  for (int c = lane; c < m; c += 32) out[ord[c]] = v[c];
}

size_t eigh_smem_bytes(int m) {
  const int M = m / 2;
  return sizeof(double) * ((size_t)((m * (m + 1) + 1) & ~1)) + sizeof(double2) * 64 + sizeof(double) * 64 +
         sizeof(int2) * 64 + sizeof(double) * (kJacobiThreads / 32) + sizeof(int) * 4 +
         sizeof(short2) * (size_t)(M * (M - 1) / 2 + 1) + 16;
}

size_t eigh_workspace_bytes(int batch, int m) {
  return sizeof(double) * eigh_log_doubles(batch, m) + sizeof(int32_t) * (size_t)batch * (m + 1) + 256;
}

cudaError_t launch_eigh(const double* Cr, double* values, double* vectors, double* scale,
                        int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                        cudaStream_t stream) {
  double* rlog = static_cast<double*>(workspace);
  int32_t* nsteps = reinterpret_cast<int32_t*>(rlog + eigh_log_doubles(batch, m));
  int32_t* order = nsteps + batch;
  const size_t smem = eigh_smem_bytes(m);
  cudaError_t err = cudaFuncSetAttribute(jacobi_values_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  jacobi_values_kernel<<<batch, kJacobiThreads, smem, stream>>>(Cr, values, scale, sweeps, status, rlog,
                                                               nsteps, order, m);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const size_t vsmem = sizeof(double) * (2 * kVecChunk * (m / 2) + kVecWarps * (m + 1));
  dim3 grid(cdiv(m, kVecWarps), batch);
  jacobi_vectors_kernel<<<grid, kVecWarps * 32, vsmem, stream>>>(rlog, nsteps, order, vectors, m);
  return cudaGetLastError();
}

}  // namespace ssn
