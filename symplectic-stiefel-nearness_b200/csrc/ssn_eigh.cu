// ssn_eigh.cu -- batched FP64 symmetric eigendecomposition (m <= 128) for the
// eigenbasis of the scaled Gram matrix, replacing the torch.linalg.eigh call of
// src/symplectic_projection/dual_recommended_hvp.py:106-108.
//
// Method: cyclic two-sided Jacobi with round-robin (circle) pair ordering; each
// step applies m/2 disjoint rotations.  Skip rule (Demmel-Veselic): rotate only
// if |a_pq| > eps * sqrt(|a_pp a_qq|); a sweep without rotations ends it.
//
// Two kernels:
//  * values (one CTA per instance, A in shared memory), one barrier per step:
//    every 2 x 2 block (pair a rows) x (pair b columns) is updated independently
//    as A' = J_a^T A J_b; the threads owning the fixed "host" blocks (which hold
//    the next step's pairs) also compute the next step's rotations.  Each
//    applied step's (c, s) is appended to a rotation log in the workspace.
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
template <class Real>
struct JReal;
template <>
struct JReal<double> {
  using V2 = double2;
  static constexpr double eps = DBL_EPSILON;
  __device__ static double2 make2(double a, double b) { return make_double2(a, b); }
};
template <>
struct JReal<float> {
  using V2 = float2;
  static constexpr float eps = FLT_EPSILON;
  __device__ static float2 make2(float a, float b) { return make_float2(a, b); }
};

template <class Real>
__device__ __forceinline__ bool make_rotation(Real app, Real aqq, Real apq, Real& c, Real& s, Real& t) {
  constexpr Real eps = JReal<Real>::eps;
  c = Real(1);
  s = Real(0);
  t = Real(0);
  if (!(apq * apq > (eps * eps) * fabs(app * aqq))) return false;
  const Real h = aqq - app, g = Real(2) * apq;
  const Real r = sqrt(h * h + g * g);
  t = (h >= Real(0) ? g : -g) / (fabs(h) + r);
  c = rsqrt(Real(1) + t * t);
  s = t * c;
  return true;
}

size_t eigh_log_doubles(int batch, int m) {
  const int M = m / 2;
  return (size_t)batch * kMaxSweeps * (m - 1) * M * 2;
}

// Circle method in slot space: after one step the index in slot u (u >= 1)
// moves to slot u - 1 (slot 1 wraps to slot m - 1); slot 0 is fixed.  Hence the
// pair a' of the next step is formed by the step-st slots (a' + 1, m - a')
// (a' >= 1) or (0, 1) (a' = 0): one entry of the 2 x 2 block of the current
// slot pairs (a' - 1, min(a' + 1, m - 2 - a')) or (0, 1).  That "host" block
// is the same for every step, so a fixed set of threads can update it and
// compute the next rotation right away, without a second barrier.
__device__ __forceinline__ int pair_of_slot(int u, int m) { return u < m - 1 - u ? u : m - 1 - u; }

__device__ __forceinline__ void host_block(int ap, int m, int& bx, int& by, int& sx, int& sy) {
  // next-step pair ap lives at step-st slots (sx, sy) inside slot-pair block (bx, by)
  if (ap == 0) {
    sx = 0;
    sy = 1;
  } else {
    sx = m - ap;
    sy = ap + 1;
  }
  bx = pair_of_slot(sx, m);
  by = pair_of_slot(sy, m);
}

template <class Real>
__global__ void __launch_bounds__(kJacobiThreads, 1)
    jacobi_values_kernel(const double* __restrict__ Cr, double* __restrict__ values,
                         double* __restrict__ scale_out, int32_t* __restrict__ sweeps_out,
                         int32_t* __restrict__ status_out, Real* __restrict__ rlog,
                         int32_t* __restrict__ nsteps_out, int32_t* __restrict__ order_out, int m,
                         int max_sweeps, int strict, float skip_corr) {
  using V2 = typename JReal<Real>::V2;
  extern __shared__ __align__(16) double sm_raw[];
  Real* sm = reinterpret_cast<Real*>(sm_raw);
  const int inst = blockIdx.x, tid = threadIdx.x;
  const int ld = m + 1, M = m / 2, m1 = m - 1;
  Real* A = sm;                                                      // m x ld
  V2* cs = reinterpret_cast<V2*>(A + ((m * ld + 3) & ~3));           // [2][64]: (c, s)
  V2* dg = cs + 2 * 64;                                              // [2][64]: diagonal entries after the rotation
  Real* tt = reinterpret_cast<Real*>(dg + 2 * 64);                   // [2][64]: tan
  int2* pq = reinterpret_cast<int2*>(tt + 2 * 64);                   // [2][64]: (p, q), p < q
  double* red = reinterpret_cast<double*>(pq + 2 * 64);              // kJacobiThreads/32
  int* ctl = reinterpret_cast<int*>(red + kJacobiThreads / 32);      // [0..1]: rotated in sweep (parity), [2]: last step+1
  short2* blk = reinterpret_cast<short2*>(ctl + 4);                  // blocks of the generic threads
  // m >= 6: warps 0-1 own the M host blocks; the other warps own the rest (incl. diagonal blocks).
  // m <= 4: host blocks coincide, so rotations are computed in a separate phase instead.
  const bool hosted = m >= 6;
  constexpr int kHostThreads = 64;
  constexpr int kHostFlag = 0x100;

  const double* C = Cr + (size_t)inst * m * m;
  Real* L = rlog + (size_t)inst * kMaxSweeps * m1 * M * 2;
  double tr = 0.0;
  for (int i = tid; i < m; i += kJacobiThreads) tr += C[(size_t)i * m + i];
  tr = block_sum<kJacobiThreads>(tr, red);
  const double scale = fmax(tr / m, 1.0);
  for (int e = tid; e < m * m; e += kJacobiThreads) {
    const int i = e / m, j = e - i * m;
    A[i * ld + j] = static_cast<Real>(C[e] / scale);
  }
  // rough basis (skip_corr > 0): when every off-diagonal correlation
  // |a_pq| / sqrt(a_pp a_qq) of the scaled Gram is below skip_corr, the identity
  // already nearly diagonalises it and no sweep is run (a CTA-wide max, so every
  // thread takes the same decision)
  int sweeps_cap = max_sweeps;
  if (skip_corr > 0.0f) {
    // c_pq^2 >= skip^2 c_pp c_qq for some pair (no square root or division per entry)
    const double s2 = static_cast<double>(skip_corr) * static_cast<double>(skip_corr);
    int keep = 0;
    for (int e = tid; e < m * m; e += kJacobiThreads) {
      const int i = e / m, j = e - i * m;
      if (i < j) {
        const double d = C[(size_t)i * m + i] * C[(size_t)j * m + j];
        const double c = fabs(C[e]);
        if (d > 0.0) keep |= (c * c >= s2 * d) ? 1 : 0;
        else if (c > 0.0 || !(d == 0.0)) keep = 1;   // non-finite or inconsistent: keep the sweeps
      }
    }
    if (!__syncthreads_or(keep)) sweeps_cap = 0;
  }
  // block list: off-diagonal blocks (a < b) row-major, then the diagonal blocks.
  // Host blocks carry kHostFlag in .y and are skipped by the generic threads.
  // Block (a, b), a < b, hosts next pair a' iff it equals (a' - 1, P1(a')) with
  // P1(a') = min(a' + 1, m - 2 - a'), or is (0, 1) (a' = 0): an O(1) test.
  const int noff = M * (M - 1) / 2, nblk = noff + M;
  for (int k = tid; k < nblk; k += kJacobiThreads) {
    int a, b;
    if (k < noff) {
      a = 0;
      int r = k;
      while (r >= M - 1 - a) { r -= M - 1 - a; ++a; }
      b = a + 1 + r;
    } else {
      a = b = k - noff;
    }
    bool host = false;
    if (hosted && a != b) {
      auto p1 = [&](int ap) { return imin(ap + 1, m - 2 - ap); };
      host = (a == 0 && b == 1) || (a + 1 < M && p1(a + 1) == b) || (b + 1 < M && p1(b + 1) == a);
    }
    blk[k] = make_short2((short)a, (short)(host ? (b | kHostFlag) : b));
  }
  if (tid == 0) { ctl[0] = 0; ctl[1] = 0; ctl[2] = 0; ctl[3] = 0; }
  __syncthreads();

  auto rotate_pair = [&](int a, int st, int buf, int g, Real app, Real aqq, Real apq, int p, int q) {
    Real c, s, t;
    const bool rot = make_rotation<Real>(app, aqq, apq, c, s, t);
    cs[buf * 64 + a] = JReal<Real>::make2(c, s);
    dg[buf * 64 + a] = JReal<Real>::make2(app - t * apq, aqq + t * apq);
    tt[buf * 64 + a] = t;
    pq[buf * 64 + a] = make_int2(p, q);
    L[((size_t)g * M + a) * 2 + 0] = c;
    L[((size_t)g * M + a) * 2 + 1] = s;
    return rot;
  };

  // rotations of step 0
  if (tid < M) {
    int p = rr_index(tid, 0, m1), q = rr_index(m - 1 - tid, 0, m1);
    if (p > q) { const int x = p; p = q; q = x; }
    if (rotate_pair(tid, 0, 0, 0, A[p * ld + p], A[q * ld + q], A[p * ld + q], p, q)) {
      ctl[0] = 1;
      ctl[2] = 1;
    }
  }
  __syncthreads();

  int g = 0, st = 0, sweep = 0;
  bool converged = false;
  const int max_steps = imin(sweeps_cap, kMaxSweeps) * m1;
  while (g < max_steps) {
    const int cur = g & 1, nxt = cur ^ 1;
    const int nsweep = (st + 1 == m1) ? sweep + 1 : sweep;
    const V2* csc = cs + cur * 64;
    const V2* dgc = dg + cur * 64;
    const int2* pqc = pq + cur * 64;
    if (hosted && tid < kHostThreads) {
      const int ap = tid;
      if (ap < M && g + 1 < max_steps) {
        int bx, by, sx, sy;
        host_block(ap, m, bx, by, sx, sy);
        const int x = rr_index(sx, st, m1), y = rr_index(sy, st, m1);   // next pair's indices
        const V2 ra = csc[bx], rb = csc[by];
        const int2 ia = pqc[bx], ib = pqc[by];
        Real nv[2][2];
        nv[0][0] = A[ia.x * ld + ib.x];
        nv[0][1] = A[ia.x * ld + ib.y];
        nv[1][0] = A[ia.y * ld + ib.x];
        nv[1][1] = A[ia.y * ld + ib.y];
        if (ra.y != Real(0) || rb.y != Real(0)) {
          const Real u0 = ra.x * nv[0][0] - ra.y * nv[1][0], u1 = ra.x * nv[0][1] - ra.y * nv[1][1];
          const Real v0 = ra.y * nv[0][0] + ra.x * nv[1][0], v1 = ra.y * nv[0][1] + ra.x * nv[1][1];
          nv[0][0] = u0 * rb.x - u1 * rb.y;
          nv[0][1] = u0 * rb.y + u1 * rb.x;
          nv[1][0] = v0 * rb.x - v1 * rb.y;
          nv[1][1] = v0 * rb.y + v1 * rb.x;
          A[ia.x * ld + ib.x] = nv[0][0];
          A[ib.x * ld + ia.x] = nv[0][0];
          A[ia.x * ld + ib.y] = nv[0][1];
          A[ib.y * ld + ia.x] = nv[0][1];
          A[ia.y * ld + ib.x] = nv[1][0];
          A[ib.x * ld + ia.y] = nv[1][0];
          A[ia.y * ld + ib.y] = nv[1][1];
          A[ib.y * ld + ia.y] = nv[1][1];
        }
        // x belongs to pair bx, y to pair by; their diagonal entries after this step
        const int ux = (x == ia.x) ? 0 : 1, uy = (y == ib.x) ? 0 : 1;
        const Real dx = ux == 0 ? dgc[bx].x : dgc[bx].y;
        const Real dy = uy == 0 ? dgc[by].x : dgc[by].y;
        const Real axy = nv[ux][uy];
        const bool xfirst = x < y;
        if (rotate_pair(ap, 0, nxt, g + 1, xfirst ? dx : dy, xfirst ? dy : dx, axy, xfirst ? x : y,
                        xfirst ? y : x)) {
          ctl[nsweep & 1] = 1;
          ctl[2] = g + 2;
        }
      }
    } else if (hosted || tid >= 0) {
      const int first = hosted ? tid - kHostThreads : tid;
      const int stride = hosted ? kJacobiThreads - kHostThreads : kJacobiThreads;
      for (int k = first; k < nblk; k += stride) {
        const short2 ab = blk[k];
        if (ab.y & kHostFlag) continue;          // owned by a host thread
        const V2 ra = csc[ab.x];
        if (ab.x == ab.y) {                      // diagonal block of pair a
          if (ra.y == Real(0)) continue;
          const int2 ia = pqc[ab.x];
          const V2 d = dgc[ab.x];
          A[ia.x * ld + ia.x] = d.x;
          A[ia.y * ld + ia.y] = d.y;
          A[ia.x * ld + ia.y] = Real(0);
          A[ia.y * ld + ia.x] = Real(0);
          continue;
        }
        const V2 rb = csc[ab.y];
        if (ra.y == Real(0) && rb.y == Real(0)) continue;
        const int2 ia = pqc[ab.x], ib = pqc[ab.y];
        const Real x = A[ia.x * ld + ib.x], y = A[ia.x * ld + ib.y];
        const Real z = A[ia.y * ld + ib.x], w = A[ia.y * ld + ib.y];
        const Real u0 = ra.x * x - ra.y * z, u1 = ra.x * y - ra.y * w;   // rows of J_a^T M
        const Real v0 = ra.y * x + ra.x * z, v1 = ra.y * y + ra.x * w;
        const Real n00 = u0 * rb.x - u1 * rb.y, n01 = u0 * rb.y + u1 * rb.x;
        const Real n10 = v0 * rb.x - v1 * rb.y, n11 = v0 * rb.y + v1 * rb.x;
        A[ia.x * ld + ib.x] = n00;
        A[ib.x * ld + ia.x] = n00;
        A[ia.x * ld + ib.y] = n01;
        A[ib.y * ld + ia.x] = n01;
        A[ia.y * ld + ib.x] = n10;
        A[ib.x * ld + ia.y] = n10;
        A[ia.y * ld + ib.y] = n11;
        A[ib.y * ld + ia.y] = n11;
      }
    }
    __syncthreads();
    if (!hosted && g + 1 < max_steps) {     // m <= 4: rotations of the next step in their own phase
      const int nst = (st + 1 == m1) ? 0 : st + 1;
      if (tid < M) {
        int p = rr_index(tid, nst, m1), q = rr_index(m - 1 - tid, nst, m1);
        if (p > q) { const int x = p; p = q; q = x; }
        if (rotate_pair(tid, nst, nxt, g + 1, A[p * ld + p], A[q * ld + q], A[p * ld + q], p, q)) {
          ctl[nsweep & 1] = 1;
          ctl[2] = g + 2;
        }
      }
      __syncthreads();
    }
    ++g;
    if (++st == m1) {  // a sweep ended: stop after a sweep without rotations
      st = 0;
      // this sweep's flag was last written before the barrier above; the next
      // writer of this parity slot is two sweeps away, behind many barriers
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
    const Real li = A[i * ld + i];
    int r = 0;
    for (int j = 0; j < m; ++j) {
      const Real lj = A[j * ld + j];
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
      status_out[inst] = !finite ? SSN_INSTANCE_NONFINITE
                         : (converged || !strict) ? SSN_INSTANCE_CONVERGED : SSN_INSTANCE_EIGH;
  }
}

constexpr int kVecWarps = 16;
constexpr int kVecChunk = 16;   // log steps staged in shared memory at a time

// V = J_1 J_2 ... J_n applied to the identity, one warp per row of V.  The CTA
// keeps the pair table of all m - 1 steps of a sweep and stages the rotation
// log through shared memory in chunks of kVecChunk steps.  Columns are written
// in ascending eigenvalue order.
template <class Real>
__global__ void __launch_bounds__(kVecWarps * 32)
    jacobi_vectors_kernel(const Real* __restrict__ rlog, const int32_t* __restrict__ nsteps,
                          const int32_t* __restrict__ order, double* __restrict__ vectors, int m) {
  using V2 = typename JReal<Real>::V2;
  extern __shared__ __align__(16) double sv_raw[];
  Real* sv = reinterpret_cast<Real*>(sv_raw);
  const int inst = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * kVecWarps + warp;
  const int M = m / 2, m1 = m - 1, ld = m + 1;
  V2* chunk = reinterpret_cast<V2*>(sv);                              // [kVecChunk][M]
  Real* v = sv + 2 * kVecChunk * M + warp * ld;
  short2* pt = reinterpret_cast<short2*>(sv + 2 * kVecChunk * M + kVecWarps * ld);  // [m1][M]
  for (int e = threadIdx.x; e < m1 * M; e += kVecWarps * 32) {
    const int st = e / M, a = e - st * M;
    int p = rr_index(a, st, m1), q = rr_index(m - 1 - a, st, m1);
    if (p > q) { const int x = p; p = q; q = x; }
    pt[e] = make_short2((short)p, (short)q);
  }
  const bool active = row < m;
  if (active)
    for (int c = lane; c < m; c += 32) v[c] = (c == row) ? Real(1) : Real(0);
  const V2* L = reinterpret_cast<const V2*>(rlog + (size_t)inst * kMaxSweeps * m1 * M * 2);
  const int n = nsteps[inst];
  int st = 0;
  for (int g0 = 0; g0 < n; g0 += kVecChunk) {
    const int cnt = imin(kVecChunk, n - g0);
    __syncthreads();                                                   // previous chunk consumed
    for (int e = threadIdx.x; e < cnt * M; e += kVecWarps * 32) chunk[e] = L[(size_t)g0 * M + e];
    __syncthreads();
    if (active) {
      for (int gg = 0; gg < cnt; ++gg) {
        const V2* cr = chunk + gg * M;
        const short2* pr = pt + st * M;
        for (int a = lane; a < M; a += 32) {
          const V2 r = cr[a];
          if (r.y == Real(0)) continue;
          const short2 ij = pr[a];
          const Real vp = v[ij.x], vq = v[ij.y];
          v[ij.x] = r.x * vp - r.y * vq;
          v[ij.y] = r.y * vp + r.x * vq;
        }
        __syncwarp();
        st = (st + 1 == m1) ? 0 : st + 1;
      }
    }
  }
  if (!active) return;
  double* out = vectors + (size_t)inst * m * m + (size_t)row * m;
  const int32_t* ord = order + (size_t)inst * m;
  for (int c = lane; c < m; c += 32) out[ord[c]] = v[c];
}

template <class Real>
static size_t eigh_smem_bytes_t(int m) {
  const int M = m / 2;
  return sizeof(Real) * ((size_t)((m * (m + 1) + 3) & ~3)) + 2 * sizeof(Real) * 4 * 64 +
         sizeof(Real) * 2 * 64 + sizeof(int2) * 2 * 64 + sizeof(double) * (kJacobiThreads / 32) +
         sizeof(int) * 4 + sizeof(short2) * (size_t)(M * (M + 1) / 2 + 1) + 16;
}

size_t eigh_smem_bytes(int m) { return eigh_smem_bytes_t<double>(m); }

size_t eigh_workspace_bytes(int batch, int m) {
  return sizeof(double) * eigh_log_doubles(batch, m) + sizeof(int32_t) * (size_t)batch * (m + 1) + 256;
}

template <class Real>
static cudaError_t launch_eigh_t(const double* Cr, double* values, double* vectors, double* scale,
                                 int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                                 int max_sweeps, bool strict, float skip_corr, cudaStream_t stream) {
  Real* rlog = static_cast<Real*>(workspace);
  int32_t* nsteps = reinterpret_cast<int32_t*>(static_cast<double*>(workspace) + eigh_log_doubles(batch, m));
  int32_t* order = nsteps + batch;
  const size_t smem = eigh_smem_bytes_t<Real>(m);
  cudaError_t err = cudaFuncSetAttribute(jacobi_values_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  jacobi_values_kernel<Real><<<batch, kJacobiThreads, smem, stream>>>(Cr, values, scale, sweeps, status, rlog,
                                                                     nsteps, order, m, max_sweeps, strict ? 1 : 0,
                                                                     skip_corr);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const size_t vsmem = sizeof(Real) * (2 * kVecChunk * (m / 2) + kVecWarps * (m + 1)) +
                       sizeof(short2) * (size_t)(m - 1) * (m / 2) + 16;
  err = cudaFuncSetAttribute(jacobi_vectors_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(vsmem));
  if (err != cudaSuccess) return err;
  dim3 grid(cdiv(m, kVecWarps), batch);
  jacobi_vectors_kernel<Real><<<grid, kVecWarps * 32, vsmem, stream>>>(rlog, nsteps, order, vectors, m);
  return cudaGetLastError();
}

cudaError_t launch_eigh(const double* Cr, double* values, double* vectors, double* scale,
                        int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                        cudaStream_t stream) {
  return launch_eigh_t<double>(Cr, values, vectors, scale, sweeps, status, batch, m, workspace, kMaxSweeps,
                               true, 0.0f, stream);
}

cudaError_t launch_eigh_approx(const double* Cr, double* values, double* vectors, double* scale,
                               int32_t* sweeps, int32_t* status, int batch, int m, void* workspace,
                               int max_sweeps, bool fp32, float skip_corr, cudaStream_t stream) {
  if (max_sweeps < 1) max_sweeps = 1;
  if (max_sweeps > kMaxSweeps) max_sweeps = kMaxSweeps;
  return fp32 ? launch_eigh_t<float>(Cr, values, vectors, scale, sweeps, status, batch, m, workspace,
                                     max_sweeps, false, skip_corr, stream)
              : launch_eigh_t<double>(Cr, values, vectors, scale, sweeps, status, batch, m, workspace,
                                      max_sweeps, false, skip_corr, stream);
}

}  // namespace ssn
