// ssn_eigh.cu -- batched FP64 symmetric eigendecomposition (m <= 128) for the
// eigenbasis of the scaled Gram matrix, replacing the torch.linalg.eigh call of
// src/symplectic_projection/dual_recommended_hvp.py:106-108.
//
// Method: cyclic two-sided Jacobi with round-robin (circle) pair ordering, so
// each step applies m/2 disjoint rotations.  A step updates every 2x2 block
// (pair a rows) x (pair b cols) as A' = J_a^T A J_b, independent per block, so
// one barrier separates the angle phase from the update phase.
//
// Layout: one 2-CTA thread-block cluster per instance.  CTA rank 0 keeps A in
// shared memory and computes angles; CTA rank 1 keeps the accumulated
// eigenvectors V in shared memory.  Rank 0 writes each step's (c, s) into
// rank 1's shared memory (distributed shared memory) and one cluster barrier per
// step hands them over, so the A and V updates run concurrently on two SMs.
// Skip rule (Demmel-Veselic): rotate only if |a_pq| > eps * sqrt(|a_pp a_qq|);
// a sweep without rotations ends the iteration (at most kMaxSweeps sweeps).
#include <cooperative_groups.h>
#include <float.h>

#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace cg = cooperative_groups;

namespace ssn {

constexpr int kEighThreads = 512;
constexpr int kMaxSweeps = 40;

struct EighCtrl {
  int stop;       // written by rank 0 into rank 1 at the end of a sweep
  int rotated;    // rank 0: any rotation in the current sweep
  int pad[2];
};

__device__ __forceinline__ int rr_index(int slot, int step, int m) {
  return slot == 0 ? 0 : 1 + (slot - 1 + step) % (m - 1);
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kEighThreads, 1)
    eigh_kernel(const double* __restrict__ Cr, double* __restrict__ values, double* __restrict__ vectors,
                double* __restrict__ scale_out, int32_t* __restrict__ sweeps_out,
                int32_t* __restrict__ status_out, int m) {
  extern __shared__ __align__(16) double sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const int inst = blockIdx.x >> 1;
  const int tid = threadIdx.x;
  const int ld = m + 1;
  const int M = m / 2;
  double* mat = sm;                                    // A (rank 0) or V (rank 1), m x ld
  double* ang = sm + m * ld;                           // [2][64][3]: c, s, t
  EighCtrl* ctrl = reinterpret_cast<EighCtrl*>(ang + 2 * 64 * 3);
  double* red = reinterpret_cast<double*>(ctrl + 1);   // kEighThreads/32 doubles
  int* rank_of = reinterpret_cast<int*>(red + kEighThreads / 32);  // [m]

  double* remote_ang = cluster.map_shared_rank(ang, 1);
  EighCtrl* remote_ctrl = cluster.map_shared_rank(ctrl, 1);
  int* remote_rank_of = cluster.map_shared_rank(rank_of, 1);

  const double* C = Cr + (size_t)inst * m * m;
  double scale = 1.0;
  if (rank == 0) {
    double tr = 0.0;
    for (int i = tid; i < m; i += kEighThreads) tr += C[(size_t)i * m + i];
    tr = block_sum<kEighThreads>(tr, red);
    scale = fmax(tr / m, 1.0);
    for (int e = tid; e < m * m; e += kEighThreads) {
      const int i = e / m, j = e - i * m;
      mat[i * ld + j] = C[e] / scale;
    }
    if (tid == 0) {
      ctrl->rotated = 0;
      ctrl->stop = 0;
    }
  } else {
    for (int e = tid; e < m * m; e += kEighThreads) {
      const int i = e / m, j = e - i * m;
      mat[i * ld + j] = (i == j) ? 1.0 : 0.0;
    }
    if (tid == 0) ctrl->stop = 0;
  }
  cluster.sync();

  int sweep = 0;
  bool converged = false;
  for (; sweep < kMaxSweeps; ++sweep) {
    for (int step = 0; step < m - 1; ++step) {
      const int buf = step & 1;
      double* a_ang = ang + buf * 64 * 3;
      if (rank == 0 && tid < M) {
        int p = rr_index(tid, step, m), q = rr_index(m - 1 - tid, step, m);
        if (p > q) {
          const int tmp = p;
          p = q;
          q = tmp;
        }
        const double app = mat[p * ld + p], aqq = mat[q * ld + q], apq = mat[p * ld + q];
        double c = 1.0, s = 0.0, tt = 0.0;
        if (apq != 0.0 && fabs(apq) > DBL_EPSILON * sqrt(fabs(app * aqq))) {
          const double zeta = (aqq - app) / (2.0 * apq);
          if (fabs(zeta) > 1e150) {
            tt = 0.5 / zeta;
          } else {
            tt = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          }
          c = 1.0 / sqrt(1.0 + tt * tt);
          s = tt * c;
          ctrl->rotated = 1;
        }
        a_ang[tid * 3 + 0] = c;
        a_ang[tid * 3 + 1] = s;
        a_ang[tid * 3 + 2] = tt;
        double* r_ang = remote_ang + buf * 64 * 3;
        r_ang[tid * 3 + 0] = c;
        r_ang[tid * 3 + 1] = s;
      }
      cluster.sync();
      if (rank == 0) {
        for (int idx = tid; idx < M * M; idx += kEighThreads) {
          const int a = idx / M, b = idx - a * M;
          if (a > b) continue;
          const double sa = a_ang[a * 3 + 1], sb = a_ang[b * 3 + 1];
          if (sa == 0.0 && sb == 0.0) continue;
          int pa = rr_index(a, step, m), qa = rr_index(m - 1 - a, step, m);
          if (pa > qa) { const int tmp = pa; pa = qa; qa = tmp; }
          if (a == b) {
            const double tt = a_ang[a * 3 + 2];
            const double apq = mat[pa * ld + qa];
            mat[pa * ld + pa] -= tt * apq;
            mat[qa * ld + qa] += tt * apq;
            mat[pa * ld + qa] = 0.0;
            mat[qa * ld + pa] = 0.0;
          } else {
            int pb = rr_index(b, step, m), qb = rr_index(m - 1 - b, step, m);
            if (pb > qb) { const int tmp = pb; pb = qb; qb = tmp; }
            const double ca = a_ang[a * 3 + 0], cb = a_ang[b * 3 + 0];
            const double x = mat[pa * ld + pb], y = mat[pa * ld + qb];
            const double z = mat[qa * ld + pb], w = mat[qa * ld + qb];
            const double u0 = ca * x - sa * z, u1 = ca * y - sa * w;  // row pa of J_a^T M
            const double v0 = sa * x + ca * z, v1 = sa * y + ca * w;  // row qa
            const double n_pp = u0 * cb - u1 * sb, n_pq = u0 * sb + u1 * cb;
            const double n_qp = v0 * cb - v1 * sb, n_qq = v0 * sb + v1 * cb;
            mat[pa * ld + pb] = n_pp;
            mat[pb * ld + pa] = n_pp;
            mat[pa * ld + qb] = n_pq;
            mat[qb * ld + pa] = n_pq;
            mat[qa * ld + pb] = n_qp;
            mat[pb * ld + qa] = n_qp;
            mat[qa * ld + qb] = n_qq;
            mat[qb * ld + qa] = n_qq;
          }
        }
        __syncthreads();
      } else {
        for (int idx = tid; idx < m * M; idx += kEighThreads) {
          const int r = idx / M, a = idx - r * M;
          const double s = a_ang[a * 3 + 1];
          if (s == 0.0) continue;
          const double c = a_ang[a * 3 + 0];
          int p = rr_index(a, step, m), q = rr_index(m - 1 - a, step, m);
          if (p > q) { const int tmp = p; p = q; q = tmp; }
          const double vp = mat[r * ld + p], vq = mat[r * ld + q];
          mat[r * ld + p] = c * vp - s * vq;
          mat[r * ld + q] = s * vp + c * vq;
        }
      }
    }
    if (rank == 0 && tid == 0) {
      const int stop = ctrl->rotated == 0 ? 1 : 0;
      ctrl->stop = stop;
      remote_ctrl->stop = stop;
      ctrl->rotated = 0;
    }
    cluster.sync();
    if (ctrl->stop) {
      converged = true;
      ++sweep;
      break;
    }
  }

  // ascending order; ties broken by index
  if (rank == 0) {
    for (int i = tid; i < m; i += kEighThreads) {
      const double li = mat[i * ld + i];
      int r = 0;
      for (int j = 0; j < m; ++j) {
        const double lj = mat[j * ld + j];
        r += (lj < li || (lj == li && j < i)) ? 1 : 0;
      }
      remote_rank_of[i] = r;
      values[(size_t)inst * m + r] = li;
    }
    if (tid == 0) {
      if (scale_out) scale_out[inst] = scale;
      if (sweeps_out) sweeps_out[inst] = sweep;
      bool finite = true;
      for (int i = 0; i < m; ++i) finite = finite && isfinite(mat[i * ld + i]);
      if (status_out) status_out[inst] = !finite ? SSN_INSTANCE_NONFINITE
                                          : (converged ? SSN_INSTANCE_CONVERGED : SSN_INSTANCE_EIGH);
    }
  }
  cluster.sync();
  if (rank == 1) {
    double* Vout = vectors + (size_t)inst * m * m;
    for (int e = tid; e < m * m; e += kEighThreads) {
      const int r = e / m, i = e - r * m;
      Vout[(size_t)r * m + rank_of[i]] = mat[r * ld + i];
    }
  }
}

size_t eigh_smem_bytes(int m) {
  return sizeof(double) * ((size_t)m * (m + 1) + 2 * 64 * 3) + sizeof(EighCtrl) +
         sizeof(double) * (kEighThreads / 32) + sizeof(int) * kMaxM;
}

cudaError_t launch_eigh(const double* Cr, double* values, double* vectors, double* scale,
                        int32_t* sweeps, int32_t* status, int batch, int m, cudaStream_t stream) {
  const size_t smem = eigh_smem_bytes(m);
  cudaError_t err = cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  eigh_kernel<<<2 * batch, kEighThreads, smem, stream>>>(Cr, values, vectors, scale, sweeps, status, m);
  return cudaGetLastError();
}

}  // namespace ssn
