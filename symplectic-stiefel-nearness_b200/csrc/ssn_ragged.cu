// ssn_ragged.cu -- ragged batches: targets of different (n, k) in one call.
//
// The reference solves one uniform batch per call (dual_recommended_hvp.py:231-242);
// a caller with targets of many shapes calls it once per shape, one after the
// other.  ssn_solve_ragged takes them all at once: instance i is T_i [2 n_i, m_i]
// at T + t_offset[i] (X_i at the same offset of X) and omega_i [m_i, m_i] at
// omega + w_offset[i].  The host groups the instances by shape; each group is
// gathered into a contiguous uniform batch, solved by the uniform pipeline and
// scattered back, and the groups run concurrently on side streams forked from
// the caller's stream, largest first, so their latency-bound Newton kernels
// share the GPU.  Every instance converges (or fails) on its own, exactly as in
// a uniform batch; the Newton kernel's CTA-or-cluster choice sees every
// instance of the call.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "ssn.h"
#include "ssn_common.cuh"
#include "ssn_internal.h"

namespace ssn {
namespace {

constexpr int kRaggedStreams = 16;
constexpr int kCopyThreads = 256;

// Group streams for one call.  Streams beyond the device's hardware work queues
// (CUDA_DEVICE_MAX_CONNECTIONS, 8 unless set before the CUDA context is created)
// share queues and serialise one another's launches, so one stream per group up to
// that count, kRaggedStreams at most.  At the 384-target ragged workload: 8 streams
// 15.6 ms with the default 8 queues (16 streams: 15.8); with 32 queues, 16 streams
// 14.7 ms (8: 15.2, 32: 15.6).
int ragged_streams() {
  const char* s = std::getenv("CUDA_DEVICE_MAX_CONNECTIONS");
  const int c = s ? std::atoi(s) : 0;
  return imax(1, imin(kRaggedStreams, c > 0 ? c : 8));
}

size_t align_256(size_t v) { return (v + 255) / 256 * 256; }

// Group b's instances (plan indices idx[0 .. count)) copied into a contiguous batch.
__global__ void __launch_bounds__(kCopyThreads)
    ragged_gather_kernel(const double* __restrict__ src, const int64_t* __restrict__ offset,
                         const int32_t* __restrict__ idx, int64_t elems, double* __restrict__ dst) {
  const int b = blockIdx.y;
  const double2* s = reinterpret_cast<const double2*>(src + offset[idx[b]]);
  double2* d = reinterpret_cast<double2*>(dst + (size_t)b * elems);
  const int64_t n2 = elems / 2;
  for (int64_t e = blockIdx.x * (int64_t)kCopyThreads + threadIdx.x; e < n2; e += (int64_t)gridDim.x * kCopyThreads)
    d[e] = s[e];
}

// The reverse, plus the per-instance scalars (blockIdx.x == 0 writes them).
__global__ void __launch_bounds__(kCopyThreads)
    ragged_scatter_kernel(const double* __restrict__ Xg, const double* __restrict__ Wg,
                          const int64_t* __restrict__ itg, const int32_t* __restrict__ stg,
                          const int64_t* __restrict__ t_offset, const int64_t* __restrict__ w_offset,
                          const int32_t* __restrict__ idx, int64_t x_elems, int64_t w_elems, double* __restrict__ X,
                          double* __restrict__ omega, int64_t* __restrict__ iterations, int32_t* __restrict__ status) {
  const int b = blockIdx.y, i = idx[b];
  const double2* xs = reinterpret_cast<const double2*>(Xg + (size_t)b * x_elems);
  double2* xd = reinterpret_cast<double2*>(X + t_offset[i]);
  for (int64_t e = blockIdx.x * (int64_t)kCopyThreads + threadIdx.x; e < x_elems / 2; e += (int64_t)gridDim.x * kCopyThreads)
    xd[e] = xs[e];
  const double2* ws = reinterpret_cast<const double2*>(Wg + (size_t)b * w_elems);
  double2* wd = reinterpret_cast<double2*>(omega + w_offset[i]);
  for (int64_t e = blockIdx.x * (int64_t)kCopyThreads + threadIdx.x; e < w_elems / 2; e += (int64_t)gridDim.x * kCopyThreads)
    wd[e] = ws[e];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    iterations[i] = itg[b];
    status[i] = stg[b];
  }
}

struct Group {
  int n, m;
  std::vector<int32_t> members;
  size_t idx_at;                   // byte offset of its plan indices in the workspace
  size_t t_at, x_at, w_at, it_at, st_at, ws_at, end;
};

struct Plan {
  size_t t_off_at, w_off_at, total;
  std::vector<Group> groups;
};

// Deterministic plan: groups ordered by decreasing (m, n), members in input order.
Plan make_plan(int count, const int* n, const int* m) {
  std::vector<std::pair<std::pair<int, int>, int>> key(count);
  for (int i = 0; i < count; ++i) key[i] = {{-m[i], -n[i]}, i};
  std::stable_sort(key.begin(), key.end(),
                   [](const auto& a, const auto& b) { return a.first < b.first; });
  Plan p;
  for (int s = 0; s < count; ++s) {
    const int i = key[s].second;
    if (p.groups.empty() || p.groups.back().n != n[i] || p.groups.back().m != m[i]) {
      Group g{};
      g.n = n[i];
      g.m = m[i];
      p.groups.push_back(g);
    }
    p.groups.back().members.push_back(i);
  }
  size_t off = 0;
  p.t_off_at = off;
  off = align_256(off + sizeof(int64_t) * count);
  p.w_off_at = off;
  off = align_256(off + sizeof(int64_t) * count);
  for (Group& g : p.groups) {
    g.idx_at = off;
    off = align_256(off + sizeof(int32_t) * g.members.size());
  }
  for (Group& g : p.groups) {
    const size_t b = g.members.size(), tn = (size_t)2 * g.n * g.m, wn = (size_t)g.m * g.m;
    g.t_at = off;
    off = align_256(off + sizeof(double) * b * tn);
    g.x_at = off;
    off = align_256(off + sizeof(double) * b * tn);
    g.w_at = off;
    off = align_256(off + sizeof(double) * b * wn);
    g.it_at = off;
    off = align_256(off + sizeof(int64_t) * b);
    g.st_at = off;
    off = align_256(off + sizeof(int32_t) * b);
    g.ws_at = off;
    off = align_256(off + solve_workspace_bytes((int)b, g.n, g.m));
    g.end = off;
  }
  p.total = off;
  return p;
}

bool ragged_shapes_ok(int count, const int* n, const int* m) {
  if (count < 1 || !n || !m) return false;
  for (int i = 0; i < count; ++i)
    if (m[i] < 2 || m[i] > kMaxM || (m[i] % 2) != 0 || n[i] < m[i] / 2) return false;
  return true;
}

int grid_for(int64_t elems, int batch) {
  const int64_t per = (elems / 2 + kCopyThreads - 1) / kCopyThreads;
  const int64_t cap = imax(1, 4 * 148 / imax(1, batch));
  return (int)(per < cap ? (per < 1 ? 1 : per) : cap);
}

}  // namespace
}  // namespace ssn

using namespace ssn;

extern "C" {

size_t ssn_ragged_workspace_bytes(int count, const int* n, const int* m) {
  if (!ragged_shapes_ok(count, n, m)) return 0;
  return make_plan(count, n, m).total;
}

int ssn_solve_ragged(const double* T, double* X, double* omega, int64_t* iterations, int32_t* status, int count,
                     const int* n, const int* m, const int64_t* t_offset, const int64_t* w_offset,
                     void* workspace, size_t workspace_bytes, const ssn_options* opt, ssn_stream_t stream_) {
  if (!ragged_shapes_ok(count, n, m) || !T || !X || !omega || !iterations || !status || !t_offset ||
      !w_offset || !solve_options_ok(opt))
    return SSN_ERR_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(T) | reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(omega)) & 15u)
    return SSN_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < count; ++i)          // 16-byte aligned instances (offsets in doubles)
    if (t_offset[i] < 0 || w_offset[i] < 0 || (t_offset[i] % 2) != 0 || (w_offset[i] % 2) != 0)
      return SSN_ERR_INVALID_ARGUMENT;
  const Plan plan = make_plan(count, n, m);
  if (!workspace || workspace_bytes < plan.total || (reinterpret_cast<uintptr_t>(workspace) & 15u))
    return SSN_ERR_WORKSPACE;
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  char* ws = static_cast<char*>(workspace);

  // the plan (offsets and group member lists) goes up in one copy from pageable
  // host memory: the runtime stages it before returning, ordered on the stream
  std::vector<char> host(plan.groups.front().t_at, 0);
  std::memcpy(host.data() + plan.t_off_at, t_offset, sizeof(int64_t) * count);
  std::memcpy(host.data() + plan.w_off_at, w_offset, sizeof(int64_t) * count);
  for (const Group& g : plan.groups)
    std::memcpy(host.data() + g.idx_at, g.members.data(), sizeof(int32_t) * g.members.size());
  cudaError_t e = cudaMemcpyAsync(ws, host.data(), host.size(), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return SSN_ERR_CUDA;
  const int64_t* t_off_d = reinterpret_cast<const int64_t*>(ws + plan.t_off_at);
  const int64_t* w_off_d = reinterpret_cast<const int64_t*>(ws + plan.w_off_at);

  // fork: one side stream per group, up to ragged_streams(), all after the plan upload; at
  // the highest priority, so the split form's digit kernels (lowest) only fill idle SMs
  const int ns = imin(ragged_streams(), (int)plan.groups.size());
  cudaStream_t side[kRaggedStreams] = {};
  cudaEvent_t forked = nullptr, joined[kRaggedStreams] = {};
  int rc = SSN_OK, least = 0, greatest = 0;
  e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&forked, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(forked, stream);
  for (int s = 0; s < ns && e == cudaSuccess; ++s) {
    e = cudaStreamCreateWithPriority(&side[s], cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&joined[s], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side[s], forked, 0);
  }
  if (e != cudaSuccess) rc = SSN_ERR_CUDA;

  for (size_t gi = 0; gi < plan.groups.size() && rc == SSN_OK; ++gi) {
    const Group& g = plan.groups[gi];
    cudaStream_t st = side[gi % ns];
    const int b = (int)g.members.size();
    const int64_t tn = 2LL * g.n * g.m, wn = (int64_t)g.m * g.m;
    const int32_t* idx_d = reinterpret_cast<const int32_t*>(ws + g.idx_at);
    double* Tg = reinterpret_cast<double*>(ws + g.t_at);
    double* Xg = reinterpret_cast<double*>(ws + g.x_at);
    double* Wg = reinterpret_cast<double*>(ws + g.w_at);
    int64_t* itg = reinterpret_cast<int64_t*>(ws + g.it_at);
    int32_t* stg = reinterpret_cast<int32_t*>(ws + g.st_at);
    ragged_gather_kernel<<<dim3(grid_for(tn, b), b), kCopyThreads, 0, st>>>(T, t_off_d, idx_d, tn, Tg);
    if (cudaGetLastError() != cudaSuccess) {
      rc = SSN_ERR_CUDA;
      break;
    }
    rc = solve_batch(Tg, Xg, Wg, itg, stg, b, g.n, g.m, ws + g.ws_at, opt, st, count);
    if (rc != SSN_OK) break;
    ragged_scatter_kernel<<<dim3(grid_for(tn, b), b), kCopyThreads, 0, st>>>(
        Xg, Wg, itg, stg, t_off_d, w_off_d, idx_d, tn, wn, X, omega, iterations, status);
    if (cudaGetLastError() != cudaSuccess) rc = SSN_ERR_CUDA;
  }
  // join every side stream back into the caller's stream (also after an error, so nothing
  // enqueued here outlives the caller's view of the stream)
  for (int s = 0; s < ns; ++s) {
    if (side[s] && joined[s]) {
      if (cudaEventRecord(joined[s], side[s]) != cudaSuccess || cudaStreamWaitEvent(stream, joined[s], 0) != cudaSuccess)
        rc = SSN_ERR_CUDA;
    }
  }
  for (int s = 0; s < ns; ++s) {
    if (joined[s]) cudaEventDestroy(joined[s]);
    if (side[s]) cudaStreamDestroy(side[s]);
  }
  if (forked) cudaEventDestroy(forked);
  return rc;
}

}  // extern "C"
