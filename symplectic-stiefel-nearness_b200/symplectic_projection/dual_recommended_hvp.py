"""Batched dual Newton-CG solver: host side of the drop-in ``solve``.

Mirrors src/symplectic_projection/dual_recommended_hvp.py of the reference:
same constants, ``solve(T) -> (X, omega, iterations)`` for CPU float64 input
(CPU output) and, additionally, CUDA input (device-resident output).  The
pipeline Gram -> eigh -> Newton-CG -> recovery is one C-ABI call
(``ssn_solve``) enqueued on torch's current stream; the host only checks the
per-instance status words afterwards and raises ``RuntimeError`` for the whole
batch on a Newton or line-search cap, as the reference does
(dual_recommended_hvp.py:189-191).
"""
from __future__ import annotations

import os
import threading
from dataclasses import dataclass

import torch

from . import _native as N
from ._workspace import workspace
from .cholesky_inverse_kernel import cholesky_k

# dual_recommended_hvp.py:13-19
ROW_CHUNK = 1024
DEVICE = "cuda"
FEAS_TOL = 1e-8
MAX_NEWTON, MAX_CG, MAX_BACKTRACK = 100, 150, 40
PINNED_OUTPUT_MIN_BYTES = 64 * 2**20

_MESSAGES = {
    3: "batched Newton iteration cap reached",
    4: "batched line search found no descent step",
    6: "Jacobi eigensolver did not converge",
}


@dataclass
class SolveResult:
    """Extended result of :func:`solve_ex` (all tensors on the input's device)."""
    X: torch.Tensor
    omega: torch.Tensor
    iterations: torch.Tensor
    status: torch.Tensor        # int32 per instance: 0 converged, 3 Newton cap, 4 line search, 5 non-finite, 6 eigh


def _check_target(T):
    if not isinstance(T, torch.Tensor) or T.dtype != torch.float64:
        raise ValueError("T must be a torch.float64 tensor; no implicit precision conversion")
    if T.ndim != 3 or T.shape[-2] % 2 or T.shape[-1] % 2 or T.shape[-1] == 0:
        raise ValueError("T must have shape [batch, 2n, 2k] with k >= 1")
    batch, rows, m = T.shape
    if m > 128:
        raise ValueError("2k <= 128 is supported")
    if rows < m:
        raise ValueError("n >= k is required")
    return batch, rows // 2, m


def _pinned_like(T: torch.Tensor) -> torch.Tensor:
    big = T.numel() * T.element_size() >= PINNED_OUTPUT_MIN_BYTES
    return torch.empty(T.shape, dtype=T.dtype, pin_memory=big)


@torch.no_grad()
def solve_ex(T: torch.Tensor, *, max_newton: int = MAX_NEWTON, max_cg: int = MAX_CG,
             max_backtrack: int = MAX_BACKTRACK, feas_tol: float = FEAS_TOL,
             precision: str = "fp64", eig_sweeps: int = 0, preconditioner: str = "eigenbasis",
             fp32_newton: bool = True, raise_on_failure: bool = False) -> SolveResult:
    """Device-resident solve with per-instance status.  T must be a CUDA tensor.

    precision="fp64" is the plain FP64 form (the reference's iterates);
    precision="split" takes the eigenbasis from ``eig_sweeps`` FP32 Jacobi
    sweeps (0: the library default) and works with the full rotated Gram, so
    it reaches the same dual optimum under the same acceptance bounds.
    preconditioner="eigenbasis" (default) is the reference's; "adaptive" uses
    the Hessian diagonal at the current omega, which keeps ill-conditioned
    targets converging where the reference's CG saturates.
    fp32_newton (split form): run the early Newton steps in FP32 where their
    state fits on chip (m <= 96), the last step(s) and the convergence test in
    FP64; False keeps every Newton step in FP64.
    """
    batch, n, m = _check_target(T)
    dev = N.require_cuda_f64(T)
    T = T.contiguous()
    X = torch.empty_like(T)
    omega = torch.empty(batch, m, m, dtype=torch.float64, device=dev)
    iterations = torch.empty(batch, dtype=torch.int64, device=dev)
    status = torch.empty(batch, dtype=torch.int32, device=dev)
    if batch == 0:
        return SolveResult(X, omega, iterations, status)
    lib = N.load()
    nbytes = lib.ssn_workspace_bytes(batch, n, m)
    ws = workspace(dev, nbytes)
    opt = N.options(max_newton, max_cg, max_backtrack, feas_tol, precision, eig_sweeps, preconditioner,
                    fp32_newton)
    N.check(lib.ssn_solve(T.data_ptr(), X.data_ptr(), omega.data_ptr(), iterations.data_ptr(),
                          status.data_ptr(), batch, n, m, ws.data_ptr(), nbytes,
                          N.ctypes.byref(opt), N.stream_handle(dev)), "ssn_solve")
    if raise_on_failure:
        raise_for_status(status)
    return SolveResult(X, omega, iterations, status)


@torch.no_grad()
def solve_ragged(targets, *, max_newton: int = MAX_NEWTON, max_cg: int = MAX_CG,
                 max_backtrack: int = MAX_BACKTRACK, feas_tol: float = FEAS_TOL,
                 precision: str = "fp64", eig_sweeps: int = 0, preconditioner: str = "eigenbasis",
                 fp32_newton: bool = True, raise_on_failure: bool = True):
    """Solve targets of different shapes in one call (ssn_solve_ragged).

    ``targets`` is a sequence of float64 [2n_i, 2k_i] tensors, all on the host or all
    on one CUDA device.  Returns (list of X_i, list of omega_i, iterations int64
    [count], status int32 [count]) on the targets' device.  Each instance gets the
    same result as solving it alone with ``solve``; with ``raise_on_failure`` a cap
    on any instance raises RuntimeError for the whole call, as ``solve`` does.
    """
    targets = list(targets)
    if not targets:
        raise ValueError("no targets")
    on_host = not targets[0].is_cuda
    ns, ms = [], []
    for t in targets:
        if t.dim() != 2 or t.dtype != torch.float64 or t.is_cuda == on_host:
            raise ValueError("targets must be 2-D float64 tensors, all on the host or all on one device")
        rows, m = t.shape
        if rows % 2 or m % 2 or m > 128 or rows // 2 < m // 2 or m == 0:
            raise ValueError(f"target shape {tuple(t.shape)} is not [2n, 2k] with 1 <= k <= 64, n >= k")
        ns.append(rows // 2)
        ms.append(m)
    dev = torch.device("cuda", torch.cuda.current_device()) if on_host else targets[0].device
    if on_host:
        with _host_lock:
            return _solve_ragged_call(targets, ns, ms, dev, True, max_newton, max_cg, max_backtrack, feas_tol,
                                      precision, eig_sweeps, preconditioner, fp32_newton, raise_on_failure)
    return _solve_ragged_call(targets, ns, ms, dev, False, max_newton, max_cg, max_backtrack, feas_tol,
                              precision, eig_sweeps, preconditioner, fp32_newton, raise_on_failure)


def _solve_ragged_call(targets, ns, ms, dev, on_host, max_newton, max_cg, max_backtrack, feas_tol, precision,
                       eig_sweeps, preconditioner, fp32_newton, raise_on_failure):
    if on_host:
        # pack into the package's cached pinned staging buffer (no per-call pinned
        # allocation), with the per-target copies spread over host threads; the copy up
        # then runs at the link's pinned rate
        total = sum(t.numel() for t in targets)
        staged = _staging_buffer(dev, _RAGGED_SLOT, (total,))
        offs = [0]
        for t in targets:
            offs.append(offs[-1] + t.numel())
        _parallel_copies([(staged[offs[i]:offs[i + 1]], t.reshape(-1)) for i, t in enumerate(targets)])
        flat = staged.to(dev, non_blocking=True)
    else:
        flat = torch.cat([t.reshape(-1) for t in targets])
    count = len(targets)
    t_off = [0] * count
    w_off = [0] * count
    tt = ww = 0
    for i in range(count):
        t_off[i], w_off[i] = tt, ww
        tt += 2 * ns[i] * ms[i]
        ww += ms[i] * ms[i]
    X = torch.empty_like(flat)
    omega = torch.empty(ww, dtype=torch.float64, device=dev)
    iterations = torch.empty(count, dtype=torch.int64, device=dev)
    status = torch.empty(count, dtype=torch.int32, device=dev)
    c_int = N.ctypes.c_int * count
    c_i64 = N.ctypes.c_int64 * count
    n_arr, m_arr, t_arr, w_arr = c_int(*ns), c_int(*ms), c_i64(*t_off), c_i64(*w_off)
    lib = N.load()
    nbytes = lib.ssn_ragged_workspace_bytes(count, n_arr, m_arr)
    ws = workspace(dev, nbytes)
    opt = N.options(max_newton, max_cg, max_backtrack, feas_tol, precision, eig_sweeps, preconditioner,
                    fp32_newton)
    N.check(lib.ssn_solve_ragged(flat.data_ptr(), X.data_ptr(), omega.data_ptr(), iterations.data_ptr(),
                                 status.data_ptr(), count, n_arr, m_arr, t_arr, w_arr, ws.data_ptr(), nbytes,
                                 N.ctypes.byref(opt), N.stream_handle(dev)), "ssn_solve_ragged")
    if raise_on_failure:
        raise_for_status(status)
    if on_host:
        # X comes back through the (now free) pinned staging buffer at the link's pinned rate,
        # then into one fresh host tensor per target, the caller's to keep
        staged_x = _staging_buffer(dev, _RAGGED_SLOT, (X.numel(),))
        staged_x.copy_(X, non_blocking=True)
        omega, iterations, status = omega.cpu(), iterations.cpu(), status.cpu()   # synchronises
        Xs = [torch.empty(2 * ns[i], ms[i], dtype=torch.float64) for i in range(count)]
        _parallel_copies([(Xs[i].view(-1), staged_x[t_off[i]:t_off[i] + 2 * ns[i] * ms[i]]) for i in range(count)])
    else:
        Xs = [X[t_off[i]:t_off[i] + 2 * ns[i] * ms[i]].view(2 * ns[i], ms[i]) for i in range(count)]
    Ws = [omega[w_off[i]:w_off[i] + ms[i] * ms[i]].view(ms[i], ms[i]) for i in range(count)]
    return Xs, Ws, iterations, status


_copy_pool = None
_COPY_WORKERS = min(16, os.cpu_count() or 1)


def _parallel_copies(pairs) -> None:
    """dst.copy_(src) for host tensor pairs, spread over a pool of host threads (torch
    releases the GIL in copy_), in chunks of about equal bytes."""
    global _copy_pool
    if _copy_pool is None:
        from concurrent.futures import ThreadPoolExecutor
        _copy_pool = ThreadPoolExecutor(max_workers=_COPY_WORKERS)
    workers = _COPY_WORKERS
    total = sum(d.numel() for d, _ in pairs)
    chunks, cur, size = [], [], 0
    for d, src in pairs:
        cur.append((d, src))
        size += d.numel()
        if size * workers >= total and len(chunks) < workers - 1:
            chunks.append(cur)
            cur, size = [], 0
    if cur:
        chunks.append(cur)

    def run(chunk):
        for d, src in chunk:
            d.copy_(src)
    for f in [_copy_pool.submit(run, c) for c in chunks]:
        f.result()


def raise_for_status(status: torch.Tensor) -> None:
    """Raise RuntimeError for the batch if any instance hit a cap (synchronises)."""
    codes = status.cpu().tolist()
    for code in (3, 4, 6):
        if code in codes:
            bad = [i for i, c in enumerate(codes) if c == code]
            raise RuntimeError(f"{_MESSAGES[code]} (instances {bad[:8]}{'...' if len(bad) > 8 else ''})")


@torch.no_grad()
def solve(T: torch.Tensor, **options):
    """(X, omega, iterations) for T float64 [batch, 2n, 2k] (dual_recommended_hvp.py:231-242).

    CPU input -> CPU outputs (X pinned when >= 64 MiB, like the reference);
    CUDA input -> CUDA outputs.  Raises RuntimeError for the whole batch on a
    Newton or line-search cap.
    """
    _check_target(T)
    if T.is_cuda:
        res = solve_ex(T, **options)
        raise_for_status(res.status)
        return res.X, res.omega, res.iterations
    return _solve_host(T, **options)


# ---- host-resident batches: chunked, stream-pipelined staging ------------------------------
CHUNK_BYTES = 64 * 2**20      # largest chunk of T, in bytes
N_STREAMS = 16                # chunks in flight; each solve is latency-bound, so they overlap
CHUNK_RAMP = (1, 2, 4, 8)     # leading (and mirrored trailing) chunk sizes, in targets
MIN_CHUNK_BYTES = 16 * 2**20  # smallest chunk between the ramps: per-chunk launch work stays small
RAMP_MIN_BYTES = 256 * 2**20  # ramps only for batches this large, where the copies dominate


def _chunk_plan(batch: int, cap: int, ramp=None):
    """Chunk sizes (targets) for the host pipeline.

    A chunk's solve costs about one Newton latency whatever its size, and the two
    copy directions run on separate engines.  Short chunks first let the copies
    back start while later targets are still going up; short chunks last shorten
    the tail (the last chunk's latency and its copy back).  Between the ramps the
    chunks are as even as possible and at most ``cap`` targets.
    """
    ramp = tuple(CHUNK_RAMP if ramp is None else ramp)
    if not ramp or batch < 2 * sum(ramp) + 1:
        n = -(-batch // cap)
        return [batch // n + (1 if i < batch % n else 0) for i in range(n)]
    middle = batch - 2 * sum(ramp)
    n = -(-middle // cap)
    mid = [middle // n + (1 if i < middle % n else 0) for i in range(n)]
    return list(ramp) + mid + list(reversed(ramp))


_streams = {}
_staging = {}
# The stream pool and the pinned staging buffers are shared per device, so host-path
# solves from several Python threads take turns (device-resident solves do not lock).
_host_lock = threading.Lock()


def _stream_pool(dev: torch.device):
    key = dev.index
    if key not in _streams:
        _streams[key] = [torch.cuda.Stream(dev) for _ in range(N_STREAMS)]
    return _streams[key]


_RAGGED_SLOT = 1 << 20          # staging slot of the ragged host path (the chunked path uses 0 ..)


def _staging_buffer(dev: torch.device, slot: int, shape) -> torch.Tensor:
    key = (dev.index, slot)
    numel = 1
    for d in shape:
        numel *= d
    buf = _staging.get(key)
    if buf is None or buf.numel() < numel:
        buf = torch.empty(numel, dtype=torch.float64, pin_memory=True)
        _staging[key] = buf
    return buf[:numel].view(shape)


def _solve_host(T: torch.Tensor, **options):
    with _host_lock:
        return _solve_host_locked(T, **options)


def _solve_host_locked(T: torch.Tensor, **options):
    """CPU-in/CPU-out solve with the batch split into chunks on a pool of streams.

    Each chunk's H2D copy, solve and D2H copy are enqueued on one stream, so
    the copies of one chunk overlap the solves of others and the two copy
    directions overlap each other.  A pageable T is staged through pinned
    per-stream buffers, like the reference's pinned 1024-row staging
    (dual_recommended_hvp.py:86-91, :204-226).
    """
    batch, n, m = _check_target(T)
    dev = torch.device("cuda", torch.cuda.current_device())
    X = _pinned_like(T)
    per = max(1, T[0].numel() * 8)
    cap = max(1, min(batch, CHUNK_BYTES // per, max(-(-batch // N_STREAMS), MIN_CHUNK_BYTES // per)))
    sizes = _chunk_plan(batch, cap, None if batch * per >= RAMP_MIN_BYTES else ())
    pinned_in, pinned_out = T.is_pinned(), X.is_pinned()
    streams = _stream_pool(dev)
    main = torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(main)
    results, done = [], []
    c1 = 0
    for idx, size in enumerate(sizes):
        c0, c1 = c1, c1 + size
        slot = idx % len(streams)
        s = streams[slot]
        s.wait_event(ready)
        with torch.cuda.stream(s):
            if pinned_in:
                src = T[c0:c1]
            else:
                if idx >= len(streams):        # the staging buffer's previous copy must be done
                    done[idx - len(streams)][0].synchronize()
                src = _staging_buffer(dev, slot, (c1 - c0, 2 * n, m))
                src.copy_(T[c0:c1])
            Td = torch.empty((c1 - c0, 2 * n, m), dtype=torch.float64, device=dev)
            Td.copy_(src, non_blocking=True)
            h2d = torch.cuda.Event()
            h2d.record(s)
            res = solve_ex(Td, **options)
            X[c0:c1].copy_(res.X, non_blocking=pinned_out)
            results.append(res)
            done.append((h2d, s))
    for s in streams:
        s.synchronize()
    status = torch.cat([r.status for r in results])
    raise_for_status(status)
    omega = torch.cat([r.omega for r in results]).cpu()
    iterations = torch.cat([r.iterations for r in results]).cpu()
    return X, omega, iterations


# ---- lower-level pieces of the reference module -------------------------------------------
@torch.no_grad()
def gram_chunks(T, blocks=None):
    """(Cr, Ci) on the device for T [batch, 2n, m] (dual_recommended_hvp.py:79-96).

    The whole batch is copied once (no 1024-row staging); if ``blocks`` is a
    list, the device copies of (A, D) are appended to it for recover_matmul.
    """
    from .gram_triangle_reflect import gram
    batch, n, m = _check_target(T)
    Td = T if T.is_cuda else T.to(DEVICE)
    A, D = Td[:, :n], Td[:, n:]
    if blocks is not None:
        blocks.append((A, D))
    return gram(A, D)


@torch.no_grad()
def eigh_scaled(Cr, precision="fp64", eig_sweeps=0):
    """(values, vectors, scale, sweeps) with Cr/scale = V diag(values) V^T, scale = max(1, tr(Cr)/m).

    Device Jacobi replacing torch.linalg.eigh at dual_recommended_hvp.py:106-108.
    precision="split" returns the rough basis of the split-precision form
    (``eig_sweeps`` FP32 sweeps; V only approximately diagonalises Cr/scale).
    """
    dev = N.require_cuda_f64(Cr)
    batch, m, _ = Cr.shape
    Cr = Cr.contiguous()
    values = torch.empty(batch, m, dtype=torch.float64, device=dev)
    vectors = torch.empty(batch, m, m, dtype=torch.float64, device=dev)
    scale = torch.empty(batch, dtype=torch.float64, device=dev)
    sweeps = torch.empty(batch, dtype=torch.int32, device=dev)
    lib = N.load()
    nbytes = lib.ssn_eigh_workspace_bytes(batch, m)
    ws = workspace(dev, nbytes)
    opt = N.options(precision=precision, eig_sweeps=eig_sweeps)
    N.check(lib.ssn_eigh(Cr.data_ptr(), values.data_ptr(), vectors.data_ptr(), scale.data_ptr(),
                         sweeps.data_ptr(), batch, m, ws.data_ptr(), nbytes, N.ctypes.byref(opt),
                         N.stream_handle(dev)), "ssn_eigh")
    return values, vectors, scale, sweeps


@torch.no_grad()
def dual_batch(Cr, Ci, final=None, **options):
    """(omega, L, iterations) from device Gram matrices (dual_recommended_hvp.py:99-191).

    If ``final`` is a list it receives (P, Q), the cached inverse parts in the
    original basis, like the reference.  L = chol(I + omega omega) is formed
    by this package's Cholesky kernel to keep the reference's return value; the
    solve path does not use it.
    """
    dev = N.require_cuda_f64(Cr, Ci)
    batch, m, _ = Cr.shape
    Cr, Ci = Cr.contiguous(), Ci.contiguous()
    omega = torch.empty(batch, m, m, dtype=torch.float64, device=dev)
    P, Q = torch.empty_like(omega), torch.empty_like(omega)
    iterations = torch.empty(batch, dtype=torch.int64, device=dev)
    status = torch.empty(batch, dtype=torch.int32, device=dev)
    lib = N.load()
    nbytes = lib.ssn_dual_workspace_bytes(batch, m)
    ws = workspace(dev, nbytes)
    opt = N.options(options.get("max_newton", MAX_NEWTON), options.get("max_cg", MAX_CG),
                    options.get("max_backtrack", MAX_BACKTRACK), options.get("feas_tol", FEAS_TOL),
                    options.get("precision", "fp64"), options.get("eig_sweeps", 0),
                    options.get("preconditioner", "eigenbasis"), options.get("fp32_newton", True))
    N.check(lib.ssn_dual(Cr.data_ptr(), Ci.data_ptr(), omega.data_ptr(), P.data_ptr(), Q.data_ptr(),
                         iterations.data_ptr(), status.data_ptr(), batch, m, ws.data_ptr(), nbytes,
                         N.ctypes.byref(opt), N.stream_handle(dev)), "ssn_dual")
    raise_for_status(status)
    if final is not None:
        final[:] = (P, Q)
    L, info = cholesky_k(omega)
    if bool((info != 0).any()):
        raise torch.linalg.LinAlgError("dual_batch: I + omega omega is not positive definite")
    return omega, L, iterations


@torch.no_grad()
def recover_matmul(T, omega, L, blocks=None, final=None):
    """X for T using the cached (P, Q) in ``final`` (dual_recommended_hvp.py:194-228)."""
    from .recovery_fused import recover_block
    batch, n, m = _check_target(T)
    if not final:
        raise ValueError("final=(P, Q) from dual_batch is required")
    P, Q = final
    if blocks:
        A, D = blocks[0]
    else:
        Td = T if T.is_cuda else T.to(P.device)
        A, D = Td[:, :n], Td[:, n:]
    Ur, Ui = recover_block(A, D, P, Q)
    X = torch.cat((Ur, Ui), dim=1)
    return X if T.is_cuda else X.cpu()
