"""ssn_gram_noalloc: the Gram products for callers that cannot allocate device memory.

Some callers cannot hand this library a workspace: a host framework whose
pooling allocator owns the whole device and will not give raw buffers to
foreign code, or a latency-critical caller that must never reach cudaMalloc
(which can synchronise the device and can fail under memory pressure).  The
entry point keeps its scratch in one fixed array inside the library instead.
These tests call it through the C ABI and compare it with ssn_gram, which uses
a caller workspace, on two calls in a row of different shapes (the shared
scratch keeps the previous call's contents), and with the CPU oracle's Gram of
the same targets; the A and D views are the two halves of each target, batch
stride 2nm, the layout the solver passes.  A call too large for the fixed
scratch must be rejected before anything runs.
"""
from __future__ import annotations

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu

SSN_ERR_SCRATCH_LIMIT = 8


def _gram_with_workspace(lib, N, A, D, stride):
    batch, rows, m = A.shape
    Cr = torch.empty(batch, m, m, dtype=torch.float64, device="cuda")
    Ci = torch.empty_like(Cr)
    nbytes = lib.ssn_gram_workspace_bytes(batch, rows, m)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    N.check(lib.ssn_gram(A.data_ptr(), D.data_ptr(), stride, Cr.data_ptr(), Ci.data_ptr(),
                         batch, rows, m, ws.data_ptr(), nbytes, None, N.stream_handle(A.device)), "ssn_gram")
    return Cr, Ci


def _gram_noalloc(lib, N, A, D, stride):
    batch, rows, m = A.shape
    Cr = torch.empty(batch, m, m, dtype=torch.float64, device="cuda")
    Ci = torch.empty_like(Cr)
    rc = lib.ssn_gram_noalloc(A.data_ptr(), D.data_ptr(), stride, Cr.data_ptr(), Ci.data_ptr(),
                              batch, rows, m, N.stream_handle(A.device))
    return rc, Cr, Ci


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_noalloc_gram_matches_workspace_gram_twice():
    from symplectic_projection import _native as N
    lib = N.load()
    assert lib.ssn_gram_noalloc_scratch_bytes() == 16 << 20
    # two calls in a row with different shapes: the second must not see the first's scratch
    for (n, k, batch, case) in [(300, 12, 5, 0), (2048, 48, 6, 1)]:
        T, _ = O.make_inputs(n, k, case, batch)
        Td = T.cuda()
        A, D = Td[:, :n], Td[:, n:]                  # halves of each target: batch stride 2 n m
        stride = 2 * n * 2 * k
        assert A.stride(0) == stride
        rc, Cr, Ci = _gram_noalloc(lib, N, A, D, stride)
        assert rc == 0
        Cr_ws, Ci_ws = _gram_with_workspace(lib, N, A, D, stride)
        torch.cuda.synchronize()
        assert _rel(Cr, Cr_ws) < 1e-13 and _rel(Ci, Ci_ws) < 1e-13
        assert torch.equal(Cr, Cr.mT) and torch.equal(Ci, -Ci.mT)
        Cr_o, Ci_o = O.gram(T)                       # the oracle's Gram of the same targets
        assert _rel(Cr.cpu(), Cr_o) < 1e-13 and _rel(Ci.cpu(), Ci_o) < 1e-13


def test_noalloc_gram_rejects_sizes_beyond_its_scratch():
    from symplectic_projection import _native as N
    lib = N.load()
    m, rows = 128, 64
    batch = (16 << 20) // (8 * 2 * m * m) + 1          # one instance more than fits
    A = torch.zeros(batch, rows, m, dtype=torch.float64, device="cuda")
    rc, _, _ = _gram_noalloc(lib, N, A, A, rows * m)
    assert rc == SSN_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.ssn_status_string(rc)
