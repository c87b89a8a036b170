"""The INT8 tensor-core building block of the split-precision form, checked bit for bit.

ssn_probe_s8_mma runs one tcgen05.mma kind::i8 chain from K-major shared-memory
operands into a TMEM accumulator and reads it back with tcgen05.ld.  Integer
products are exact, so the result must equal the int64 matmul exactly, for
every shape class the Ozaki kernels use (N from 16 to 256, K from 32 to 256)
and for the full int8 range including -128.
"""
from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k", [(16, 32), (64, 64), (96, 128), (112, 96), (192, 256), (256, 256)])
def test_s8_mma_is_exact(n, k):
    from symplectic_projection import _native as N
    lib = N.load()
    g = torch.Generator().manual_seed(1000 * n + k)
    A = torch.randint(-128, 128, (128, k), generator=g, dtype=torch.int8)
    B = torch.randint(-128, 128, (n, k), generator=g, dtype=torch.int8)
    Ad, Bd = A.cuda(), B.cuda()
    C = torch.full((128, n), -7, dtype=torch.int32, device="cuda")
    stall = torch.zeros(1, dtype=torch.int32, device="cuda")
    N.check(lib.ssn_probe_s8_mma(Ad.data_ptr(), Bd.data_ptr(), C.data_ptr(), n, k, stall.data_ptr(),
                                 N.stream_handle(Ad.device)), "ssn_probe_s8_mma")
    torch.cuda.synchronize()
    assert int(stall.item()) == 0
    ref = A.to(torch.int64) @ B.to(torch.int64).T
    assert torch.equal(C.cpu().to(torch.int64), ref)


def test_s8_mma_rejects_bad_shapes():
    from symplectic_projection import _native as N
    lib = N.load()
    buf = torch.zeros(128 * 256, dtype=torch.int8, device="cuda")
    out = torch.zeros(128 * 256, dtype=torch.int32, device="cuda")
    stall = torch.zeros(1, dtype=torch.int32, device="cuda")
    for n, k in [(8, 32), (24, 32), (272, 32), (64, 16), (64, 48), (64, 288)]:
        rc = lib.ssn_probe_s8_mma(buf.data_ptr(), buf.data_ptr(), out.data_ptr(), n, k, stall.data_ptr(),
                                  N.stream_handle(buf.device))
        assert rc == 1, (n, k)
