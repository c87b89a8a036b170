"""Primal recovery products (recovery_fused.py:19-30)."""
import torch

from . import _native as N


def initialize_kernels():
    N.load()


@torch.no_grad()
def recover_block(A, D, P, Q):
    """Ur = A P^T + D Q^T, Ui = D P^T - A Q^T; A, D [batch, rows, m], P, Q [batch, m, m]."""
    dev = N.require_cuda_f64(A, D, P, Q)
    batch, rows, m = A.shape
    if D.shape != A.shape or P.shape != (batch, m, m) or Q.shape != (batch, m, m):
        raise ValueError("shape mismatch")
    A, D, P, Q = (x.contiguous() for x in (A, D, P, Q))
    Ur, Ui = torch.empty_like(A), torch.empty_like(A)
    N.check(N.load().ssn_recover(A.data_ptr(), D.data_ptr(), rows * m, P.data_ptr(), Q.data_ptr(),
                                 Ur.data_ptr(), Ui.data_ptr(), rows * m, batch, rows, m,
                                 N.stream_handle(dev)), "ssn_recover")
    return Ur, Ui
