"""Primal recovery products (recovery_fused.py:19-30)."""
import torch

from . import _native as N
from ._workspace import workspace


def initialize_kernels():
    N.load()


@torch.no_grad()
def recover_block(A, D, P, Q, precision="fp64"):
    """Ur = A P^T + D Q^T, Ui = D P^T - A Q^T; A, D [batch, rows, m], P, Q [batch, m, m].

    precision="split": INT8 Ozaki tensor-core products (six balanced digits per
    row, exact INT32 accumulation); "fp64": FP64 tensor-core products.
    """
    dev = N.require_cuda_f64(A, D, P, Q)
    batch, rows, m = A.shape
    if D.shape != A.shape or P.shape != (batch, m, m) or Q.shape != (batch, m, m):
        raise ValueError("shape mismatch")
    A, D, ab_stride = N.row_halves(A, D)
    P, Q = P.contiguous(), Q.contiguous()
    Ur = torch.empty(batch, rows, m, dtype=torch.float64, device=dev)
    Ui = torch.empty_like(Ur)
    lib = N.load()
    nbytes = lib.ssn_recover_workspace_bytes(batch, rows, m)
    ws = workspace(dev, nbytes)
    opt = N.options(precision=precision)
    N.check(lib.ssn_recover(A.data_ptr(), D.data_ptr(), ab_stride, P.data_ptr(), Q.data_ptr(),
                            Ur.data_ptr(), Ui.data_ptr(), rows * m, batch, rows, m, ws.data_ptr(), nbytes,
                            N.ctypes.byref(opt), N.stream_handle(dev)), "ssn_recover")
    return Ur, Ui
