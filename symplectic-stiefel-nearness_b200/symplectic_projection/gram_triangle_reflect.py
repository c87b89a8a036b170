"""Gram products of the stacked halves of T (gram_triangle_reflect.py:19-36)."""
import torch

from . import _native as N
from ._workspace import workspace


def initialize_kernels():
    N.load()


@torch.no_grad()
def gram(A, D, precision="fp64"):
    """Return (Cr, Ci) = (A^T A + D^T D, A^T D - D^T A) for CUDA float64 [batch, rows, m].

    precision="split" uses the INT8 Ozaki tensor-core products (about 1e-12
    relative to max|T|^2 per entry); "fp64" the FP64 tensor-core products.
    """
    dev = N.require_cuda_f64(A, D)
    batch, rows, m = A.shape
    if D.shape != A.shape:
        raise ValueError("A and D must have the same shape")
    A, D, stride = N.row_halves(A, D)
    Cr = torch.empty(batch, m, m, dtype=torch.float64, device=dev)
    Ci = torch.empty_like(Cr)
    lib = N.load()
    nbytes = lib.ssn_gram_workspace_bytes(batch, rows, m)
    ws = workspace(dev, nbytes)
    opt = N.options(precision=precision)
    N.check(lib.ssn_gram(A.data_ptr(), D.data_ptr(), stride, Cr.data_ptr(), Ci.data_ptr(),
                         batch, rows, m, ws.data_ptr(), nbytes, N.ctypes.byref(opt), N.stream_handle(dev)),
            "ssn_gram")
    return Cr, Ci


@torch.no_grad()
def cross_gram(Ga, Gd, A, D):
    """Return (Mr, Mi) = (Ga^T A + Gd^T D, Ga^T D - Gd^T A), FP64 tensor-core products.

    All four operands are CUDA float64 [batch, rows, m]; the halves of one
    stacked [batch, 2 rows, m] tensor pass without a copy.
    """
    dev = N.require_cuda_f64(Ga, Gd, A, D)
    batch, rows, m = A.shape
    if Ga.shape != A.shape or Gd.shape != A.shape or D.shape != A.shape:
        raise ValueError("all operands must have the same shape")
    Ga, Gd, g_stride = N.row_halves(Ga, Gd)
    A, D, ab_stride = N.row_halves(A, D)
    Mr = torch.empty(batch, m, m, dtype=torch.float64, device=dev)
    Mi = torch.empty_like(Mr)
    lib = N.load()
    nbytes = lib.ssn_cross_gram_workspace_bytes(batch, rows, m)
    ws = workspace(dev, nbytes)
    N.check(lib.ssn_cross_gram(Ga.data_ptr(), Gd.data_ptr(), g_stride, A.data_ptr(), D.data_ptr(), ab_stride,
                               Mr.data_ptr(), Mi.data_ptr(), batch, rows, m, ws.data_ptr(), nbytes,
                               N.stream_handle(dev)), "ssn_cross_gram")
    return Mr, Mi


@torch.no_grad()
def gram_add_(A, D, Cr, Ci, split_diagonal=True):
    """Cr += A.T@A + D.T@D; Ci += A.T@D - D.T@A (inputs and outputs must not alias)."""
    batch, rows, m = A.shape
    if D.shape != A.shape or Cr.shape != (batch, m, m) or Ci.shape != (batch, m, m):
        raise ValueError("shape mismatch")
    N.require_cuda_f64(A, D, Cr, Ci)
    cr, ci = gram(A, D)
    Cr.add_(cr)
    Ci.add_(ci)
