"""Inverse from a Cholesky factor (cholesky_inverse_kernel.py:27-39), any m <= 128."""
import torch

from . import _native as N


def initialize_kernels():
    N.load()


@torch.no_grad()
def inverse_from_cholesky(L):
    """Return (L L^T)^-1 for a CUDA float64 [batch, m, m] lower Cholesky factor."""
    if L.ndim != 3 or L.shape[-1] != L.shape[-2] or not L.is_cuda or L.dtype != torch.float64:
        raise ValueError("expected a CUDA float64 tensor of shape [batch, m, m]")
    batch, m, _ = L.shape
    P = torch.empty(L.shape, dtype=L.dtype, device=L.device)
    if batch == 0:
        return P
    L = L.contiguous()
    N.check(N.load().ssn_inverse_from_cholesky(L.data_ptr(), P.data_ptr(), batch, m,
                                               N.stream_handle(L.device)), "ssn_inverse_from_cholesky")
    return P


@torch.no_grad()
def spd_inverse(K):
    """(K^-1, info) for SPD K [batch, m, m]; info[b] == 0 iff every pivot was positive."""
    dev = N.require_cuda_f64(K)
    batch, m, _ = K.shape
    K = K.contiguous()
    P = torch.empty_like(K)
    info = torch.empty(batch, dtype=torch.int32, device=dev)
    N.check(N.load().ssn_spd_inverse(K.data_ptr(), P.data_ptr(), info.data_ptr(), batch, m,
                                     N.stream_handle(dev)), "ssn_spd_inverse")
    return P, info


@torch.no_grad()
def cholesky_k(omega):
    """(L, info): L = chol(I + omega omega) for skew omega [batch, m, m] (dual_recommended_hvp.py:63).

    info[b] == 0 iff I + omega omega is positive definite (else the 1-based
    order of the first leading minor that is not).
    """
    dev = N.require_cuda_f64(omega)
    batch, m, _ = omega.shape
    omega = omega.contiguous()
    L = torch.empty_like(omega)
    info = torch.empty(batch, dtype=torch.int32, device=dev)
    N.check(N.load().ssn_cholesky_k(omega.data_ptr(), L.data_ptr(), info.data_ptr(), batch, m,
                                    N.stream_handle(dev)), "ssn_cholesky_k")
    return L, info
