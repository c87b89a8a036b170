"""Newton-CG building blocks as stand-alone device operations.

Mirrors the wrappers of src/symplectic_projection/hvp_fused.py (same names,
argument meaning and outputs).  Inputs may be non-contiguous; outputs are new
contiguous CUDA float64 tensors.  The persistent solver runs the same
arithmetic fused in one kernel; these exist for composition and parity tests.
"""
import torch

from . import _native as N


def initialize_kernels():
    N.load()


def _mats(*xs):
    dev = N.require_cuda_f64(*xs)
    first = xs[0]
    if first.ndim != 3 or first.shape[-1] != first.shape[-2]:
        raise ValueError("expected [batch, m, m] matrices")
    if any(x.shape != first.shape for x in xs):
        raise ValueError("shape mismatch")
    return dev, first.shape[0], first.shape[-1], [x.contiguous() for x in xs]


@torch.no_grad()
def inner_products(E, Sr, Si):
    """U = E@Sr, V = E@Si (hvp_fused.py:22-34)."""
    dev, b, m, (E, Sr, Si) = _mats(E, Sr, Si)
    U, V = torch.empty_like(E), torch.empty_like(E)
    N.check(N.load().ssn_inner_products(E.data_ptr(), Sr.data_ptr(), Si.data_ptr(), U.data_ptr(),
                                        V.data_ptr(), b, m, N.stream_handle(dev)), "ssn_inner_products")
    return U, V


@torch.no_grad()
def outer_skew(P, Q, U, V):
    """Z - Z.T with Z = P@U - Q@V (hvp_fused.py:37-53)."""
    dev, b, m, (P, Q, U, V) = _mats(P, Q, U, V)
    H = torch.empty_like(P)
    N.check(N.load().ssn_outer_skew(P.data_ptr(), Q.data_ptr(), U.data_ptr(), V.data_ptr(),
                                    H.data_ptr(), b, m, N.stream_handle(dev)), "ssn_outer_skew")
    return H


@torch.no_grad()
def sandwich_front(values, Ci, P, Q):
    """P*values - Q@Ci, P@Ci + Q*values (hvp_fused.py:56-69)."""
    dev, b, m, (Ci, P, Q) = _mats(Ci, P, Q)
    if values.shape != (b, m):
        raise ValueError("values must be [batch, m]")
    values = values.to(device=dev, dtype=torch.float64).contiguous()
    Yr, Yi = torch.empty_like(P), torch.empty_like(P)
    N.check(N.load().ssn_sandwich_front(values.data_ptr(), Ci.data_ptr(), P.data_ptr(), Q.data_ptr(),
                                        Yr.data_ptr(), Yi.data_ptr(), b, m, N.stream_handle(dev)),
            "ssn_sandwich_front")
    return Yr, Yi


@torch.no_grad()
def line_change(gradient, delta, V, delta_Sr, trial, delta_Si):
    """Per-instance <gradient, delta> + <V, delta_Sr + trial@delta_Si> (hvp_fused.py:72-87)."""
    dev, b, m, xs = _mats(gradient, delta, V, delta_Sr, trial, delta_Si)
    out = torch.empty(b, dtype=torch.float64, device=dev)
    N.check(N.load().ssn_line_change(*[x.data_ptr() for x in xs], out.data_ptr(), b, m,
                                     N.stream_handle(dev)), "ssn_line_change")
    return out


@torch.no_grad()
def fused_precondition(R, denominator):
    """skew(R / denominator), reading both positions (hvp_fused.py:110-117)."""
    dev, b, m, (R, den) = _mats(R, denominator)
    out = torch.empty_like(R)
    N.check(N.load().ssn_precondition(R.data_ptr(), den.data_ptr(), out.data_ptr(), b, m,
                                      N.stream_handle(dev)), "ssn_precondition")
    return out


@torch.no_grad()
def cg_update(direction, r, p, Hp, alpha):
    """(direction + alpha p, r - alpha Hp), separately rounded (hvp_fused.py:120-130)."""
    dev, b, m, (d, r, p, Hp) = _mats(direction, r, p, Hp)
    if alpha.shape != (b,) or alpha.dtype != torch.float64:
        raise ValueError("alpha must be float64 [batch]")
    alpha = alpha.to(dev).contiguous()
    nd, nr = torch.empty_like(d), torch.empty_like(d)
    N.check(N.load().ssn_cg_update(d.data_ptr(), r.data_ptr(), p.data_ptr(), Hp.data_ptr(),
                                   alpha.data_ptr(), nd.data_ptr(), nr.data_ptr(), b, m,
                                   N.stream_handle(dev)), "ssn_cg_update")
    return nd, nr


@torch.no_grad()
def cg_next(z, p, beta, cg_active):
    """where(cg_active, z + beta p, 0) (hvp_fused.py:133-143)."""
    dev, b, m, (z, p) = _mats(z, p)
    if beta.shape != (b,) or cg_active.shape != (b,) or cg_active.dtype != torch.bool:
        raise ValueError("beta must be float64 [batch] and cg_active bool [batch]")
    beta = beta.to(dev).contiguous()
    active = cg_active.to(dev).to(torch.uint8).contiguous()
    out = torch.empty_like(z)
    N.check(N.load().ssn_cg_next(z.data_ptr(), p.data_ptr(), beta.data_ptr(), active.data_ptr(),
                                 out.data_ptr(), b, m, N.stream_handle(dev)), "ssn_cg_next")
    return out
