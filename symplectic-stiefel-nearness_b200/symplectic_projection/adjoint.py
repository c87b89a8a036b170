"""Gradient through the solve, and a torch.autograd.Function around it.

The reference solves under torch.no_grad (dual_recommended_hvp.py:231) and has
no backward pass.  ``solve_backward`` calls ``ssn_adjoint``: implicit
differentiation of the dual optimality condition Im(K C K) = J_m at the
converged omega (K = (I + i omega)^-1, C = b^H b, b = A + iD), which costs one
preconditioned CG solve with the solver's Hessian-vector product per instance
and four tall-skinny FP64 products (a cross Gram and two recoveries).  X is
recomputed from K, never stored for the backward pass.
"""
from __future__ import annotations

import torch

from . import _native as N
from ._workspace import workspace
from .dual_recommended_hvp import _check_target, raise_for_status, solve_ex

_MESSAGES = {3: "adjoint CG reached its iteration cap", 5: "adjoint: non-finite input or I + omega^2 not positive definite"}


@torch.no_grad()
def solve_backward(T: torch.Tensor, omega: torch.Tensor, grad_X: torch.Tensor | None = None,
                   grad_omega: torch.Tensor | None = None, *, precision: str = "fp64", max_cg: int = 0,
                   raise_on_failure: bool = True):
    """(dL/dT, status, cg_iterations) for L with dL/dX = grad_X and dL/d omega = grad_omega.

    T [batch, 2n, 2k] and omega [batch, 2k, 2k] (the solve's multiplier) are CUDA
    float64 tensors; either gradient may be None (treated as zero).  precision="split"
    runs the Gram of T and the two recovery products as INT8 Ozaki products on the
    tensor cores; the Hessian solve is FP64 in both forms.
    """
    batch, n, m = _check_target(T)
    dev = N.require_cuda_f64(T, omega)
    T, omega = T.contiguous(), omega.contiguous()
    if grad_X is not None:
        N.require_cuda_f64(grad_X)
        grad_X = grad_X.contiguous()
        if grad_X.shape != T.shape:
            raise ValueError("grad_X must have the shape of T")
    if grad_omega is not None:
        N.require_cuda_f64(grad_omega)
        grad_omega = grad_omega.contiguous()
        if grad_omega.shape != omega.shape:
            raise ValueError("grad_omega must have the shape of omega")
    dT = torch.empty_like(T)
    status = torch.empty(batch, dtype=torch.int32, device=dev)
    iters = torch.empty(batch, dtype=torch.int32, device=dev)
    lib = N.load()
    nbytes = lib.ssn_adjoint_workspace_bytes(batch, n, m)
    ws = workspace(dev, nbytes)
    opt = N.options(max_cg=max(1, max_cg), precision=precision) if max_cg else N.options(precision=precision)
    N.check(lib.ssn_adjoint(T.data_ptr(), omega.data_ptr(), N.ptr(grad_X), N.ptr(grad_omega), dT.data_ptr(),
                            status.data_ptr(), iters.data_ptr(), batch, n, m, ws.data_ptr(), nbytes,
                            N.ctypes.byref(opt) if opt is not None else None, N.stream_handle(dev)), "ssn_adjoint")
    if raise_on_failure:
        codes = status.cpu().tolist()
        for code, msg in _MESSAGES.items():
            if code in codes:
                raise RuntimeError(f"{msg} (instances {[i for i, c in enumerate(codes) if c == code][:8]})")
    return dT, status, iters


class SymplecticProjection(torch.autograd.Function):
    """(X, omega) = solve(T) with a backward pass through ``ssn_adjoint``."""

    @staticmethod
    def forward(ctx, T, options):
        res = solve_ex(T, **options)
        raise_for_status(res.status)
        ctx.save_for_backward(T, res.omega)
        ctx.precision = options.get("precision", "fp64")
        return res.X, res.omega

    @staticmethod
    def backward(ctx, grad_X, grad_omega):
        T, omega = ctx.saved_tensors
        dT, _, _ = solve_backward(T, omega, grad_X, grad_omega, precision=ctx.precision)
        return dT, None


def project(T: torch.Tensor, **options):
    """Differentiable (X, omega) for a CUDA float64 T [batch, 2n, 2k]; ``options`` as for solve_ex."""
    return SymplecticProjection.apply(T, options)
