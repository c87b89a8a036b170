"""B200 (sm_100a) batched solver for the nearest real symplectic Stiefel matrix.

Drop-in for the reference package of the same name
(yulinxie20/symplectic-stiefel-nearness, ``src/symplectic_projection/__init__.py``):

    initialize_kernels()            # idempotent; loads the native library
    X, omega, iterations = solve(T) # T: float64 [batch, 2n, 2k]

``solve`` accepts CPU tensors (returns CPU tensors, like the reference) or CUDA
tensors (returns CUDA tensors, device-resident).  All compute runs in
hand-written sm_100a kernels behind the C ABI of ``include/ssn.h``; there is
no CPU fallback.
"""
from . import cholesky_inverse_kernel, gram_triangle_reflect, hvp_fused, recovery_fused
from ._native import load as _load
from .dual_recommended_hvp import solve, solve_ex, solve_ragged

__all__ = ["initialize_kernels", "solve", "solve_ex", "solve_ragged"]

_initialized = False


def initialize_kernels():
    """Load libssn.so once per process (src/symplectic_projection/__init__.py:10-19)."""
    global _initialized
    if _initialized:
        return
    _load()
    for mod in (gram_triangle_reflect, hvp_fused, recovery_fused, cholesky_inverse_kernel):
        mod.initialize_kernels()
    _initialized = True
