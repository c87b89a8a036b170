"""Gradient through the solve (ssn_adjoint) against three CPU routes.

The reference has no backward pass, so the checks are: the dense KKT solve of
the primal problem (independent of the dual formulation), central finite
differences of L(T) through the CPU solve (step 1e-6; the north-star bound is
1e-6 relative), and the closed-form dual adjoint restated on the CPU with a
dense Hessian solve (for sizes where the KKT system is too large).
"""
from __future__ import annotations

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b).clamp_min(1e-300))


@pytest.fixture(scope="module")
def sp():
    import symplectic_projection as sp
    sp.initialize_kernels()
    return sp


def _grads(shape, m, seed):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, dtype=torch.float64, generator=g),
            torch.randn(shape[0], m, m, dtype=torch.float64, generator=g))


def _device_grad(T, G, Gw=None, precision="fp64"):
    from symplectic_projection.adjoint import solve_backward
    from symplectic_projection.dual_recommended_hvp import solve_ex
    res = solve_ex(T.cuda(), precision=precision)
    assert res.status.cpu().tolist() == [0] * T.shape[0]
    dT, st, it = solve_backward(T.cuda(), res.omega, G.cuda() if G is not None else None,
                                Gw.cuda() if Gw is not None else None, precision=precision)
    assert st.cpu().tolist() == [0] * T.shape[0]
    return dT.cpu(), it.cpu()


def test_adjoint_matches_dense_kkt_and_finite_differences(sp):
    # the differentiation check size: 8 targets, n = 32, k = 4
    T, _ = O.make_inputs(32, 4, 0, 8)
    G, _ = _grads(T.shape, 8, 11)
    dT, it = _device_grad(T, G)
    kkt = O.adjoint_kkt(T, G)
    for b in range(8):
        assert rel(dT[b], kkt[b]) < 1e-8, b
    fd, V = O.adjoint_fd(T, G, h=1e-6, seed=5)
    ad = (dT * V).sum(dim=(-2, -1))
    assert float(((ad - fd).abs() / fd.abs()).max()) < 1e-6
    assert int(it.max()) < 80


def test_adjoint_with_omega_gradient(sp):
    T, _ = O.make_inputs(40, 6, 1, 4)
    G, Gw = _grads(T.shape, 12, 12)
    dT, _ = _device_grad(T, G, Gw)
    ref = O.adjoint_formula(T, G, Gw)
    assert rel(dT, ref) < 1e-9
    fd, V = O.adjoint_fd(T, G, Gw, h=1e-6, seed=6)
    ad = (dT * V).sum(dim=(-2, -1))
    assert float(((ad - fd).abs() / fd.abs()).max()) < 1e-6
    # omega gradient alone (no grad_X)
    dT0, _ = _device_grad(T, None, Gw)
    assert rel(dT0, O.adjoint_formula(T, torch.zeros_like(T), Gw)) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("n,k,count", [(2048, 32, 4), (256, 64, 2), (100, 1, 3)])
def test_adjoint_against_dual_closed_form(sp, n, k, count, precision):
    """The differentiation workload's shape (n = 2048, k = 32) and the size extremes, both forms.
    The split form differentiates at its own omega, which is within a few 1e-9 of the FP64
    oracle's (its INT8 Gram and recoveries are accurate to about 1e-13), hence 1e-8 there."""
    T, _ = O.make_inputs(n, k, 0, count)
    G, _ = _grads(T.shape, 2 * k, n + k)
    dT, _ = _device_grad(T, G, precision=precision)
    assert rel(dT, O.adjoint_formula(T, G)) < (1e-9 if precision == "fp64" else 1e-8)


def test_autograd_function(sp):
    from symplectic_projection.adjoint import project, solve_backward
    T, _ = O.make_inputs(64, 8, 2, 3)
    G, Gw = _grads(T.shape, 16, 13)
    Td = T.cuda().requires_grad_(True)
    X, W = project(Td)
    loss = (X * G.cuda()).sum() + (W * Gw.cuda()).sum()
    loss.backward()
    ref, _, _ = solve_backward(T.cuda(), W.detach(), G.cuda(), Gw.cuda())
    assert torch.equal(Td.grad, ref)
    assert rel(Td.grad, O.adjoint_formula(T, G, Gw)) < 1e-9


def test_adjoint_rejects_an_infeasible_multiplier(sp):
    from symplectic_projection.adjoint import solve_backward
    T, _ = O.make_inputs(32, 2, 0, 2)
    W = torch.zeros(2, 4, 4, dtype=torch.float64)
    W[1, 0, 1], W[1, 1, 0] = 2.0, -2.0              # ||omega|| > 1: I + omega^2 is indefinite
    dT, st, _ = solve_backward(T.cuda(), W.cuda(), torch.ones_like(T).cuda(), raise_on_failure=False)
    assert st.cpu().tolist() == [0, 5]
    assert bool(torch.isfinite(dT[0]).all()) and not bool(torch.isfinite(dT[1]).all())
