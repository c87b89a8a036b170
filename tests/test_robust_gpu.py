"""Ill-conditioned targets: the adaptive preconditioner on the device.

Targets T = U diag(s) V^T with s log-uniform in [1e-2, 1e2] make the reference's
dual Newton-CG stall: its eigenbasis preconditioner is exact only at omega = 0,
CG saturates and the Newton cap is reached.  The adaptive preconditioner (the
Hessian diagonal at the current omega, with the full rotated Gram in the
sandwich) keeps CG short.  Device results are compared with the CPU oracle
running the same preconditioner, and every instance must pass the reference's
acceptance test.  On these targets the Newton path, with long backtracking, is
too sensitive to rounding to compare step counts.
"""
from __future__ import annotations

import pytest
import torch

from conftest import load_golden
from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu

XTOL = 1e-8


def rel_per_instance(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    num = torch.linalg.vector_norm((a - b).flatten(1), dim=1)
    den = torch.linalg.vector_norm(b.flatten(1), dim=1).clamp_min(1e-300)
    return (num / den).max().item()


@pytest.fixture(scope="module")
def sp():
    import symplectic_projection as sp
    sp.initialize_kernels()
    return sp


@pytest.fixture(scope="module")
def illcond():
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(512, 16, 2)
    Xo, Wo, Io = O.solve(T, preconditioner="adaptive")
    return T, Xo, Wo, Io


def test_reference_preconditioner_stalls_like_the_reference(sp, illcond):
    T = illcond[0]
    with pytest.raises(RuntimeError):
        sp.solve(T, preconditioner="eigenbasis")
    res = sp.solve_ex(T.cuda(), preconditioner="eigenbasis")
    assert 3 in res.status.cpu().tolist()                 # Newton cap on at least one instance


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_adaptive_preconditioner_solves_illconditioned_targets(sp, illcond, precision):
    T, Xo, Wo, Io = illcond
    X, W, it = sp.solve(T, precision=precision, preconditioner="adaptive")
    assert rel_per_instance(X, Xo) < XTOL and rel_per_instance(W, Wo) < XTOL
    assert int(it.max()) < 100
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


@pytest.mark.parametrize("name", ["n64_k8_b4", "n100_k20_b2", "n192_k48_b2", "n96_k64_b1", "n64_k4_b2_illcond"])
def test_adaptive_preconditioner_keeps_reference_solutions(sp, name):
    data = load_golden(name)
    T = torch.from_numpy(data["T"])
    X, W, it = sp.solve(T, preconditioner="adaptive")
    assert rel_per_instance(X, torch.from_numpy(data["X"])) < XTOL
    assert rel_per_instance(W, torch.from_numpy(data["omega"])) < XTOL
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_config5_width_illconditioned(sp, precision):
    """m = 128 (k = 64) ill-conditioned targets, the stress workload's width, at n = 2048."""
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(2048, 64, 2, seed=2026102501)
    res = sp.solve_ex(T.cuda(), precision=precision, preconditioner="adaptive")
    assert res.status.cpu().tolist() == [0, 0]
    for rec in O.inspect_output(T, res.X.cpu()):
        assert O.passes(rec), rec


@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_stress_instance_19_alone_at_full_size(sp, precision):
    """Target 19 of the stress batch (32768 x 128, Gram condition ~1e8) solved alone: it
    converges and passes the acceptance test in both forms, with no rerun."""
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(16384, 64, 20)[19:20].contiguous()
    res = sp.solve_ex(T.cuda(), precision=precision, preconditioner="adaptive")
    assert res.status.cpu().tolist() == [0]
    for rec in O.inspect_output(T, res.X.cpu()):
        assert O.passes(rec), rec


@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_adaptive_solution_is_a_consistent_inverse_pair(sp, precision):
    """With the adaptive preconditioner the returned P, Q stay an exact inverse pair of
    I + i omega: P symmetric, and P = (I + omega^2)^-1, Q = -omega P to rounding.  (X = T K^-1
    is then stationary, whatever the Gram's error.)"""
    from symplectic_projection import dual_recommended_hvp as D
    from symplectic_projection.gram_triangle_reflect import gram
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(2048, 64, 2, seed=2026102501).cuda()
    n = T.shape[1] // 2
    Cr, Ci = gram(T[:, :n], T[:, n:], precision=precision)
    final = []
    W, _, _ = D.dual_batch(Cr, Ci, final, precision=precision, preconditioner="adaptive")
    P, Q = (x.cpu() for x in final)
    W = W.cpu()
    eye = torch.eye(W.shape[-1], dtype=torch.float64)
    for b in range(W.shape[0]):
        Pn = torch.linalg.norm(P[b])
        assert torch.linalg.norm(P[b] - P[b].mT) / Pn < 1e-12
        Pi = torch.linalg.inv(eye + W[b] @ W[b])
        assert torch.linalg.norm(P[b] - Pi) / Pn < 1e-10
        assert torch.linalg.norm(Q[b] + W[b] @ P[b]) / Pn < 1e-10


def test_certified_solve_reruns_failures_in_the_other_form(sp):
    """solve_certified: passing instances keep the first form's result; a failure is
    rerun in the fallback form and replaced only where that passes."""
    from symplectic_projection.certify import solve_certified
    from symplectic_projection.inputs import illcond_targets
    T = torch.cat((O.make_inputs(64, 4, 0, 2)[0], illcond_targets(64, 4, 2))).cuda()
    X, W, it, rep = solve_certified(T, precision="split", fallback="fp64", preconditioner="adaptive")
    assert rep["passed"].all()
    ref = sp.solve_ex(T, precision="split", preconditioner="adaptive")
    keep = [i for i in range(4) if i not in rep["rerun"].tolist()]
    assert torch.equal(X[keep], ref.X[keep])
    for rec in O.inspect_output(T.cpu(), X.cpu()):
        assert O.passes(rec), rec
    # a forced cap fails every instance; with no fallback nothing is rerun
    X2, _, _, rep2 = solve_certified(T, precision="split", fallback=None, max_newton=1)
    assert not rep2["passed"].any() and rep2["rerun"].tolist() == [0, 1, 2, 3]
