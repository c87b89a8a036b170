"""The split form's FP32 early Newton phase (dual32_kernel) on the device.

In the split form the early Newton steps run in FP32 with the state on chip,
until the FP32 residual is below 1e-5; the FP64 Newton kernel then starts from
that omega (FP64 inverse with the positive-definiteness test) and takes the
last step(s), with the FP64 residual deciding convergence.  The results must
stay within 1e-8 relative of the CPU oracle's (the reference algorithm), pass
the reference's acceptance test, and take the same Newton path as the split
form with every step in FP64.  The counters of ssn_newton show that the FP32
phase ran and how many steps each phase took.
"""
from __future__ import annotations

import pytest
import torch

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


def newton_counters(T, precision="split", **opts):
    """ssn_newton on the split form's Gram and basis; returns (counters [B, 8], status, iterations)."""
    from symplectic_projection import _native as N
    from symplectic_projection import dual_recommended_hvp as D
    from symplectic_projection.gram_triangle_reflect import gram
    Td = T.cuda()
    B, rows, m = Td.shape
    n = rows // 2
    Cr, Ci = gram(Td[:, :n], Td[:, n:], precision=precision)
    values, vectors, scale, _ = D.eigh_scaled(Cr, precision=precision)
    lib = N.load()
    omega, P, Q = (torch.empty(B, m, m, dtype=torch.float64, device="cuda") for _ in range(3))
    iters = torch.empty(B, dtype=torch.int64, device="cuda")
    status = torch.empty(B, dtype=torch.int32, device="cuda")
    counters = torch.full((B, 8), -1, dtype=torch.int32, device="cuda")
    nbytes = lib.ssn_newton_workspace_bytes(B, m)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    opt = N.options(precision=precision, **opts)
    N.check(lib.ssn_newton(Cr.data_ptr(), Ci.data_ptr(), values.data_ptr(), vectors.data_ptr(),
                           scale.data_ptr(), None, omega.data_ptr(), P.data_ptr(), Q.data_ptr(),
                           iters.data_ptr(), status.data_ptr(), counters.data_ptr(), B, m, ws.data_ptr(),
                           nbytes, N.ctypes.byref(opt), N.stream_handle(Td.device)), "ssn_newton")
    return counters.cpu(), status.cpu(), iters.cpu()


# (n, k, batch): m = 24 (one CTA, 32-padded), 32, 64 (a cluster), 80 (a cluster, 96-padded), 96,
# and a single target (the golden fixtures' square and near-square targets run the split form in
# the split-form parity tests)
SHAPES = [(96, 12, 4), (2048, 16, 8), (256, 32, 6), (300, 40, 3), (4096, 48, 4), (4096, 48, 1)]


@pytest.mark.parametrize("n,k,B", SHAPES)
def test_fp32_phase_reaches_the_oracle_solution(sp, n, k, B):
    T, _ = O.make_inputs(n, k, 0, B)
    X, W, it = sp.solve(T, precision="split")
    Xo, Wo, Io = O.solve(T)
    assert rel_per_instance(X, Xo) < XTOL and rel_per_instance(W, Wo) < XTOL
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


@pytest.mark.parametrize("n,k,B", SHAPES)
def test_fp32_phase_runs_and_hands_over(sp, n, k, B):
    T, _ = O.make_inputs(n, k, 1, B)
    cnt, st, it = newton_counters(T)
    assert st.tolist() == [0] * B
    f64_steps, f32_steps = cnt[:, 0], cnt[:, 4]
    assert bool((f32_steps >= 2).all())                  # the FP32 phase ran
    assert bool((f64_steps <= 3).all())                  # the FP64 iteration only finishes
    # the same Newton path (up to one step) as the split form with every step in FP64
    cnt64, st64, it64 = newton_counters(T, fp32_newton=False)
    assert bool((cnt64[:, 4:] == 0).all())
    assert int((it - it64).abs().max()) <= 1


def test_fp32_phase_runs_for_more_instances_than_half_the_sms(sp):
    # m = 96 with 80 instances: the default cluster rule gives one CTA per instance there,
    # where the FP32 phase cannot hold its state; the split form takes the 2-CTA cluster
    # instead, so the FP32 phase still runs
    B = 80
    T, _ = O.make_inputs(128, 48, 3, B)
    cnt, st, _ = newton_counters(T)
    assert st.tolist() == [0] * B
    assert bool((cnt[:, 4] >= 2).all())
    X, W, it = sp.solve(T, precision="split")
    Xo, Wo, Io = O.solve(T[:4])
    assert rel_per_instance(X[:4], Xo) < XTOL and rel_per_instance(W[:4], Wo) < XTOL
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


def test_fp32_phase_agrees_with_all_fp64_newton(sp):
    T, _ = O.make_inputs(4096, 48, 5, 8)
    Td = T.cuda()
    a = sp.solve_ex(Td, precision="split")
    b = sp.solve_ex(Td, precision="split", fp32_newton=False)
    assert a.status.tolist() == b.status.tolist() == [0] * 8
    # both stop at a residual below feas_tol / 2 = 5e-9, so they agree to about that, and to
    # the parity bound that holds each against the oracle
    assert rel_per_instance(a.X, b.X) < XTOL and rel_per_instance(a.omega, b.omega) < XTOL


def test_fp32_phase_with_the_adaptive_preconditioner(sp):
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(512, 16, 2)
    Xo, Wo, Io = O.solve(T, preconditioner="adaptive")
    X, W, it = sp.solve(T, precision="split", preconditioner="adaptive")
    assert rel_per_instance(X, Xo) < XTOL and rel_per_instance(W, Wo) < XTOL
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec
    cnt, st, _ = newton_counters(T, preconditioner="adaptive")
    assert st.tolist() == [0, 0] and bool((cnt[:, 4] >= 1).all())


@pytest.mark.parametrize("n,k", [(512, 48), (300, 40)])
def test_fp32_phase_with_the_adaptive_preconditioner_on_a_cluster(sp, n, k):
    # m = 96 and m = 80 run the FP32 phase on a 2-CTA cluster with the adaptive denominators
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(n, k, 2)
    Xo, Wo, Io = O.solve(T, preconditioner="adaptive")
    X, W, it = sp.solve(T, precision="split", preconditioner="adaptive")
    assert rel_per_instance(X, Xo) < XTOL and rel_per_instance(W, Wo) < XTOL
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec
    cnt, st, _ = newton_counters(T, preconditioner="adaptive")
    assert st.tolist() == [0, 0] and bool((cnt[:, 4] >= 1).all())


def test_fp32_phase_isolates_a_nonfinite_instance(sp):
    T, _ = O.make_inputs(256, 32, 2, 3)
    T[1, 5, 3] = float("nan")
    res = sp.solve_ex(T.cuda(), precision="split")
    st = res.status.cpu().tolist()
    assert st[1] == 5 and st[0] == 0 and st[2] == 0
    X = res.X.cpu()
    for j in (0, 2):
        assert O.passes(O.inspect_output(T[j:j + 1], X[j:j + 1])[0])


def test_fp32_phase_counts_toward_the_newton_cap(sp):
    T, _ = O.make_inputs(256, 32, 3, 2)
    res = sp.solve_ex(T.cuda(), precision="split", max_newton=2)
    assert res.status.cpu().tolist() == [3, 3]
