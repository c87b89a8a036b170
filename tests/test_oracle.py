"""The CPU oracle against the reference's own outputs (golden fixtures)."""
from __future__ import annotations

import pytest
import torch

from conftest import golden_manifest, load_golden
from oracle import ssn_oracle as O

CASES = sorted(golden_manifest())


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / max(torch.linalg.vector_norm(b), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name, manifest):
    meta = manifest[name]
    data = load_golden(name)
    T = torch.from_numpy(data["T"])
    stats = O.DualStats()
    if "error" in meta:
        with pytest.raises(RuntimeError):
            O.solve(T, stats)
        return
    X, omega, it = O.solve(T, stats)
    assert it.tolist() == meta["iterations"]
    assert stats.hvps == meta["counts"]["hvp_outer"]
    assert stats.trials == meta["counts"]["line_change"]
    assert _rel(X, torch.from_numpy(data["X"])) < 1e-10
    assert _rel(omega, torch.from_numpy(data["omega"])) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_inspect_output_matches_reference(name, manifest):
    meta = manifest[name]
    if "error" in meta:
        pytest.skip("the reference raised on this input; no output to inspect")
    data = load_golden(name)
    T, X = torch.from_numpy(data["T"]), torch.from_numpy(data["X"])
    recs = O.inspect_output(T, X)
    ref = data["metrics"]
    for rec, row in zip(recs, ref):
        assert O.passes(rec)
        for key, want in zip(("feasibility", "stationarity", "delta"), row):
            # the metrics are residual-sized: compare on an absolute scale of the thresholds
            assert abs(rec[key] - want) <= 1e-3 * O.THRESHOLDS[key] + 1e-6 * abs(want)


def test_make_inputs_seed_rule():
    T, seeds = O.make_inputs(8, 2, 1, 3)
    assert seeds == [2026102100 + 1000 + j for j in range(3)]
    g = torch.Generator().manual_seed(seeds[2])
    want = torch.randn(16, 4, dtype=torch.float64, generator=g) / 4.0
    assert torch.equal(T[2], want)


def test_gram_fixture():
    data = load_golden("n48_k12_b3")
    Cr, Ci = O.gram(torch.from_numpy(data["T"]))
    assert _rel(Cr, torch.from_numpy(data["Cr"])) < 1e-14
    assert _rel(Ci, torch.from_numpy(data["Ci"])) < 1e-14


def test_adaptive_denominator_is_the_hessian_diagonal():
    """The adaptive preconditioner (this build's extension) is diag(H) on the skew basis."""
    torch.manual_seed(7)
    m = 10
    Cr = torch.randn(m, m, dtype=torch.float64)
    Cr = Cr @ Cr.mT + m * torch.eye(m, dtype=torch.float64)
    values = torch.linalg.eigvalsh(Cr)[None]
    Ci = O.skew(torch.randn(1, m, m, dtype=torch.float64))
    W = O.skew(torch.randn(1, m, m, dtype=torch.float64)) * 0.3
    P = torch.linalg.inv(torch.eye(m, dtype=torch.float64) + W @ W)
    Q = -W @ P
    Sr, Si = O.sandwich(values, Ci, P, Q)
    den = O.adaptive_denominator(P, Q, Sr, Si)[0]
    for i in range(m):
        for j in range(m):
            if i == j:
                continue
            E = torch.zeros(1, m, m, dtype=torch.float64)
            E[0, i, j], E[0, j, i] = 1.0, -1.0
            assert abs(float(O.hvp(P, Q, Sr, Si, E)[0, i, j]) - float(den[i, j])) < 1e-12 * float(den.abs().max())


def test_adaptive_preconditioner_converges_where_the_reference_stalls():
    """Ill-conditioned targets (singular values log-uniform in [1e-2, 1e2]): the reference's
    preconditioner lets CG saturate and the Newton cap is reached; the adaptive one converges."""
    from symplectic_projection.inputs import illcond_targets
    T = illcond_targets(512, 16, 2)
    with pytest.raises(RuntimeError):
        O.solve(T, preconditioner="eigenbasis")
    X, W, it = O.solve(T, preconditioner="adaptive")
    assert all(O.passes(r) for r in O.inspect_output(T, X))


def test_adjoint_routes_agree_on_cpu():
    """The dual closed-form adjoint equals the dense primal KKT adjoint and finite differences."""
    T, _ = O.make_inputs(12, 2, 0, 2)
    g = torch.Generator().manual_seed(4)
    G = torch.randn(T.shape, dtype=torch.float64, generator=g)
    Gw = torch.randn(2, 4, 4, dtype=torch.float64, generator=g)
    a = O.adjoint_formula(T, G)
    k = O.adjoint_kkt(T, G)
    assert float(torch.linalg.vector_norm(a - k) / torch.linalg.vector_norm(k)) < 1e-10
    fd, V = O.adjoint_fd(T, G, Gw, h=1e-6, seed=2)
    ad = (O.adjoint_formula(T, G, Gw) * V).sum(dim=(-2, -1))
    assert float(((ad - fd).abs() / fd.abs()).max()) < 1e-6
