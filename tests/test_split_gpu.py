"""Parity of the split-precision form with the reference (golden fixtures) and the CPU oracle.

The split form takes the eigenbasis of the scaled Gram from a few FP32 Jacobi
sweeps, re-orthogonalises it in FP64 and runs the Newton iteration with the
full rotated Gram.  It solves the same dual problem, so X and omega must match
the reference's within the same 1e-8 relative bound as the FP64 form and every
instance must pass the reference's acceptance test (r_F <= 1e-8, r_G <= 1e-9,
delta <= 1e-8).  On the benchmark workloads the Newton path stays within one
step of the reference's.
"""
from __future__ import annotations

import pytest
import torch

from conftest import golden_manifest, load_golden
from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu

XTOL = 1e-8      # X and omega within 1e-8 relative of the reference's, per instance


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


@pytest.mark.parametrize("name", sorted(golden_manifest()))
def test_split_matches_reference_fixture(sp, name, manifest):
    meta = manifest[name]
    data = load_golden(name)
    T = torch.from_numpy(data["T"])
    if "error" in meta:
        # the reference raises on these; the split form must raise too or return accepted results
        try:
            X, omega, it = sp.solve(T, precision="split")
        except RuntimeError:
            return
        assert all(O.passes(r) for r in O.inspect_output(T, X))
        return
    X, omega, it = sp.solve(T, precision="split")
    assert rel_per_instance(X, torch.from_numpy(data["X"])) < XTOL
    assert rel_per_instance(omega, torch.from_numpy(data["omega"])) < XTOL
    if not (meta.get("transform") and meta["transform"][0] == "illcond"):
        # Another basis gives another Newton path to the same optimum: on the near-square fixtures
        # (Gram condition ~1e2) the split form can take fewer steps than the reference (11 vs 21 at
        # n=96, k=64).  Guard only against a blow-up here; the benchmark workloads below hold the
        # path to within one step.  (The ill-conditioned fixture, Gram condition 1e8 with long
        # backtracking, has a chaotic path: even FP64 rotations with 3 vs 5 sweeps give 56 vs 35
        # steps against the reference's 37.)
        assert all(a <= 2 * b + 2 for a, b in zip(it.tolist(), meta["iterations"])), \
            (it.tolist(), meta["iterations"])
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


@pytest.mark.parametrize("sweeps", [1, 2, 3, 5, 12])
def test_split_sweep_count_does_not_change_the_solution(sp, sweeps):
    data = load_golden("n100_k20_b2")
    T = torch.from_numpy(data["T"]).cuda()
    res = sp.solve_ex(T, precision="split", eig_sweeps=sweeps)
    assert res.status.cpu().tolist() == [0, 0]
    assert rel_per_instance(res.X, torch.from_numpy(data["X"])) < XTOL
    assert rel_per_instance(res.omega, torch.from_numpy(data["omega"])) < XTOL


def test_split_rough_basis_is_orthogonal_after_refinement(sp):
    """The FP32 basis is only roughly orthogonal; the Newton kernel's FP64 refinement fixes it."""
    from symplectic_projection.dual_recommended_hvp import eigh_scaled
    T, _ = O.make_inputs(512, 32, 0, 3)
    Cr, _ = O.gram(T)
    values, V, scale, sweeps = eigh_scaled(Cr.cuda(), precision="split", eig_sweeps=3)
    V = V.cpu()
    m = V.shape[-1]
    orth = (V.mT @ V - torch.eye(m, dtype=torch.float64)).abs().max().item()
    assert 0 < orth < 1e-4                                  # FP32 rotations: roughly orthogonal
    assert sweeps.cpu().tolist() == [3, 3, 3]
    Vr = V
    for _ in range(2):                                      # the Newton kernel's two Newton-Schulz steps
        Vr = Vr @ (3 * torch.eye(m, dtype=torch.float64) - Vr.mT @ Vr) / 2
    assert (Vr.mT @ Vr - torch.eye(m, dtype=torch.float64)).abs().max().item() < 1e-14
    # V roughly diagonalises Cr/scale: off-diagonal mass well below the diagonal
    R = Vr.mT @ (Cr / scale.cpu()[:, None, None]) @ Vr
    off = torch.linalg.vector_norm(R - torch.diag_embed(R.diagonal(dim1=-2, dim2=-1)), dim=(-2, -1))
    assert float((off / torch.linalg.vector_norm(R, dim=(-2, -1))).max()) < 0.05


def test_split_dual_entry_point(sp):
    from symplectic_projection.dual_recommended_hvp import dual_batch
    data = load_golden("n64_k8_b4")
    T = torch.from_numpy(data["T"])
    Cr, Ci = O.gram(T)
    final = []
    omega, L, it = dual_batch(Cr.cuda(), Ci.cuda(), final, precision="split")
    assert rel_per_instance(omega, torch.from_numpy(data["omega"])) < XTOL
    assert rel_per_instance(final[0], torch.from_numpy(data["P"])) < XTOL


def test_split_caps_and_nonfinite(sp):
    data = load_golden("n64_k8_b4")
    with pytest.raises(RuntimeError):
        sp.solve(torch.from_numpy(data["T"]), max_newton=2, precision="split")
    T, _ = O.make_inputs(16, 4, 0, 2)
    T[1, 3, 2] = float("nan")
    codes = sp.solve_ex(T.cuda(), precision="split").status.cpu().tolist()
    assert codes[0] == 0 and codes[1] != 0


@pytest.mark.parametrize("n,k,case", [(2048, 16, 0), (4096, 48, 5)])
def test_split_benchmark_config_parity(sp, n, k, case):
    """Full 64-target batches of the protocol cases: split form against the CPU oracle."""
    T, _ = O.make_inputs(n, k, case, 64)
    Xo, Wo, Io = O.solve(T)
    X, W, I = sp.solve(T, precision="split")
    assert rel_per_instance(X, Xo) < XTOL
    assert rel_per_instance(W, Wo) < XTOL
    assert int((I - Io).abs().max()) <= 1
    recs = O.inspect_output(T, X)
    assert all(O.passes(r) for r in recs), O.worst(recs)


def test_split_default_basis_choice(sp):
    """With the default sweep count the split form keeps the identity basis for nearly
    diagonal Grams (Gaussian targets) and runs one sweep otherwise; explicit counts are kept."""
    from symplectic_projection.dual_recommended_hvp import eigh_scaled
    from symplectic_projection.inputs import illcond_targets
    Tg, _ = O.make_inputs(4096, 48, 5, 3)                   # largest correlation ~ 4/sqrt(8192)
    Ti = illcond_targets(512, 16, 2)
    Crg, _ = O.gram(Tg)
    Cri, _ = O.gram(Ti)
    _, Vg, _, sw_g = eigh_scaled(Crg.cuda(), precision="split")
    _, Vi, _, sw_i = eigh_scaled(Cri.cuda(), precision="split")
    assert sw_g.cpu().tolist() == [0, 0, 0] and sw_i.cpu().tolist() == [1, 1]
    Vg = Vg.cpu()
    assert torch.equal(Vg.abs().sum(dim=1), torch.ones(3, 96, dtype=torch.float64))   # a permutation
    _, _, _, sw_x = eigh_scaled(Crg.cuda(), precision="split", eig_sweeps=2)
    assert sw_x.cpu().tolist() == [2, 2, 2]
    # and the identity basis still solves to the oracle's X
    res = sp.solve_ex(Tg.cuda(), precision="split")
    Xo, Wo, _ = O.solve(Tg)
    assert res.status.cpu().tolist() == [0, 0, 0]
    assert rel_per_instance(res.X, Xo) < XTOL and rel_per_instance(res.omega, Wo) < XTOL
