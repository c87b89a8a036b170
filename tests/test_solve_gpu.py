"""End-to-end parity of the device solver with the reference (golden fixtures)
and with the CPU oracle at the benchmark sizes."""
from __future__ import annotations

import pytest
import torch

from conftest import golden_manifest, load_golden
from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu

XTOL = 1e-8    # X and omega within 1e-8 relative of the reference's


def rel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))


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
def test_solve_matches_reference_fixture(sp, name, manifest):
    meta = manifest[name]
    data = load_golden(name)
    T = torch.from_numpy(data["T"])
    if "error" in meta:
        with pytest.raises(RuntimeError):
            sp.solve(T)
        return
    X, omega, it = sp.solve(T)
    assert X.device.type == "cpu" and omega.device.type == "cpu" and it.dtype == torch.int64
    assert rel_per_instance(X, torch.from_numpy(data["X"])) < XTOL
    assert rel_per_instance(omega, torch.from_numpy(data["omega"])) < XTOL
    if meta.get("transform") and meta["transform"][0] == "illcond":
        # graded spectra with long backtracking: rounding can shift the Newton path by a step or two
        assert all(abs(a - b) <= max(2, b // 10) for a, b in zip(it.tolist(), meta["iterations"]))
    else:
        assert it.tolist() == meta["iterations"]
    for rec in O.inspect_output(T, X):
        assert O.passes(rec), rec


def test_device_resident_solve_and_status(sp):
    data = load_golden("n48_k12_b3")
    T = torch.from_numpy(data["T"]).cuda()
    res = sp.solve_ex(T)
    assert res.X.is_cuda and res.omega.is_cuda
    assert res.status.cpu().tolist() == [0, 0, 0]
    assert rel(res.X, torch.from_numpy(data["X"])) < XTOL


def test_single_target_form(sp):
    # experiment.call_method "dual_sequential": solve(t.unsqueeze(0)) per target
    data = load_golden("n64_k8_b4")
    T = torch.from_numpy(data["T"])
    for j in range(T.shape[0]):
        X, omega, it = sp.solve(T[j].unsqueeze(0))
        assert rel(X[0], torch.from_numpy(data["X"][j])) < XTOL
        assert int(it[0]) == data["iterations"][j]


def test_newton_cap_raises(sp):
    data = load_golden("n64_k8_b4")
    with pytest.raises(RuntimeError):
        sp.solve(torch.from_numpy(data["T"]), max_newton=2)
    res = sp.solve_ex(torch.from_numpy(data["T"]).cuda(), max_newton=2)
    assert set(res.status.cpu().tolist()) == {3}


def test_line_search_cap_raises(sp):
    data = load_golden("n64_k4_b2_illcond")      # needs backtracking (127 reference trials)
    T = torch.from_numpy(data["T"])
    with pytest.raises(RuntimeError):
        O.solve(T, max_backtrack=1)
    with pytest.raises(RuntimeError):
        sp.solve(T, max_backtrack=1)
    res = sp.solve_ex(T.cuda(), max_backtrack=1)
    assert 4 in res.status.cpu().tolist()


def test_nonfinite_input_flagged(sp):
    T, _ = O.make_inputs(16, 4, 0, 2)
    T[1, 3, 2] = float("nan")
    res = sp.solve_ex(T.cuda())
    codes = res.status.cpu().tolist()
    assert codes[0] == 0 and codes[1] != 0


@pytest.mark.parametrize("n,k,case", [(2048, 16, 0), (4096, 48, 5)])
def test_benchmark_config_parity(sp, n, k, case):
    """Full 64-target batches of the protocol cases against the CPU oracle."""
    T, _ = O.make_inputs(n, k, case, 64)
    torch.set_num_threads(max(1, torch.get_num_threads()))
    Xo, Wo, Io = O.solve(T)
    X, W, I = sp.solve(T)
    assert rel_per_instance(X, Xo) < XTOL
    assert rel_per_instance(W, Wo) < XTOL
    assert I.tolist() == Io.tolist()
    recs = O.inspect_output(T, X)
    assert all(O.passes(r) for r in recs), O.worst(recs)


def test_batch_composition_independence(sp):
    """Per-instance results do not depend on the other instances of the batch."""
    T, _ = O.make_inputs(64, 8, 3, 6)
    Xa, Wa, Ia = sp.solve(T)
    Xb, Wb, Ib = sp.solve(T[2:5].contiguous())
    # the Gram split-K count depends on the batch size, so only rounding may differ
    assert rel(Xa[2:5], Xb) < 1e-12 and rel(Wa[2:5], Wb) < 1e-12 and torch.equal(Ia[2:5], Ib)


@pytest.mark.parametrize("pinned", [False, True])
def test_chunked_host_pipeline(sp, pinned, monkeypatch):
    """CPU-in/CPU-out solves split into stream-pipelined chunks match the device-resident solve."""
    from symplectic_projection import dual_recommended_hvp as D
    T, _ = O.make_inputs(256, 24, 4, 21)
    if pinned:
        T = T.pin_memory()
    monkeypatch.setattr(D, "CHUNK_BYTES", 4 * T[0].numel() * 8)   # 4 targets per chunk -> 6 chunks
    X, W, I = sp.solve(T)
    Xd, Wd, Id = sp.solve(T.cuda())
    assert rel(X, Xd) < 1e-12 and rel(W, Wd) < 1e-12 and torch.equal(I, Id.cpu())
    assert X.shape == T.shape and W.shape == (21, 48, 48)
