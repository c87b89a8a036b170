"""Ragged batches (ssn_solve_ragged): targets of different (n, k) in one call.

Every instance must get the result of solving it alone: the same X and omega as
the CPU oracle within 1e-8 relative (the bound of the uniform solve), the
oracle's iteration count, and the acceptance test.  Groups run concurrently,
so the test also mixes shapes whose Newton kernels use different CTA counts.
"""
from __future__ import annotations

import pytest
import torch

from oracle import ssn_oracle as O
from symplectic_projection.inputs import ragged_shapes, ragged_targets

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b).clamp_min(1e-300))


@pytest.fixture(scope="module")
def sp():
    import symplectic_projection as sp
    sp.initialize_kernels()
    return sp


SHAPES = [(64, 4), (100, 20), (64, 4), (300, 48), (40, 2), (100, 20), (64, 4), (128, 64), (300, 48), (33, 1)]


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("device_input", [True, False])
def test_ragged_matches_the_oracle_per_instance(sp, precision, device_input):
    targets = ragged_targets(len(SHAPES), seed=77, shapes=SHAPES)
    ins = [t.cuda() for t in targets] if device_input else targets
    Xs, Ws, it, st = sp.solve_ragged(ins, precision=precision)
    assert st.cpu().tolist() == [0] * len(SHAPES)
    for i, t in enumerate(targets):
        Xo, Wo, Io = O.solve(t.unsqueeze(0))
        assert Xs[i].shape == t.shape and Ws[i].shape == (t.shape[1], t.shape[1])
        assert Xs[i].is_cuda == device_input
        assert rel(Xs[i], Xo[0]) < 1e-8, (i, SHAPES[i])
        assert rel(Ws[i], Wo[0]) < 1e-8, (i, SHAPES[i])
        if precision == "fp64":
            assert int(it[i]) == int(Io[0]), (i, SHAPES[i])
        else:                          # another basis, another Newton path to the same optimum
            assert int(it[i]) <= 2 * int(Io[0]) + 2, (i, SHAPES[i])
        rec = O.inspect_output(t.unsqueeze(0), Xs[i].cpu().unsqueeze(0))[0]
        assert O.passes(rec), rec


def test_ragged_equals_uniform_solves(sp):
    """Within a shape group the ragged call is the uniform pipeline: same X as ssn_solve."""
    targets = ragged_targets(6, seed=5, shapes=[(256, 16)] * 3 + [(128, 8)] * 3)
    Xs, Ws, it, st = sp.solve_ragged([t.cuda() for t in targets])
    for lo in (0, 3):
        T = torch.stack(targets[lo:lo + 3]).cuda()
        X, W, I = sp.solve(T)
        for j in range(3):
            assert rel(Xs[lo + j], X[j]) < 1e-12 and int(it[lo + j]) == int(I[j])


def test_ragged_reports_per_instance_failures(sp):
    targets = ragged_targets(4, seed=9, shapes=[(64, 4), (64, 8), (64, 4), (32, 2)])
    targets[2] = targets[2].clone()
    targets[2][5, 1] = float("nan")
    Xs, Ws, it, st = sp.solve_ragged([t.cuda() for t in targets], raise_on_failure=False)
    codes = st.cpu().tolist()
    assert codes[2] == 5 and codes[0] == codes[1] == codes[3] == 0
    with pytest.raises(RuntimeError):
        sp.solve_ragged([t.cuda() for t in targets[:2]], max_newton=1)


def test_ragged_workload_sample(sp):
    """A 24-target sample of the ragged workload's shape distribution, host in and out."""
    shapes = ragged_shapes(384)[:24]
    targets = ragged_targets(24, shapes=shapes)
    Xs, Ws, it, st = sp.solve_ragged(targets, precision="split")
    assert st.tolist() == [0] * 24
    recs = [O.inspect_output(t.unsqueeze(0), X.unsqueeze(0))[0] for t, X in zip(targets, Xs)]
    assert all(O.passes(r) for r in recs), O.worst(recs)
