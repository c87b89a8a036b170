"""Every entry of the committed autotune table: the tuned schedule solves its class to
the same result as the built-in schedule, and both pass the reference's acceptance test."""
from __future__ import annotations

import json

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu


def _entries():
    from pathlib import Path
    p = Path(__file__).resolve().parents[1] / "symplectic-stiefel-nearness_b200" / "symplectic_projection" / "tuning_b200.json"
    return json.loads(p.read_text())["entries"] if p.exists() else []


ENTRIES = _entries()


@pytest.mark.parametrize("e", ENTRIES, ids=[f"{e['precision']}-n{e['n_min']}-m{e['m']}-b{e['batch_min']}" for e in ENTRIES])
def test_tuned_entry_matches_builtin_schedule(e):
    import symplectic_projection as sp
    from symplectic_projection import autotune
    from symplectic_projection.certify import certify
    n, k = e["n_min"], e["m"] // 2
    batch = e["batch_min"] if e["batch_max"] == e["batch_min"] else 4
    T = O.make_inputs(n, k, 3, batch)[0].cuda()
    saved = autotune.installed()
    try:
        autotune.install([e])
        tuned = sp.solve_ex(T, precision=e["precision"])
        autotune.install([])
        plain = sp.solve_ex(T, precision=e["precision"])
    finally:
        autotune.install(saved)
    assert tuned.status.tolist() == plain.status.tolist() == [0] * batch
    num = torch.linalg.vector_norm((tuned.X - plain.X).flatten(1), dim=1)
    den = torch.linalg.vector_norm(plain.X.flatten(1), dim=1)
    assert float((num / den).max()) < 1e-8
    assert int((tuned.iterations - plain.iterations).abs().max()) <= 1
    assert bool(certify(T, tuned.X)["passed"].all())
