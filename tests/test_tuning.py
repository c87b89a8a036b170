"""The autotuned launch-parameter table (ssn_set_tuning): validation and sizing, host only."""
from __future__ import annotations

import json

import pytest

pytest.importorskip("torch")


@pytest.fixture()
def at():
    from symplectic_projection import _native as N
    from symplectic_projection import autotune
    if not N.LIB_PATH.exists():
        pytest.skip("native library not built")
    saved = autotune.installed()
    yield autotune
    autotune.install(saved)


def entry(**kw):
    e = {"precision": "split", "m": 96, "n_min": 4096, "n_max": 4096, "batch_min": 64, "batch_max": 64,
         "gram_splits": 0, "gram_chunks": 2, "recover_parts": 8, "cluster": 2}
    e.update(kw)
    return e


def test_install_and_read_back(at):
    es = [entry(), entry(precision="fp64", gram_splits=4, gram_chunks=0, recover_parts=0, cluster=1)]
    at.install(es)
    got = at.installed()
    assert len(got) == 2
    for a, b in zip(got, es):
        assert {k: a[k] for k in b} == b
    at.install([])
    assert at.installed() == []


@pytest.mark.parametrize("bad", [dict(cluster=2, m=32), dict(cluster=3), dict(gram_splits=65),
                                 dict(gram_chunks=-1), dict(recover_parts=2000), dict(m=130),
                                 dict(m=7), dict(n_min=10, n_max=5), dict(batch_min=0)])
def test_invalid_entries_are_refused_and_leave_the_table(at, bad):
    at.install([entry()])
    with pytest.raises(RuntimeError):
        at.install([entry(), entry(**bad)])
    assert len(at.installed()) == 1


def test_workspace_follows_the_tuned_fp64_gram_splits(at):
    from symplectic_projection import _native as N
    lib = N.load()
    at.install([])
    base = lib.ssn_workspace_bytes(2, 200000, 8)
    at.install([entry(precision="fp64", m=8, n_min=200000, n_max=200000, batch_min=2, batch_max=2,
                      gram_splits=64, gram_chunks=0, recover_parts=0, cluster=0)])
    more = lib.ssn_workspace_bytes(2, 200000, 8)
    assert more >= base
    at.install([])
    assert lib.ssn_workspace_bytes(2, 200000, 8) == base


def test_committed_table_is_valid(at):
    if not at.TABLE_PATH.exists():
        pytest.skip("no committed table")
    entries = json.loads(at.TABLE_PATH.read_text())["entries"]
    assert entries
    at.install(entries)
    assert len(at.installed()) == len(entries)
    for e in entries:
        assert any(e[f] for f in at.FIELDS)
        assert e["tuned_ms"] <= e["builtin_ms"]


def test_parallel_host_copies():
    import torch
    from symplectic_projection.dual_recommended_hvp import _parallel_copies
    g = torch.Generator().manual_seed(5)
    srcs = [torch.randn(int(n), dtype=torch.float64, generator=g) for n in torch.randint(1, 5000, (97,), generator=g)]
    flat = torch.empty(sum(s.numel() for s in srcs), dtype=torch.float64)
    offs = [0]
    for s in srcs:
        offs.append(offs[-1] + s.numel())
    _parallel_copies([(flat[offs[i]:offs[i + 1]], s) for i, s in enumerate(srcs)])
    assert torch.equal(flat, torch.cat(srcs))
    outs = [torch.empty_like(s) for s in srcs]
    _parallel_copies([(o, flat[offs[i]:offs[i + 1]]) for i, o in enumerate(outs)])
    assert all(torch.equal(o, s) for o, s in zip(outs, srcs))
