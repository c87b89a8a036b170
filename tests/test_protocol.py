"""The reference's timing protocol (reproduce.py:13-34, experiment.py:140-262) on this package.

CPU tests cover the host logic (schedule, seeds, shuffles, validation rule and
summary); the GPU test runs a reduced protocol through the public solve.
"""
from __future__ import annotations

import math
import random

import pytest
import torch

from oracle import ssn_oracle as O
from symplectic_projection import protocol as P


def test_round_orders_cover_every_case_once_per_round():
    names = [c["name"] for c in P.PROTOCOL["cases"]]
    assert names == ["n2048_k16", "n2048_k32", "n2048_k48", "n4096_k16", "n4096_k32", "n4096_k48"]
    assert len(P.PROTOCOL["round_orders"]) == P.PROTOCOL["rounds"] == 3
    for order in P.PROTOCOL["round_orders"]:
        assert sorted(order) == sorted(names)


def test_case_inputs_follow_the_seed_rule():
    proto = dict(P.PROTOCOL, targets_per_case=3)
    case = dict(name="n64_k4", n=64, k=4)
    T, seeds = P.case_inputs(case, 2, proto)
    assert seeds == [2026102100 + 2000 + j for j in range(3)]
    To, seeds_o = O.make_inputs(64, 4, 2, 3)
    assert list(seeds_o) == seeds
    assert torch.equal(T, To)


def test_schedule_matches_the_reference_order():
    proto = dict(P.PROTOCOL, targets_per_case=5)
    for case_index in range(6):
        for rnd in (1, 2, 3):
            steps = list(P.schedule(proto, case_index, rnd))
            warm_single = [s for s in steps if s[0] == "warmup" and s[1] == "single"]
            meas_single = [s for s in steps if s[0] == "measured" and s[1] == "single"]
            warm_batch = [s for s in steps if s[0] == "warmup" and s[1] == "batch"]
            meas_batch = [s[2] for s in steps if s[0] == "measured" and s[1] == "batch"]
            assert len(warm_single) == 2 and [s[3] for s in meas_single] == list(range(5))
            assert [s[2] for s in warm_batch] == ["dual_sequential", "dual"]
            expect = ["dual", "dual_sequential"] if (rnd - 1 + case_index) % 2 else ["dual_sequential", "dual"]
            assert meas_batch == expect
            # warm-ups come first, the batch experiment last
            assert steps.index(warm_batch[0]) > steps.index(meas_single[-1])


def test_shuffle_is_the_reference_rule():
    order = list(range(64))
    random.Random(202610210000 + 100 * 2 + 5).shuffle(order)
    again = list(range(64))
    random.Random(P.PROTOCOL["shuffle_seed_base"] + 100 * 2 + 5).shuffle(again)
    assert order == again and sorted(order) == list(range(64)) and order != list(range(64))


def test_numeric_pass_rule():
    th = P.PROTOCOL["thresholds"]
    assert P.numeric_pass(dict(feasibility=1e-9, stationarity=1e-10, delta=-1e-9), th)
    assert not P.numeric_pass(dict(feasibility=2e-8, stationarity=1e-10, delta=0.0), th)
    assert not P.numeric_pass(dict(feasibility=1e-9, stationarity=math.nan, delta=0.0), th)
    assert not P.numeric_pass(dict(feasibility=1e-9, delta=0.0), th)


def test_summary_means_and_speedup():
    proto = dict(P.PROTOCOL, targets_per_case=2)
    ok = [dict(index=0, feasibility=1e-12, stationarity=1e-13, delta=1e-12)]
    rows = []
    for rnd, (seq, bat) in enumerate([(10.0, 2.0), (14.0, 2.0)], 1):
        for pos, ms in enumerate((1.0, 3.0)):
            rows.append(dict(case="n2048_k16", round=rnd, phase="measured", experiment="single", method="dual",
                             item=pos, milliseconds=ms, exception=None, validation=ok, success=True))
        rows.append(dict(case="n2048_k16", round=rnd, phase="measured", experiment="batch",
                         method="dual_sequential", item=None, milliseconds=seq, exception=None,
                         validation=ok * 2, success=True))
        rows.append(dict(case="n2048_k16", round=rnd, phase="measured", experiment="batch", method="dual",
                         item=None, milliseconds=bat, exception=None, validation=ok * 2, success=True))
    s = P.summarize(rows, proto)
    item = s["cases"][0]
    assert item["single"]["dual"]["milliseconds"]["mean"] == 2.0
    assert item["batch"]["dual_sequential"]["round_mean_ms"] == [10.0, 14.0]
    assert item["batch"]["speedups"]["dual_sequential"] == 6.0
    assert item["batch"]["solves_per_s"] == 1000.0
    assert s["all_calls_successful"] and s["accuracy"]["max_delta"] == 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_reduced_protocol_on_the_device(tmp_path, precision):
    import symplectic_projection as sp
    sp.initialize_kernels()
    proto = dict(P.PROTOCOL, targets_per_case=4)
    s = P.run_protocol(proto, rounds=1, cases=["n2048_k16", "n4096_k48"], precision=precision,
                       output=tmp_path / "run")
    assert s["all_calls_successful"], s["failure_records"]
    assert s["counts"]["formal_calls"] == 2 * (4 + 2)
    for item in s["cases"]:
        assert item["batch"]["speedups"]["dual_sequential"] > 1.0     # one batched call beats four single ones
    assert (tmp_path / "run" / "summary.json").exists() and (tmp_path / "run" / "raw.jsonl").exists()


def test_ragged_workload_rule():
    from symplectic_projection.inputs import RAGGED_K, RAGGED_N, ragged_shapes, ragged_targets
    shapes = ragged_shapes(384)
    assert len(shapes) == 384 and ragged_shapes(384) == shapes
    assert {n for n, _ in shapes} == set(RAGGED_N) and {k for _, k in shapes} == set(RAGGED_K)
    assert 1.2e9 < sum(2 * n * 2 * k * 8 for n, k in shapes) < 1.35e9         # about 1.25 GB of T
    t = ragged_targets(3, shapes=[(64, 4), (32, 2), (64, 4)])
    assert [tuple(x.shape) for x in t] == [(128, 8), (64, 4), (128, 8)] and not torch.equal(t[0], t[2])
    g = torch.Generator().manual_seed(2026102300 + 1 + 2)
    assert torch.equal(t[2], torch.randn(128, 8, dtype=torch.float64, generator=g) / math.sqrt(128))


def test_host_chunk_plan():
    from symplectic_projection.dual_recommended_hvp import _chunk_plan
    for batch in (1, 3, 7, 15, 16, 30, 31, 64, 100):
        for cap in (1, 4, 8):
            for ramp in ((), (1, 2, 4, 8), (2, 4)):
                sizes = _chunk_plan(batch, cap, ramp)
                assert sum(sizes) == batch and min(sizes) >= 1
    assert _chunk_plan(64, 4, (1, 2, 4, 8)) == [1, 2, 4, 8] + [4] * 7 + [3, 3] + [8, 4, 2, 1]
    assert _chunk_plan(10, 4, (1, 2, 4, 8)) == [4, 3, 3]               # too short for the ramps
