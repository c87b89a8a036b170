"""Several GPUs as independent replicas: the host logic, on CPU with gloo ranks.

The batch is split by estimated cost with no data-path collective; the only
collectives are the max-over-ranks step time and the gather of per-rank
results.  Two gloo ranks on 127.0.0.1 run the same plan and exchange results.
"""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from symplectic_projection import replicas as R
from symplectic_projection.inputs import ragged_shapes


def test_partition_covers_every_target_once_and_balances():
    shapes = ragged_shapes(384)
    for world in (1, 2, 3, 8):
        parts = R.partition_by_cost(shapes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(384))
        loads = [sum(R.target_cost(*shapes[i]) for i in p) for p in parts]
        # largest-first greedy: no rank exceeds the mean by more than one target's cost
        biggest = max(R.target_cost(*s) for s in shapes)
        assert max(loads) - sum(loads) / world <= biggest
    assert R.partition_by_cost([(64, 4)] * 4, 2) == [[0, 2], [1, 3]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, shapes, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        parts = R.partition_by_cost(shapes, world)
        local = {i: ("solved", i, rank) for i in parts[rank]}       # stands in for this rank's solves
        merged = R.gather_results(local, parts)
        step = R.max_over_ranks(1.5 + rank)
        dist.barrier()
        out.put((rank, parts, merged, step))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_a_ragged_batch():
    shapes = ragged_shapes(40, seed=11)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, shapes, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, parts0, merged0, step0), (r1, parts1, merged1, step1) = res
    assert parts0 == parts1 == R.partition_by_cost(shapes, 2)      # the same plan on every rank
    assert merged0 == merged1 and [m[1] for m in merged0] == list(range(40))
    assert {m[2] for m in merged0} == {0, 1}
    assert step0 == step1 == 2.5                                  # the slower rank's time


def test_single_process_paths():
    assert R.max_over_ranks(3.25) == 3.25
    parts = R.partition_by_cost([(32, 2), (64, 8)], 1)
    assert R.gather_results({0: "a", 1: "b"}, parts) == ["a", "b"]
    with pytest.raises(RuntimeError):
        R.gather_results({0: "a"}, parts)
