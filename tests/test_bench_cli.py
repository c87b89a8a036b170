"""bench.py's launcher on the CPU: ``--gpus N`` runs N ranks, and a mismatched world aborts.

The reference arm needs no GPU (it times the CPU FP64 restatement), so it runs the
same multi-rank path here: ``bench.py --gpus 2`` started without torchrun re-executes
itself under torch.distributed.run with two ranks on 127.0.0.1; rank 0 prints the one
JSON line and the other rank exits 0.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
SMALL = ["--impl", "reference", "--steps", "2", "--warmup", "1", "--batch", "2", "--n", "16", "--k", "2"]


def _run(args, env=None):
    e = dict(os.environ)
    for key in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(key, None)
    e.update(env or {})
    e["OMP_NUM_THREADS"] = "1"
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=300)


def _lines(out):
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def test_gpus_two_launches_two_ranks():
    res = _run(["--gpus", "2", *SMALL])
    assert res.returncode == 0, res.stderr[-2000:]
    lines = _lines(res.stdout)
    assert len(lines) == 1, res.stdout                       # rank 0 alone prints
    line = lines[0]
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2 and line["ranks_launched"] == 2
    assert line["steps"] == 2 and line["warmup"] == 1        # the arm honours --steps / --warmup
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_single_rank_runs_in_process():
    res = _run(["--gpus", "1", *SMALL])
    assert res.returncode == 0, res.stderr[-2000:]
    (line,) = _lines(res.stdout)
    assert line["n_gpus"] == 1 and line["ranks_launched"] == 1


def test_world_size_mismatch_aborts():
    res = _run(["--gpus", "2", *SMALL], env={"WORLD_SIZE": "3", "RANK": "0"})
    assert res.returncode != 0
    assert "WORLD_SIZE=3" in res.stderr
