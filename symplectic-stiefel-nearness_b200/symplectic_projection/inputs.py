"""Seeded synthetic targets with the reference protocol's generator rule.

Target j of protocol case ``case_index`` draws ``torch.randn(2n, 2k)`` from a
CPU generator seeded with base_seed + 1000*case_index + j and divides by
sqrt(2n) (src/symplectic_projection/experiment.py:43-51, base seed 2026102100
at reproduce.py:21), i.e. i.i.d. N(0, 1/(2n)) entries.
"""
from __future__ import annotations

import math

import torch

BASE_SEED = 2026102100
PROTOCOL_CASES = [(n, k) for n in (2048, 4096) for k in (16, 32, 48)]   # reproduce.py:14-15


def case_index(n: int, k: int) -> int:
    """Position of (n, k) in the protocol's case list (n-major)."""
    return PROTOCOL_CASES.index((n, k))


def gaussian_targets(n: int, k: int, count: int, case: int, base_seed: int = BASE_SEED,
                     pin_memory: bool = False) -> torch.Tensor:
    out = torch.empty(count, 2 * n, 2 * k, dtype=torch.float64, pin_memory=pin_memory)
    for j in range(count):
        gen = torch.Generator(device="cpu").manual_seed(base_seed + 1000 * case + j)
        out[j] = torch.randn(2 * n, 2 * k, dtype=torch.float64, generator=gen) / math.sqrt(2 * n)
    return out
