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


ILLCOND_SEED = 2026102500


def illcond_targets(n: int, k: int, count: int, seed: int = ILLCOND_SEED,
                    pin_memory: bool = False) -> torch.Tensor:
    """Ill-conditioned stress targets T = U diag(s) V^T.

    U (2n x 2k) and V (2k x 2k) have orthonormal columns from QR factors of
    Gaussian matrices, s is log-uniform in [1e-2, 1e2], and every target is
    scaled so that ||T||_F^2 = 2k.  One CPU generator seeded with ``seed``
    draws all targets in order.  The reference's dual Newton-CG stalls on these
    (its CG saturates and the Newton cap is reached); the adaptive
    preconditioner keeps them converging.
    """
    gen = torch.Generator(device="cpu").manual_seed(seed)
    out = torch.empty(count, 2 * n, 2 * k, dtype=torch.float64, pin_memory=pin_memory)
    lo, hi = math.log(1e-2), math.log(1e2)
    for j in range(count):
        U, _ = torch.linalg.qr(torch.randn(2 * n, 2 * k, generator=gen, dtype=torch.float64))
        V, _ = torch.linalg.qr(torch.randn(2 * k, 2 * k, generator=gen, dtype=torch.float64))
        s = torch.exp(torch.empty(2 * k, dtype=torch.float64).uniform_(lo, hi, generator=gen))
        T = U @ torch.diag(s) @ V.T
        out[j] = T * (math.sqrt(2 * k) / torch.linalg.norm(T))
    return out


RAGGED_SEED = 2026102300
RAGGED_N = (512, 1024, 2048, 4096, 8192)
RAGGED_K = (8, 16, 24, 32, 48, 64)


def ragged_shapes(count: int = 384, seed: int = RAGGED_SEED):
    """(n, k) of each target of the ragged workload: n uniform over RAGGED_N and k
    uniform over RAGGED_K, drawn by one CPU generator seeded with ``seed``."""
    gen = torch.Generator(device="cpu").manual_seed(seed)
    ni = torch.randint(0, len(RAGGED_N), (count,), generator=gen).tolist()
    ki = torch.randint(0, len(RAGGED_K), (count,), generator=gen).tolist()
    return [(RAGGED_N[a], RAGGED_K[b]) for a, b in zip(ni, ki)]


def ragged_targets(count: int = 384, seed: int = RAGGED_SEED, shapes=None):
    """Targets of the ragged workload: target j is N(0, 1/(2n_j)) of shape [2n_j, 2k_j]
    from a CPU generator seeded with seed + 1 + j (the reference generator's rule,
    with per-target seeds)."""
    shapes = shapes if shapes is not None else ragged_shapes(count, seed)
    out = []
    for j, (n, k) in enumerate(shapes):
        gen = torch.Generator(device="cpu").manual_seed(seed + 1 + j)
        out.append(torch.randn(2 * n, 2 * k, dtype=torch.float64, generator=gen) / math.sqrt(2 * n))
    return out
