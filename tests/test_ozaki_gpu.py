"""The split-precision (INT8 Ozaki, tcgen05) Gram products against FP64 references.

Every value x of column j in a row chunk is written as F = rint(x 2^(46-E_j))
in six balanced 8-bit digits (|x| < 2^E_j over the chunk); the 21 digit pairs
with p + q <= 5 are accumulated exactly in INT32 and recombined in FP64.
Per entry the error is then at most about K 2^-45 M_i M_j (K summed rows,
M_i the largest |entry| of column i), and for random data it is far smaller.
Integer-valued inputs with few significant bits are represented exactly by the
top digits, so their Gram must come out exact.
"""
from __future__ import annotations

import math

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu


def _gram_split(T):
    from symplectic_projection.gram_triangle_reflect import gram
    n = T.shape[1] // 2
    Td = T.cuda()
    Cr, Ci = gram(Td[:, :n], Td[:, n:], precision="split")
    torch.cuda.synchronize()
    return Cr.cpu(), Ci.cpu()


@pytest.mark.parametrize("n,k,batch", [(5, 1, 3), (77, 4, 2), (512, 12, 3), (1000, 16, 2), (2048, 48, 2),
                                       (333, 64, 2), (4096, 48, 3), (64, 3, 4)])
def test_ozaki_gram_error_bound(n, k, batch):
    T, _ = O.make_inputs(n, k, 1, batch)
    Cr, Ci = _gram_split(T)
    Cr64, Ci64 = O.gram(T)
    # rigorous per-entry bound: 2n rows summed, column maxima over the whole instance
    M = T.abs().amax(dim=1)                                   # [batch, m]
    bound = 2 * (2 * n) * 2.0 ** -45 * M[:, :, None] * M[:, None, :]
    assert bool(((Cr - Cr64).abs() <= bound).all())
    assert bool(((Ci - Ci64).abs() <= bound).all())
    # typical error: Frobenius-relative well below FP64 needs of the solver
    assert float(torch.linalg.vector_norm(Cr - Cr64) / torch.linalg.vector_norm(Cr64)) < 1e-11
    assert float(torch.linalg.vector_norm(Ci - Ci64) / torch.linalg.vector_norm(Cr64)) < 1e-11
    # structure: Cr exactly symmetric, Ci exactly antisymmetric
    assert torch.equal(Cr, Cr.mT) and torch.equal(Ci, -Ci.mT)


@pytest.mark.parametrize("n,k", [(300, 8), (4096, 48), (97, 64)])
def test_ozaki_gram_exact_on_short_integers(n, k):
    g = torch.Generator().manual_seed(n * 131 + k)
    T = torch.randint(-1000, 1001, (2, 2 * n, 2 * k), generator=g).double()
    T[:, :, 1] *= 2.0 ** -20                                  # power-of-two column scaling stays exact
    Cr, Ci = _gram_split(T)
    # every product and partial sum is a multiple of 2^-20 below 2^33: FP64 is exact in any order
    Cr_ref, Ci_ref = O.gram(T)
    assert torch.equal(Cr, Cr_ref)
    assert torch.equal(Ci, Ci_ref)


def test_ozaki_gram_graded_columns():
    # columns spanning 1e-150 .. 1e150: per-column scales keep the relative accuracy
    T, _ = O.make_inputs(256, 8, 2, 2)
    scales = torch.logspace(-150, 150, 16, dtype=torch.float64)
    T = T * scales
    Cr, Ci = _gram_split(T)
    Cr64, Ci64 = O.gram(T)
    d = torch.sqrt(Cr64.diagonal(dim1=-2, dim2=-1))
    norm = d[:, :, None] * d[:, None, :]
    assert float(((Cr - Cr64).abs() / norm).max()) < 1e-10
    assert float(((Ci - Ci64).abs() / norm).max()) < 1e-10


def test_ozaki_gram_nonfinite_poisons_only_its_instance():
    T, _ = O.make_inputs(128, 8, 3, 3)
    T[1, 40, 5] = float("inf")
    Cr, Ci = _gram_split(T)
    assert bool(torch.isfinite(Cr[0]).all()) and bool(torch.isfinite(Cr[2]).all())
    assert not bool(torch.isfinite(Cr[1]).all())
    Cr64, _ = O.gram(T[[0, 2]])
    assert float((Cr[[0, 2]] - Cr64).abs().max()) < 1e-12


def test_ozaki_gram_zero_and_tiny_columns():
    T, _ = O.make_inputs(100, 4, 4, 2)
    T[:, :, 0] = 0.0
    T[:, :, 3] *= 1e-300
    Cr, Ci = _gram_split(T)
    Cr64, Ci64 = O.gram(T)
    assert bool(torch.isfinite(Cr).all())
    assert torch.equal(Cr[:, 0], torch.zeros_like(Cr[:, 0]))
    scale = Cr64.abs().amax()
    assert float((Cr - Cr64).abs().max() / scale) < 1e-12
