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


# ---------------------------------------------------------------- recovery
def _recover_split(T, P, Q):
    from symplectic_projection.recovery_fused import recover_block
    n = T.shape[1] // 2
    Td = T.cuda()
    Ur, Ui = recover_block(Td[:, :n], Td[:, n:], P.cuda(), Q.cuda(), precision="split")
    torch.cuda.synchronize()
    return Ur.cpu(), Ui.cpu()


def _pq(batch, m, scale, seed):
    """P, Q of a skew omega of the given size: P + iQ = (I + i omega)^-1."""
    g = torch.Generator().manual_seed(seed)
    W = torch.randn(batch, m, m, generator=g, dtype=torch.float64) * scale
    W = (W - W.mT) / 2
    P = torch.linalg.inv(torch.eye(m, dtype=torch.float64) + W @ W)
    return P, -W @ P


@pytest.mark.parametrize("n,k,batch,scale", [(77, 4, 2, 0.1), (512, 12, 3, 0.02), (4096, 48, 2, 0.02),
                                             (333, 64, 2, 0.5), (100, 1, 3, 1.0), (1000, 20, 2, 3.0)])
def test_ozaki_recover_error_bound(n, k, batch, scale):
    T, _ = O.make_inputs(n, k, 2, batch)
    m = 2 * k
    P, Q = _pq(batch, m, scale, n + k)
    Ur, Ui = _recover_split(T, P, Q)
    Ur64, Ui64 = O.recover(T[:, :n], T[:, n:], P, Q)
    # rows [P | Q] (Ur) and [-Q | P] (Ui): per-entry bound from the row maxima of both factors
    W = torch.cat((T[:, :n], T[:, n:]), dim=2)                       # [batch, n, 2m]
    B1 = torch.cat((P, Q), dim=2)
    B2 = torch.cat((-Q, P), dim=2)
    wmax = W.abs().amax(dim=2)                                       # [batch, n]
    bound1 = 2 * (2 * m) * 2.0 ** -45 * wmax[:, :, None] * B1.abs().amax(dim=2)[:, None, :] + 1e-300
    bound2 = 2 * (2 * m) * 2.0 ** -45 * wmax[:, :, None] * B2.abs().amax(dim=2)[:, None, :] + 1e-300
    ulp = 2.0 ** -52 * (Ur64.abs() + 1e-300)
    assert bool(((Ur - Ur64).abs() <= bound1 + 4 * ulp).all())
    assert bool(((Ui - Ui64).abs() <= bound2 + 4 * 2.0 ** -52 * Ui64.abs()).all())


def test_ozaki_recover_identity_within_digit_rounding():
    # P = I, Q = 0: X = T up to the rounding of each row to 46 fraction bits of its largest entry
    T, _ = O.make_inputs(300, 8, 3, 2)
    m = 16
    P = torch.eye(m, dtype=torch.float64).expand(2, m, m).contiguous()
    Q = torch.zeros(2, m, m, dtype=torch.float64)
    Ur, Ui = _recover_split(T, P, Q)
    W = torch.cat((T[:, :300], T[:, 300:]), dim=2)
    tol = 2.0 ** -46 * W.abs().amax(dim=2, keepdim=True)
    assert bool(((Ur - T[:, :300]).abs() <= tol).all()) and bool(((Ui - T[:, 300:]).abs() <= tol).all())


def test_ozaki_recover_nonfinite_row_is_flagged():
    T, _ = O.make_inputs(200, 6, 4, 2)
    T[1, 17, 3] = float("nan")
    P, Q = _pq(2, 12, 0.1, 5)
    Ur, Ui = _recover_split(T, P, Q)
    assert not bool(torch.isfinite(Ur[1, 17]).all())
    assert bool(torch.isfinite(Ur[0]).all()) and bool(torch.isfinite(Ui[0]).all())
    Ur64, _ = O.recover(T[:1, :200], T[:1, 200:], P[:1], Q[:1])
    assert float((Ur[0] - Ur64[0]).abs().max()) < 1e-12
