"""Each device operation against the CPU FP64 oracle's restatement of it."""
from __future__ import annotations

import pytest
import torch

from oracle import ssn_oracle as O

pytestmark = pytest.mark.gpu

MS = [2, 6, 16, 24, 40, 64, 96, 128]
TOL = 1e-12   # relative, FP64 products of O(1) matrices with different summation order


def rel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))


def rand(batch, m, seed, skew=False, sym=False):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn(batch, m, m, dtype=torch.float64, generator=g)
    if skew:
        x = (x - x.mT) / 2
    if sym:
        x = (x + x.mT) / 2
    return x


@pytest.fixture(scope="module")
def sp():
    import symplectic_projection as sp
    sp.initialize_kernels()
    return sp


@pytest.mark.parametrize("m", MS)
def test_inner_products(sp, m):
    E, Sr, Si = rand(3, m, 1, skew=True), rand(3, m, 2, sym=True), rand(3, m, 3, skew=True)
    U, V = sp.hvp_fused.inner_products(E.cuda(), Sr.cuda(), Si.cuda())
    assert rel(U, E @ Sr) < TOL and rel(V, E @ Si) < TOL


@pytest.mark.parametrize("m", MS)
def test_outer_skew(sp, m):
    P, Q, U, V = rand(3, m, 4, sym=True), rand(3, m, 5, skew=True), rand(3, m, 6), rand(3, m, 7)
    H = sp.hvp_fused.outer_skew(*(x.cuda() for x in (P, Q, U, V)))
    Z = P @ U - Q @ V
    assert rel(H, Z - Z.mT) < TOL
    assert torch.equal(H.cpu(), -H.cpu().mT)


@pytest.mark.parametrize("m", MS)
def test_hvp_matches_oracle(sp, m):
    P, Q, Sr, Si, E = (rand(2, m, 10 + i) for i in range(5))
    U, V = sp.hvp_fused.inner_products(E.cuda(), Sr.cuda(), Si.cuda())
    H = sp.hvp_fused.outer_skew(P.cuda(), Q.cuda(), U, V)
    assert rel(H, O.hvp(P, Q, Sr, Si, E)) < TOL


@pytest.mark.parametrize("m", MS)
def test_sandwich_front(sp, m):
    g = torch.Generator().manual_seed(8)
    values = torch.rand(3, m, dtype=torch.float64, generator=g) + 0.5
    Ci, P, Q = rand(3, m, 9, skew=True), rand(3, m, 10, sym=True), rand(3, m, 11, skew=True)
    Yr, Yi = sp.hvp_fused.sandwich_front(values.cuda(), Ci.cuda(), P.cuda(), Q.cuda())
    wr, wi = O.sandwich_front(values, Ci, P, Q)
    assert rel(Yr, wr) < TOL and rel(Yi, wi) < TOL


@pytest.mark.parametrize("m", MS)
def test_line_change(sp, m):
    xs = [rand(4, m, 20 + i) for i in range(6)]
    got = sp.hvp_fused.line_change(*(x.cuda() for x in xs))
    want = O.line_change(*xs)
    assert torch.allclose(got.cpu(), want, rtol=1e-12, atol=1e-12 * m)


@pytest.mark.parametrize("m", [2, 24, 96, 128])
def test_precondition_and_cg_ops_bitwise(sp, m):
    R = rand(3, m, 30)
    lam = torch.rand(3, m, dtype=torch.float64, generator=torch.Generator().manual_seed(31)) + 0.1
    den = lam[:, :, None] + lam[:, None, :]
    z = sp.hvp_fused.fused_precondition(R.cuda(), den.cuda()).cpu()
    assert torch.equal(z, O.precondition(R, den))          # elementwise, correctly rounded
    d, r, p, Hp = (rand(3, m, 40 + i) for i in range(4))
    alpha = torch.tensor([0.5, -1.25, 3.0], dtype=torch.float64)
    nd, nr = sp.hvp_fused.cg_update(d.cuda(), r.cuda(), p.cuda(), Hp.cuda(), alpha.cuda())
    assert torch.equal(nd.cpu(), d + alpha[:, None, None] * p)
    assert torch.equal(nr.cpu(), r - alpha[:, None, None] * Hp)
    active = torch.tensor([True, False, True])
    out = sp.hvp_fused.cg_next(d.cuda(), p.cuda(), alpha.cuda(), active.cuda()).cpu()
    want = torch.where(active[:, None, None], d + alpha[:, None, None] * p, torch.zeros_like(d))
    assert torch.equal(out, want)


@pytest.mark.parametrize("m", [2, 8, 24, 96, 128])
def test_inverse_from_cholesky(sp, m):
    A = rand(3, m, 50)
    K = A @ A.mT / m + torch.eye(m, dtype=torch.float64)
    L = torch.linalg.cholesky(K)
    P = sp.cholesky_inverse_kernel.inverse_from_cholesky(L.cuda())
    assert rel(P, O.inverse_from_factor(L)) < 1e-12


@pytest.mark.parametrize("m", [2, 8, 24, 96, 128])
def test_spd_inverse_and_pd_flag(sp, m):
    W = rand(4, m, 60, skew=True)
    W = W / torch.linalg.matrix_norm(W, ord=2)[:, None, None]
    W[0] *= 0.5
    W[1] *= 0.999
    W[2] *= 1.5            # I + W W not positive definite
    W[3] *= 0.0
    K = torch.eye(m, dtype=torch.float64) + W @ W
    P, info = sp.cholesky_inverse_kernel.spd_inverse(K.cuda())
    _, ref_info = torch.linalg.cholesky_ex(K)
    assert info.cpu().ne(0).tolist() == ref_info.ne(0).tolist()
    ok = ref_info == 0
    assert rel(P.cpu()[ok], torch.linalg.inv(K[ok])) < 1e-9


@pytest.mark.parametrize("m", [2, 6, 24, 64, 96, 128])
def test_eigh(sp, m):
    from symplectic_projection.dual_recommended_hvp import eigh_scaled
    T, _ = O.make_inputs(max(m, 40), m // 2, 0, 3)
    Cr, _ = O.gram(T)
    Cr = Cr * 3.0   # trace/m > 1 so the scale is exercised
    values, vectors, scale, sweeps = eigh_scaled(Cr.cuda())
    values, vectors, scale = values.cpu(), vectors.cpu(), scale.cpu()
    s = (Cr.diagonal(dim1=-2, dim2=-1).sum(-1) / m).clamp_min(1)
    assert torch.allclose(scale, s, rtol=1e-14)
    A = Cr / s[:, None, None]
    ref = torch.linalg.eigvalsh(A)
    assert torch.allclose(values, ref, rtol=1e-13, atol=1e-14)
    assert torch.all(values[:, 1:] >= values[:, :-1])
    eye = torch.eye(m, dtype=torch.float64)
    assert rel(vectors.mT @ vectors, eye.expand(3, m, m)) < 1e-13
    assert rel(vectors @ torch.diag_embed(values) @ vectors.mT, A) < 1e-13
    assert int(sweeps.max()) < 40


@pytest.mark.parametrize("m,rows", [(2, 5), (24, 48), (40, 100), (96, 256), (96, 4096), (128, 333)])
def test_gram(sp, m, rows):
    T, _ = O.make_inputs(rows, m // 2, 1, 3)
    Cr, Ci = sp.gram_triangle_reflect.gram(T[:, :rows].cuda(), T[:, rows:].cuda())
    wr, wi = O.gram(T)
    assert rel(Cr, wr) < 1e-13 and rel(Ci, wi) < 1e-13
    assert torch.equal(Cr.cpu(), Cr.cpu().mT) and torch.equal(Ci.cpu(), -Ci.cpu().mT)


def test_gram_add_accumulates(sp):
    T, _ = O.make_inputs(50, 6, 2, 2)
    A, D = T[:, :50].cuda(), T[:, 50:].cuda()
    Cr = torch.ones(2, 12, 12, dtype=torch.float64, device="cuda")
    Ci = torch.zeros_like(Cr)
    sp.gram_triangle_reflect.gram_add_(A, D, Cr, Ci)
    wr, wi = O.gram(T)
    assert rel(Cr.cpu(), wr + 1) < 1e-13 and rel(Ci.cpu(), wi) < 1e-13


@pytest.mark.parametrize("m,rows", [(2, 7), (24, 100), (96, 1000), (128, 129), (64, 4096)])
def test_recover_block(sp, m, rows):
    A, D, P, Q = torch.randn(3, rows, m, dtype=torch.float64), torch.randn(3, rows, m, dtype=torch.float64), \
        rand(3, m, 70, sym=True), rand(3, m, 71, skew=True)
    Ur, Ui = sp.recovery_fused.recover_block(A.cuda(), D.cuda(), P.cuda(), Q.cuda())
    wr, wi = O.recover(A, D, P, Q)
    assert rel(Ur, wr) < 1e-13 and rel(Ui, wi) < 1e-13


@pytest.mark.parametrize("m,rows", [(2, 5), (24, 100), (96, 1000), (128, 129), (96, 4096)])
def test_cross_gram(sp, m, rows):
    g = torch.Generator().manual_seed(80 + m)
    Ga, Gd, A, D = (torch.randn(3, rows, m, dtype=torch.float64, generator=g) for _ in range(4))
    Mr, Mi = sp.gram_triangle_reflect.cross_gram(Ga.cuda(), Gd.cuda(), A.cuda(), D.cuda())
    assert rel(Mr, Ga.mT @ A + Gd.mT @ D) < 1e-13
    assert rel(Mi, Ga.mT @ D - Gd.mT @ A) < 1e-13


def test_products_take_the_halves_of_a_stacked_batch_without_a_copy(sp):
    # T[:, :n] and T[:, n:] share one batch stride: the entry points read them in place
    T, _ = O.make_inputs(300, 20, 4, 3)
    Td = T.cuda()
    n = 300
    A, D = Td[:, :n], Td[:, n:]
    from symplectic_projection import _native as N
    a, d, stride = N.row_halves(A, D)
    assert a.data_ptr() == A.data_ptr() and d.data_ptr() == D.data_ptr() and stride == 2 * n * 40
    Cr, Ci = sp.gram_triangle_reflect.gram(A, D)
    wr, wi = O.gram(T)
    assert rel(Cr, wr) < 1e-13 and rel(Ci, wi) < 1e-13
    P, Q = rand(3, 40, 72, sym=True), rand(3, 40, 73, skew=True)
    Ur, Ui = sp.recovery_fused.recover_block(A, D, P.cuda(), Q.cuda())
    vr, vi = O.recover(T[:, :n], T[:, n:], P, Q)
    assert rel(Ur, vr) < 1e-13 and rel(Ui, vi) < 1e-13
    Mr, Mi = sp.gram_triangle_reflect.cross_gram(A, D, D, A)
    assert rel(Mr, T[:, :n].mT @ T[:, n:] + T[:, n:].mT @ T[:, :n]) < 1e-13


@pytest.mark.parametrize("m", [2, 8, 24, 96, 128])
def test_cholesky_k_and_pd_flag(sp, m):
    W = rand(4, m, 90, skew=True)
    W = W / torch.linalg.matrix_norm(W, ord=2)[:, None, None]
    W[0] *= 0.5
    W[1] *= 0.99
    W[2] *= 1.5            # I + W W not positive definite
    W[3] *= 0.0
    K = torch.eye(m, dtype=torch.float64) + W @ W
    L, info = sp.cholesky_inverse_kernel.cholesky_k(W.cuda())
    ref, ref_info = torch.linalg.cholesky_ex(K)
    assert info.cpu().ne(0).tolist() == ref_info.ne(0).tolist()
    ok = ref_info == 0
    L = L.cpu()
    assert torch.equal(L[ok], L[ok].tril())
    assert rel(L[ok], ref[ok]) < 1e-12
    if m > 2:
        bad = int(info[2])
        assert 1 <= bad <= m and bool((L[2][:, bad - 1:] == 0).all())


def test_dual_batch_returns_the_cholesky_factor(sp):
    from symplectic_projection.dual_recommended_hvp import dual_batch
    T, _ = O.make_inputs(64, 8, 6, 3)
    Cr, Ci = O.gram(T)
    final = []
    omega, L, it = dual_batch(Cr.cuda(), Ci.cuda(), final)
    m = omega.shape[-1]
    K = torch.eye(m, dtype=torch.float64) + omega.cpu() @ omega.cpu()
    assert rel(L, torch.linalg.cholesky(K)) < 1e-12


@pytest.mark.parametrize("n,k,B", [(64, 8, 4), (2048, 48, 3)])
def test_certify_matches_the_oracle_acceptance_test(sp, n, k, B):
    from symplectic_projection.certify import certify
    T, _ = O.make_inputs(n, k, 7, B)
    X, _, _ = O.solve(T)
    X = X.clone()
    X[1] += 1e-6 * torch.randn(X[1].shape, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    cert = certify(T.cuda(), X.cuda())
    recs = O.inspect_output(T, X)
    for key in ("feasibility", "stationarity"):
        got = cert[key].cpu()
        want = torch.tensor([r[key] for r in recs], dtype=torch.float64)
        assert torch.allclose(got, want, rtol=1e-6, atol=1e-15), key
    delta = cert["delta"].cpu()
    want = torch.tensor([r["delta"] for r in recs], dtype=torch.float64)
    assert torch.allclose(delta, want, rtol=1e-3, atol=1e-12)
    assert cert["passed"].cpu().tolist() == [O.passes(r) for r in recs]
    assert cert["passed"].cpu().tolist()[1] is False
