"""CPU FP64 oracle for the batched dual Newton–CG symplectic Stiefel projection.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm of
``bench.py`` may use it, and only as the checker (or as the timed CPU
baseline), never as the thing measured or shipped.

It is a plain torch-FP64 restatement of the reference solver
``symplectic_projection.solve`` (yulinxie20/symplectic-stiefel-nearness) and
of its independent acceptance checker ``inspect_output``.  Every function
cites the reference file:line it follows (paths relative to the reference
project root).  Pinning: ``tests/golden/make_golden.py`` runs the reference's
own ``dual_batch`` / ``inspect_output`` (imported in a container that has the
reference) and stores the results under ``tests/golden``; ``tests/test_oracle.py``
checks this restatement against those fixtures.

Problem: given T (2n x 2k, FP64) find X minimising ||X - T||_F^2 subject to
X^T J_2n X = J_2k with J_2r = [[0, I_r], [-I_r, 0]].  Notation m = 2k,
A = T[:n], D = T[n:].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

# src/symplectic_projection/dual_recommended_hvp.py:13-16
ROW_CHUNK = 1024
FEAS_TOL = 1e-8
MAX_NEWTON, MAX_CG, MAX_BACKTRACK = 100, 150, 40
ARMIJO = 1e-4                      # dual_recommended_hvp.py:180
BASE_SEED = 2026102100             # reproduce.py:21
THRESHOLDS = {"feasibility": 1e-8, "stationarity": 1e-9, "delta": 1e-8}  # reproduce.py:28


# --------------------------------------------------------------------------
# inputs
# --------------------------------------------------------------------------
def make_inputs(n: int, k: int, case_index: int, count: int, base_seed: int = BASE_SEED):
    """Seeded Gaussian targets, entries N(0, 1/(2n)).

    Follows src/symplectic_projection/experiment.py:43-51: target j of case
    ``case_index`` uses seed base_seed + 1000*case_index + j and one
    ``torch.randn(2n, 2k)`` draw from a CPU generator, divided by sqrt(2n).
    """
    seeds = [base_seed + 1000 * case_index + j for j in range(count)]
    out = torch.empty(count, 2 * n, 2 * k, dtype=torch.float64)
    for j, seed in enumerate(seeds):
        gen = torch.Generator(device="cpu").manual_seed(seed)
        out[j] = torch.randn(2 * n, 2 * k, dtype=torch.float64, generator=gen) / math.sqrt(2 * n)
    return out, seeds


# protocol case positions, reproduce.py:14-15 (n-major over n in (2048,4096), k in (16,32,48))
def protocol_case_index(n: int, k: int) -> int:
    return [(a, b) for a in (2048, 4096) for b in (16, 32, 48)].index((n, k))


# --------------------------------------------------------------------------
# small helpers, dual_recommended_hvp.py:22-36
# --------------------------------------------------------------------------
def swap_rows(x: torch.Tensor) -> torch.Tensor:
    """J applied from the left: [x_bottom; -x_top] (dual_recommended_hvp.py:22-24)."""
    h = x.shape[-2] // 2
    return torch.cat((x[..., h:, :], -x[..., :h, :]), dim=-2)


def skew(a: torch.Tensor) -> torch.Tensor:
    return (a - a.mT) / 2


def frob_inner(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return (a * b).sum(dim=(-2, -1))


def frob_norm(a: torch.Tensor) -> torch.Tensor:
    return torch.linalg.vector_norm(a, dim=(-2, -1))


# --------------------------------------------------------------------------
# kernel-level operations (the reference's CUDA wrappers, restated)
# --------------------------------------------------------------------------
def gram(T: torch.Tensor):
    """Cr = A^T A + D^T D and Ci = A^T D - D^T A.

    gram_triangle_reflect.py:19-36 / gram_triangle_reflect.cu:2-13 accumulate
    these over 1024-row chunks (dual_recommended_hvp.py:79-96); the sum is
    the same Gram over all n rows.
    """
    n = T.shape[-2] // 2
    A, D = T[..., :n, :], T[..., n:, :]
    Cr = A.mT @ A + D.mT @ D
    AD = A.mT @ D
    Ci = AD - AD.mT
    return Cr, Ci


def recover(A, D, P, Q):
    """Ur = A P^T + D Q^T, Ui = D P^T - A Q^T (recovery_fused.cu:2-41)."""
    return A @ P.mT + D @ Q.mT, D @ P.mT - A @ Q.mT


def sandwich_front(values, Ci, P, Q):
    """Yr = P diag(values) - Q Ci, Yi = P Ci + Q diag(values) (hvp_fused.cu:41-80)."""
    return P * values[..., None, :] - Q @ Ci, P @ Ci + Q * values[..., None, :]


def sandwich(values, Ci, P, Q):
    """S = K^-1 (Lambda + i Ci) K^-1 split into (sym Re, skew Im); dual_recommended_hvp.py:67-71."""
    Yr, Yi = sandwich_front(values, Ci, P, Q)
    Sr, Si = recover(Yr, Yi, P, Q)
    return (Sr + Sr.mT) / 2, skew(Si)


def hvp(P, Q, Sr, Si, E):
    """H(E) = Z - Z^T with Z = P (E Sr) - Q (E Si); dual_recommended_hvp.py:74-76, hvp_fused.cu:2-148."""
    Z = P @ (E @ Sr) - Q @ (E @ Si)
    return Z - Z.mT


def precondition(R, denominator):
    """skew(R / (lambda_i + lambda_j)) reading both positions (hvp_fused.cu:374-387)."""
    a = R / denominator
    return (a - a.mT) * 0.5


def line_change(gradient, delta, V, dSr, trial, dSi):
    """Exact dual-objective change of a trial step (hvp_fused.cu:259-371).

    change = <gradient, delta> + <V, dSr + trial @ dSi>.
    """
    first = frob_inner(gradient, delta)
    tail = frob_inner(V, dSr + trial @ dSi)
    return first + tail


def inverse_from_factor(L):
    """(L L^T)^-1 (cholesky_solve(I, L), dual_recommended_hvp.py:39-43; cholesky_inverse_kernel.cu)."""
    eye = torch.eye(L.shape[-1], dtype=L.dtype).expand_as(L)
    return torch.cholesky_solve(eye, L)


# --------------------------------------------------------------------------
# the dual Newton–CG, dual_recommended_hvp.py:99-191
# --------------------------------------------------------------------------
@dataclass
class DualStats:
    newton_steps: int = 0          # batched Newton iterations executed (incl. the final check)
    hvps: int = 0                  # batched Hessian-vector products
    trials: int = 0                # batched line-search trials
    cg_per_step: list = field(default_factory=list)


def adaptive_denominator(P, Q, Sr, Si):
    """Diagonal of the Hessian H(E) = Z - Z^T, Z = P E Sr - Q E Si, on the skew basis
    e_i e_j^T - e_j e_i^T:  P_ii Sr_jj + P_jj Sr_ii - 2 P_ij Sr_ij + 2 Q_ij Si_ij.

    NOT part of the reference: the restatement of this build's adaptive
    preconditioner (preconditioner="adaptive").  At omega = 0 (P = I, Q = 0,
    Sr = diag(lambda)) it equals the reference's lambda_i + lambda_j.
    """
    dP, dS = P.diagonal(dim1=-2, dim2=-1), Sr.diagonal(dim1=-2, dim2=-1)
    return dP[..., :, None] * dS[..., None, :] + dP[..., None, :] * dS[..., :, None] - 2 * P * Sr + 2 * Q * Si


@torch.no_grad()
def dual_batch(Cr: torch.Tensor, Ci: torch.Tensor, stats: DualStats | None = None,
               max_newton: int = MAX_NEWTON, max_cg: int = MAX_CG,
               max_backtrack: int = MAX_BACKTRACK, preconditioner: str = "eigenbasis"):
    """Dual Newton–CG in the eigenbasis of the scaled Cr.

    Returns (omega, L, P, Q, iterations) in the original basis, where
    P + iQ = (I + i omega)^-1 is the inverse cached at the accepted step and
    L = chol(I + omega omega).  Raises RuntimeError on the Newton or
    line-search cap, like dual_recommended_hvp.py:189-191.
    preconditioner="eigenbasis" is the reference's; "adaptive" is this build's
    extension (``adaptive_denominator``, entries that are not positive fall back
    to lambda_i + lambda_j), used for the CG steps.
    """
    batch, m, _ = Cr.shape
    eye = torch.eye(m, dtype=Cr.dtype).expand(batch, m, m)
    omega = torch.zeros_like(Cr)
    L = eye.clone()
    P = eye.clone()
    # scaling and eigenbasis, :106-111
    scale = (Cr.diagonal(dim1=-2, dim2=-1).sum(-1) / m).clamp_min(1.0)
    Cr = Cr / scale[:, None, None]
    Ci = Ci / scale[:, None, None]
    values, vectors = torch.linalg.eigh(Cr)
    den = values[:, :, None] + values[:, None, :]
    Ci_e = skew(vectors.mT @ Ci @ vectors)                     # :53-56
    J_e = skew(vectors.mT @ swap_rows(vectors)) / scale[:, None, None]

    active = torch.ones(batch, dtype=torch.bool)
    iterations = torch.zeros(batch, dtype=torch.int64)
    for newton_step in range(max_newton):
        if stats is not None:
            stats.newton_steps += 1
        if newton_step == 0:
            Q = torch.zeros_like(omega)
            Sr, Si = torch.diag_embed(values), Ci_e
        else:
            Q = -omega @ P
            Sr, Si = sandwich(values, Ci_e, P, Q)
        g = J_e - Si                                             # :126
        gnorm = frob_norm(g)
        residual = gnorm * scale / math.sqrt(m)                  # :128
        active &= residual >= FEAS_TOL / 2
        if not bool(active.any()):
            # from_eigenbasis, :58-64
            omega_o = skew(vectors @ omega @ vectors.mT)
            P_o = vectors @ P @ vectors.mT
            Q_o = vectors @ Q @ vectors.mT
            L_o = torch.linalg.cholesky(eye + omega_o @ omega_o)
            return omega_o, L_o, P_o, Q_o, iterations
        iterations += active.to(torch.int64)

        masked_neg_g = torch.where(active[:, None, None], -g, torch.zeros_like(g))
        if newton_step == 0:                                     # :138-140
            first_z = precondition(masked_neg_g, den)
            direction = first_z
            if stats is not None:
                stats.cg_per_step.append(0)
        else:                                                    # :142-161
            den_s = den
            if preconditioner == "adaptive":
                den_a = adaptive_denominator(P, Q, Sr, Si)
                den_s = torch.where(den_a > 0, den_a, den)
            direction = torch.zeros_like(g)
            r = masked_neg_g
            z = precondition(r, den_s)
            first_z = z
            p = z.clone()
            rz = frob_inner(r, z)
            tol = residual.sqrt().clamp(1e-8, 0.1) * gnorm
            cg_on = active.clone()
            cg_count = 0
            for _ in range(max_cg):
                Hp = hvp(P, Q, Sr, Si, p)
                cg_count += 1
                curvature = frob_inner(p, Hp)
                cg_on &= curvature > 0
                alpha = torch.where(cg_on, rz / torch.where(cg_on, curvature, torch.ones_like(curvature)),
                                    torch.zeros_like(rz))
                direction = direction + alpha[:, None, None] * p
                r = r - alpha[:, None, None] * Hp
                cg_on &= frob_norm(r) > tol
                if not bool(cg_on.any()):
                    break
                z = precondition(r, den_s)
                rz_next = frob_inner(r, z)
                beta = rz_next / torch.where(cg_on, rz, torch.ones_like(rz))
                p = torch.where(cg_on[:, None, None], z + beta[:, None, None] * p, torch.zeros_like(p))
                rz = rz_next
            if stats is not None:
                stats.hvps += cg_count
                stats.cg_per_step.append(cg_count)
        # non-descent fallback, :163-164
        fallback = active & (frob_inner(g, direction) >= 0)
        direction = torch.where(fallback[:, None, None], first_z, direction)

        # Armijo backtracking with exact change, :167-190
        slope = frob_inner(g, direction)
        step = torch.ones_like(slope)
        pending = active.clone()
        for _ in range(max_backtrack):
            if stats is not None:
                stats.trials += 1
            delta = torch.where(pending, step, torch.zeros_like(step))[:, None, None] * direction
            trial = skew(omega + delta)
            new_L, info = torch.linalg.cholesky_ex(eye + trial @ trial)
            valid = info == 0
            safe_L = torch.where(valid[:, None, None], new_L, L)
            P_trial = inverse_from_factor(safe_L)
            V = P_trial @ delta
            change = line_change(g, delta, V, delta @ Sr, trial, delta @ Si)
            accept = pending & valid & (change <= ARMIJO * step * slope)
            omega = torch.where(accept[:, None, None], trial, omega)
            L = torch.where(accept[:, None, None], new_L, L)
            P = torch.where(accept[:, None, None], P_trial, P)
            pending &= ~accept
            if not bool(pending.any()):
                break
            step = torch.where(pending, step / 2, step)
        else:
            raise RuntimeError("batched line search found no descent step")
    raise RuntimeError("batched Newton iteration cap reached")


@torch.no_grad()
def solve(T: torch.Tensor, stats: DualStats | None = None, **caps):
    """CPU FP64 (X, omega, iterations) for T [B, 2n, 2k]; dual_recommended_hvp.py:231-242."""
    if T.dtype != torch.float64 or T.ndim != 3:
        raise ValueError("T must be float64 [batch, 2n, 2k]")
    n = T.shape[-2] // 2
    Cr, Ci = gram(T)
    omega, L, P, Q, iterations = dual_batch(Cr, Ci, stats, **caps)
    Ur, Ui = recover(T[:, :n], T[:, n:], P, Q)               # recover_matmul, :194-228
    X = torch.cat((Ur, Ui), dim=-2)
    return X, omega, iterations


# --------------------------------------------------------------------------
# independent acceptance check, experiment.py:105-137 and baselines/geometry.py
# --------------------------------------------------------------------------
def _projection_with_multiplier(y: torch.Tensor, value: torch.Tensor):
    """baselines/geometry.py:22-40: project ``value`` onto the tangent space at y."""
    g = y.mT @ y
    values, vectors = torch.linalg.eigh((g + g.mT) / 2)
    if not bool(torch.isfinite(values).all()) or float(values.min()) <= 0:
        raise FloatingPointError("Gram matrix at the base point is not positive definite")
    den = values[:, None] + values[None, :]
    jy = swap_rows(y)
    coupling = jy.mT @ value
    rhs = coupling - coupling.mT
    rotated = vectors.mT @ rhs @ vectors
    multiplier = skew(vectors @ (rotated / den) @ vectors.mT)
    return value - jy @ multiplier, multiplier


@torch.no_grad()
def inspect_output(target: torch.Tensor, x: torch.Tensor):
    """Per-instance r_F (feasibility), r_G (stationarity), delta (duality gap).

    Restates src/symplectic_projection/experiment.py:105-137.  Pass test:
    finite and r_F <= 1e-8, r_G <= 1e-9, delta <= 1e-8 (reproduce.py:28).
    """
    records = []
    m, n = target.shape[-1], target.shape[-2] // 2
    jm = swap_rows(torch.eye(m, dtype=torch.float64))
    ident = torch.eye(m, dtype=torch.complex128)
    for index in range(len(target)):
        rec = dict(index=index, feasibility=None, stationarity=None, delta=None)
        try:
            t, y = target[index].to(torch.float64), x[index].to(torch.float64)
            if y.shape != t.shape or not bool(torch.isfinite(y).all()):
                raise ValueError("output has the wrong shape or non-finite values")
            err = y - t
            objective = float((err * err).sum())
            tscale = max(1.0, float(torch.linalg.vector_norm(t)))
            rec["feasibility"] = float(torch.linalg.vector_norm(y.T @ swap_rows(y) - jm) / math.sqrt(m))
            grad, mult = _projection_with_multiplier(y, 2 * err)
            omega = mult / 2
            if not bool(torch.isfinite(grad).all() and torch.isfinite(omega).all()):
                raise FloatingPointError("projected gradient or multiplier not finite")
            rec["stationarity"] = float(torch.linalg.vector_norm(grad) / (2 * tscale))
            factor = torch.linalg.cholesky(ident + 1j * omega)
            b = torch.complex(t[:n], t[n:])
            solved = torch.linalg.solve_triangular(factor, b.mH, upper=False)
            dual = float((t * t).sum() - (solved.abs() ** 2).sum() - (omega * jm).sum())
            rec["delta"] = abs((objective - dual) / max(1.0, abs(objective)))
        except Exception as exc:  # recorded, like the reference
            rec["exception"] = f"{type(exc).__name__}: {exc}"
        records.append(rec)
    return records


def passes(record, thresholds=THRESHOLDS) -> bool:
    """experiment.py:100-102."""
    return all(record.get(key) is not None and math.isfinite(record[key])
               and abs(record[key]) <= tol for key, tol in thresholds.items())


def worst(records):
    """Largest r_F, r_G, delta over a batch (None entries count as inf)."""
    out = {}
    for key in THRESHOLDS:
        vals = [r.get(key) for r in records]
        out[key] = max((float("inf") if v is None else v) for v in vals)
    return out


# --------------------------------------------------------------------------
# gradient through the solve (no counterpart in the reference, whose solve runs
# under torch.no_grad, dual_recommended_hvp.py:231): three independent routes
# --------------------------------------------------------------------------
def _loss(T, G, Gw=None):
    X, omega, _ = solve(T)
    val = frob_inner(G, X)
    if Gw is not None:
        val = val + frob_inner(Gw, omega)
    return val


def adjoint_formula(T: torch.Tensor, G: torch.Tensor, Gw: torch.Tensor | None = None) -> torch.Tensor:
    """dL/dT for L = <G, X*(T)> + <Gw, omega(T)>, by implicit differentiation of the dual.

    Complex form: b = A + iD, g = G_top + i G_bottom, K = (I + i omega)^-1, S = K b^H b K.
    omega solves Im(S) = J_m; differentiating, H(d omega) = Im(K dC K) with
    H(E) = Z - Z^T, Z = Re(K E S) (the solver's HVP).  Then
      Gamma = -skew(Im(K g^H b K)) + skew(Gw),  H mu = Gamma (dense solve here),
      dL/db = g K + 2i b K mu K,  dL/dT = [Re; Im].
    """
    _, omega, _ = solve(T)
    B, rows, m = T.shape
    n = rows // 2
    b = torch.complex(T[:, :n], T[:, n:])
    g = torch.complex(G[:, :n], G[:, n:])
    eye = torch.eye(m, dtype=torch.complex128)
    K = torch.linalg.inv(eye + 1j * omega.to(torch.complex128))
    S = K @ (b.mH @ b) @ K
    Sr, Si = (S.real + S.real.mT) / 2, skew(S.imag)
    P, Q = K.real, K.imag
    R = K @ (g.mH @ b) @ K
    Gamma = -skew(R.imag)
    if Gw is not None:
        Gamma = Gamma + skew(Gw)
    iu = torch.triu_indices(m, m, 1)
    p = iu.shape[1]
    mu = torch.zeros(B, m, m, dtype=torch.float64)
    for inst in range(B):
        cols = []
        for c in range(p):
            E = torch.zeros(m, m, dtype=torch.float64)
            E[iu[0, c], iu[1, c]] = 1.0
            E[iu[1, c], iu[0, c]] = -1.0
            HE = hvp(P[inst], Q[inst], Sr[inst], Si[inst], E)
            cols.append(HE[iu[0], iu[1]])
        Hm = torch.stack(cols, dim=1)
        coef = torch.linalg.solve(Hm, Gamma[inst][iu[0], iu[1]])
        mu[inst][iu[0], iu[1]] = coef
        mu[inst][iu[1], iu[0]] = -coef
    N = 2j * K @ mu.to(torch.complex128) @ K
    grad = g @ K + b @ N
    return torch.cat((grad.real, grad.imag), dim=-2)


def adjoint_fd(T, G, Gw=None, direction=None, h=1e-6, seed=0):
    """Central difference (L(T + hV) - L(T - hV)) / 2h along V (seeded Gaussian when None), per instance."""
    if direction is None:
        gen = torch.Generator().manual_seed(seed)
        direction = torch.randn(T.shape, dtype=torch.float64, generator=gen)
    return (_loss(T + h * direction, G, Gw) - _loss(T - h * direction, G, Gw)) / (2 * h), direction


def adjoint_kkt(T: torch.Tensor, G: torch.Tensor) -> torch.Tensor:
    """dL/dT for L = <G, X*(T)> from the dense KKT system of the primal problem.

    Stationarity of 1/2 ||X - T||^2 + 1/2 <Lam, X^T J X - J_m> (Lam skew) is
    F1 = X - T - J X Lam = 0, feasibility F2 = upper(X^T J X - J_m) = 0.  With
    z = (X, upper(Lam)), dL/dT is the X block of w solving (dF/dz)^T w = (G, 0).
    Small sizes only (dense (2nm + m(m-1)/2)^2 system).
    """
    X, _, _ = solve(T)
    B, rows, m = T.shape
    iu = torch.triu_indices(m, m, 1)
    jm = swap_rows(torch.eye(m, dtype=torch.float64))
    out = torch.empty_like(T)
    for inst in range(B):
        t, x = T[inst], X[inst]
        jx = swap_rows(x)
        lam = torch.linalg.lstsq(jx, x - t).solution
        lam = skew(lam)
        z0 = torch.cat((x.reshape(-1), lam[iu[0], iu[1]]))

        def F(z, t=t):
            xx = z[: rows * m].reshape(rows, m)
            L = torch.zeros(m, m, dtype=torch.float64)
            L = L.index_put((iu[0], iu[1]), z[rows * m:])
            L = L - L.mT
            f1 = xx - t - swap_rows(xx) @ L
            f2 = (xx.mT @ swap_rows(xx) - jm)[iu[0], iu[1]]
            return torch.cat((f1.reshape(-1), f2))

        Jz = torch.autograd.functional.jacobian(F, z0)
        rhs = torch.cat((G[inst].reshape(-1), torch.zeros(iu.shape[1], dtype=torch.float64)))
        w = torch.linalg.solve(Jz.mT, rhs)
        out[inst] = w[: rows * m].reshape(rows, m)
    return out
