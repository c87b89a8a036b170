"""On-device acceptance metrics for a solved batch (FP64).

Computes, per instance, the three quantities of the reference's independent
checker ``inspect_output`` (src/symplectic_projection/experiment.py:105-137):

  r_F   = ||X^T J X - J_m||_F / sqrt(m)
  r_G   = ||P_X(2(X - T))||_F / (2 max(1, ||T||_F))   (tangent projection,
          baselines/geometry.py:22-40)
  delta = |f - f_dual| / max(1, |f|),  f = ||X - T||^2,
          f_dual = ||T||^2 - Re tr((I + i w)^-1 C) - <w, J_m>,  w = multiplier/2,
          C = b^H b with b = T_top + i T_bottom (the same value as the
          reference's ||L^-1 b^H||^2, written through the Gram matrix).

Every tall-skinny contraction runs on this package's FP64 tensor-core kernels:
the Grams of X and T (ssn_gram), the cross product (J X)^T E (ssn_cross_gram)
and the tangent correction [-Yb M; Yt M] (ssn_recover with P = 0, Q = M); so do
the eigendecomposition and the SPD inverse.  The m x m products of the
multiplier's eigenbasis transform and the element-wise norms use torch on the
GPU.  It runs outside any timed region: it is the batch's self-certificate.
"""
from __future__ import annotations

import math

import torch

from .cholesky_inverse_kernel import spd_inverse
from .dual_recommended_hvp import eigh_scaled
from .gram_triangle_reflect import cross_gram, gram
from .recovery_fused import recover_block

THRESHOLDS = {"feasibility": 1e-8, "stationarity": 1e-9, "delta": 1e-8}


@torch.no_grad()
def certify(T: torch.Tensor, X: torch.Tensor) -> dict:
    """Per-instance tensors 'feasibility', 'stationarity', 'delta' and a bool 'passed'."""
    if T.shape != X.shape or not T.is_cuda or not X.is_cuda:
        raise ValueError("T and X must be CUDA tensors of the same shape")
    batch, rows, m = T.shape
    n, k = rows // 2, m // 2
    dev = T.device
    Yt, Yb = X[:, :n], X[:, n:]
    Tt, Tb = T[:, :n], T[:, n:]
    jm = torch.zeros(m, m, dtype=torch.float64, device=dev)
    jm[:k, k:] = torch.eye(k, dtype=torch.float64, device=dev)
    jm[k:, :k] = -torch.eye(k, dtype=torch.float64, device=dev)

    # feasibility: X^T J X = Yt^T Yb - Yb^T Yt is the Ci of X
    CrY, CiY = gram(Yt, Yb)
    feas = torch.linalg.vector_norm(CiY - jm, dim=(-2, -1)) / math.sqrt(m)

    # stationarity: multiplier of the tangent projection of 2(X - T)
    E = 2 * (X - T)
    Et, Eb = E[:, :n], E[:, n:]
    values, vectors, scale, _ = eigh_scaled(CrY)
    lam = values * scale[:, None]
    den = lam[:, :, None] + lam[:, None, :]
    # (J X)^T E = Yb^T Et - Yt^T Eb = -Mi of the cross Gram of (X, E)
    _, Mi = cross_gram(Yt, Yb, Et, Eb)
    rhs = Mi.mT - Mi
    rotated = vectors.mT @ rhs @ vectors
    mult = vectors @ (rotated / den) @ vectors.mT
    mult = (mult - mult.mT) / 2
    # [Et - Yb mult; Eb + Yt mult] = E + recovery of (Yt, Yb) with P = 0, Q = mult (skew)
    Ut, Ub = recover_block(Yt, Yb, torch.zeros_like(mult), mult)
    grad = torch.cat((Et + Ut, Eb + Ub), dim=1)
    gnorm = torch.linalg.vector_norm(grad, dim=(-2, -1))
    tnorm = torch.linalg.vector_norm(T, dim=(-2, -1))
    stat = gnorm / (2 * tnorm.clamp_min(1.0))

    # duality gap
    w = mult / 2
    objective = torch.linalg.vector_norm(X - T, dim=(-2, -1)) ** 2
    CrT, CiT = gram(Tt, Tb)
    eye = torch.eye(m, dtype=torch.float64, device=dev)
    P, info = spd_inverse(eye + w @ w)
    Q = -w @ P
    tr = (P * CrT.mT).sum((-2, -1)) - (Q * CiT.mT).sum((-2, -1))
    dual = tnorm ** 2 - tr - (w * jm).sum((-2, -1))
    delta = (objective - dual).abs() / objective.abs().clamp_min(1.0)
    delta = torch.where(info == 0, delta, torch.full_like(delta, float("inf")))

    finite = torch.isfinite(X).flatten(1).all(1)
    passed = finite & (feas <= THRESHOLDS["feasibility"]) & (stat <= THRESHOLDS["stationarity"]) \
        & (delta <= THRESHOLDS["delta"])
    return {"feasibility": feas, "stationarity": stat, "delta": delta, "passed": passed}


@torch.no_grad()
def solve_certified(T: torch.Tensor, precision: str = "split", fallback: str | None = "fp64", **options):
    """Solve, certify every instance on the device, and rerun the ones that fail.

    T is a CUDA float64 [batch, 2n, 2k].  The batch is solved in ``precision``
    (options as for ``solve_ex``) and certified with the reference's acceptance
    test.  Instances that did not converge or do not pass are solved again, alone
    as one smaller batch, in the ``fallback`` form (None: no rerun); a rerun result
    replaces the first one only where it passes.  The two forms take different
    Newton paths, so on ill-conditioned batches they tend to miss different
    instances.  Returns (X, omega, iterations, report) with report holding the
    per-instance metrics, ``passed``, and the indices that were rerun.
    """
    from .dual_recommended_hvp import solve_ex
    res = solve_ex(T, precision=precision, **options)
    X, omega, iterations = res.X, res.omega, res.iterations.clone()
    cert = certify(T, X)
    passed = cert["passed"] & (res.status == 0)
    rerun = (~passed).nonzero().flatten()
    if fallback is not None and rerun.numel() > 0:
        sub = solve_ex(T[rerun].contiguous(), precision=fallback, **options)
        sub_cert = certify(T[rerun].contiguous(), sub.X)
        ok = sub_cert["passed"] & (sub.status == 0)
        take = rerun[ok]
        if take.numel() > 0:
            X[take] = sub.X[ok]
            omega[take] = sub.omega[ok]
            iterations[take] = sub.iterations[ok]
            for key in ("feasibility", "stationarity", "delta"):
                cert[key][take] = sub_cert[key][ok]
            passed[take] = True
    report = {key: cert[key] for key in ("feasibility", "stationarity", "delta")}
    report["passed"] = passed
    report["rerun"] = rerun
    return X, omega, iterations, report
