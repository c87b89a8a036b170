"""Generate the golden fixtures in this directory from the reference itself.

Run with a checkout of the reference project (read-only) available:

    python tests/golden/make_golden.py [--reference PATH]

The reference root is, in order: ``--reference PATH``, the environment
variable SSN_REFERENCE_ROOT, or ``reference`` beside this repository's root
directory (``<repo>/../reference``).  It must contain ``src/symplectic_projection``.

What it does:
  * installs a stub ``cupy`` module (the reference imports CuPy at module
    import time but only uses it to compile/launch its GPU kernels);
  * imports the reference's ``dual_recommended_hvp`` and ``experiment``;
  * replaces the nine CuPy kernel wrappers that ``dual_batch`` calls with
    torch CPU FP64 operations that follow each wrapper's documented contract
    (the reference's own Python driver logic -- scaling, eigenbasis, Newton,
    PCG, Armijo line search, exits -- runs unmodified);
  * records per-case T, X, omega, iterations, the final (P, Q), the call
    counts of the HVP / line-change wrappers, and the reference's own
    ``inspect_output`` metrics.

The fixtures are small (a few hundred KB in total) so they travel with the
repository; nothing at test time reads the reference.
"""
from __future__ import annotations

import json
import math
import os
import sys
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def reference_root(argv=None) -> Path:
    """--reference PATH, else $SSN_REFERENCE_ROOT, else <repo>/../reference."""
    import argparse
    p = argparse.ArgumentParser(description="generate the golden fixtures from the reference")
    p.add_argument("--reference", default=None, help="root of the reference project checkout")
    args, _ = p.parse_known_args(argv)
    root = args.reference or os.environ.get("SSN_REFERENCE_ROOT") or str(REPO.parent / "reference")
    return Path(root).resolve()


REF = reference_root([] if __name__ != "__main__" else None)

# (name, n, k, batch, case_index, target transform)
CASES = [
    ("n64_k8_b4", 64, 8, 4, 0, None),
    ("n48_k12_b3", 48, 12, 3, 1, None),
    ("n5_k1_b3", 5, 1, 3, 2, None),
    ("n6_k6_b2", 6, 6, 2, 3, None),          # square T (n == k)
    ("n100_k20_b2", 100, 20, 2, 4, None),
    ("n64_k48_b1", 64, 48, 1, 5, None),       # m = 96, near-square: the reference fails
    ("n192_k48_b2", 192, 48, 2, 9, None),     # m = 96, the headline width
    ("n96_k64_b1", 96, 64, 1, 6, None),       # m = 128, widest supported
    ("n40_k8_b3_scaled3", 40, 8, 3, 7, ("scale", 3.0)),   # larger ||T||: backtracking
    ("n64_k4_b2_illcond", 64, 4, 2, 8, ("illcond", 1e-2)),  # graded singular values
]


def _install_cupy_stub():
    stub = types.ModuleType("cupy")
    stub.__version__ = "stub"

    class RawModule:  # never called on the CPU path
        def __init__(self, *a, **k):
            raise RuntimeError("cupy stub: GPU kernels are not available")

    stub.RawModule = RawModule
    sys.modules["cupy"] = stub


def _load_reference():
    _install_cupy_stub()
    sys.path.insert(0, str(REF / "src"))
    import symplectic_projection.dual_recommended_hvp as dual
    import symplectic_projection.experiment as experiment
    return dual, experiment


COUNTS = {"hvp_outer": 0, "line_change": 0, "sandwich": 0}


def _patch(dual):
    """CPU FP64 stand-ins for the CuPy wrappers, per their docstrings."""
    def inner_products(E, Sr, Si):            # hvp_fused.py:22-23
        return E @ Sr, E @ Si

    def outer_skew(P, Q, U, V):               # hvp_fused.py:37-38
        COUNTS["hvp_outer"] += 1
        Z = P @ U - Q @ V
        return Z - Z.mT

    def sandwich_front(values, Ci, P, Q):     # hvp_fused.py:56-57
        COUNTS["sandwich"] += 1
        return P * values[:, None, :] - Q @ Ci, P @ Ci + Q * values[:, None, :]

    def line_change(gradient, delta, V, delta_Sr, trial, delta_Si):  # hvp_fused.py:72-73
        COUNTS["line_change"] += 1
        first = (gradient * delta).sum(dim=(-2, -1))
        tail = (V * (delta_Sr + trial @ delta_Si)).sum(dim=(-2, -1))
        return first + tail

    def fused_precondition(R, denominator):   # hvp_fused.py:110-111
        a = R / denominator
        return (a - a.mT) * 0.5

    def cg_update(direction, r, p, Hp, alpha):  # hvp_fused.py:120-121
        return direction + alpha[:, None, None] * p, r - alpha[:, None, None] * Hp

    def cg_next(z, p, beta, cg_active):       # hvp_fused.py:133-134
        nxt = z + beta[:, None, None] * p
        return torch.where(cg_active[:, None, None], nxt, torch.zeros_like(nxt))

    def recover_block(A, D, P, Q):            # recovery_fused.py:159-160
        return A @ P.mT + D @ Q.mT, D @ P.mT - A @ Q.mT

    dual.inner_products = inner_products
    dual.outer_skew = outer_skew
    dual.sandwich_front = sandwich_front
    dual.line_change = line_change
    dual.fused_precondition = fused_precondition
    dual.cg_update = cg_update
    dual.cg_next = cg_next
    dual.recover_block = recover_block
    dual.DEVICE = "cpu"


def _targets(experiment, n, k, batch, case_index, transform):
    proto = dict(base_seed=2026102100, targets_per_case=batch)
    T, seeds = experiment.make_inputs(dict(n=n, k=k), case_index, proto)
    if transform is not None and transform[0] == "scale":
        T = T * transform[1]
    elif transform is not None and transform[0] == "illcond":
        # T = U diag(s) V^T with s log-spaced in [smin, 1/smin], ||T||_F^2 = 2k
        smin = transform[1]
        out = torch.empty_like(T)
        for j in range(batch):
            g = torch.Generator().manual_seed(2026102500 + j)
            U, _ = torch.linalg.qr(torch.randn(2 * n, 2 * k, dtype=torch.float64, generator=g))
            V, _ = torch.linalg.qr(torch.randn(2 * k, 2 * k, dtype=torch.float64, generator=g))
            s = torch.exp(torch.linspace(math.log(smin), -math.log(smin), 2 * k, dtype=torch.float64))
            t = U @ torch.diag(s) @ V.mT
            out[j] = t * math.sqrt(2 * k) / torch.linalg.vector_norm(t)
        T = out
    return T.contiguous(), seeds


def main():
    dual, experiment = _load_reference()
    _patch(dual)
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    manifest = {}
    for name, n, k, batch, case_index, transform in CASES:
        for key in COUNTS:
            COUNTS[key] = 0
        T, seeds = _targets(experiment, n, k, batch, case_index, transform)
        A, D = T[:, :n], T[:, n:]
        Cr = A.mT @ A + D.mT @ D
        Ci = A.mT @ D - D.mT @ A
        final = []
        try:
            omega, L, iterations = dual.dual_batch(Cr, Ci, final)
        except RuntimeError as exc:
            # the reference's own failure (e.g. its line-search cap); keep the input
            np.savez_compressed(HERE / f"{name}.npz", T=T.numpy())
            manifest[name] = dict(n=n, k=k, batch=batch, case_index=case_index, seeds=seeds,
                                  transform=transform, counts=dict(COUNTS),
                                  error=f"{type(exc).__name__}")
            print(name, "reference raised", type(exc).__name__, dict(COUNTS))
            continue
        P, Q = final
        Ur, Ui = A @ P.mT + D @ Q.mT, D @ P.mT - A @ Q.mT
        X = torch.cat((Ur, Ui), dim=1)
        records = experiment.inspect_output(T, X)
        metrics = np.array([[r["feasibility"], r["stationarity"], r["delta"]] for r in records],
                           dtype=np.float64)
        np.savez_compressed(
            HERE / f"{name}.npz", T=T.numpy(), X=X.numpy(), omega=omega.numpy(),
            P=P.numpy(), Q=Q.numpy(), iterations=iterations.numpy(), Cr=Cr.numpy(), Ci=Ci.numpy(),
            metrics=metrics)
        manifest[name] = dict(n=n, k=k, batch=batch, case_index=case_index, seeds=seeds,
                              transform=transform, counts=dict(COUNTS),
                              iterations=iterations.tolist(),
                              worst=dict(zip(("feasibility", "stationarity", "delta"),
                                             metrics.max(axis=0).tolist())))
        print(name, manifest[name]["iterations"], manifest[name]["counts"], manifest[name]["worst"])
    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=1) + "\n")


if __name__ == "__main__":
    main()
