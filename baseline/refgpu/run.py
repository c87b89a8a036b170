"""Time the reference's own GPU solve on this GPU (baseline infrastructure only).

Runs the UNMODIFIED reference package installed under ``baseline/_ref`` through
its public API (``initialize_kernels``, ``solve``) and its own kernels
(compiled from its ``.cu`` sources by the NVRTC stand-in for CuPy in this
directory), on seeded Gaussian targets from the reference's generator rule
(src/symplectic_projection/experiment.py:43-51).  Two modes, as in the
reference protocol:

* cpu_to_cpu: ``solve(T)`` on a CPU T, returning CPU X, timed between two
  ``torch.cuda.synchronize()`` calls (experiment.py:140-161);
* device_resident: T already on the GPU as the reference's own 1024-row
  (A, D) blocks (dual_recommended_hvp.py:86-96); timed are its Gram kernels
  over the blocks, ``dual_batch`` and its recovery kernel per block, with no
  host copies.

Prints one JSON line.  Nothing in the product imports this file.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = HERE.parents[1] / "baseline" / "_ref"


def targets(n, k, count, case, base_seed=2026102100):
    import torch
    out = torch.empty(count, 2 * n, 2 * k, dtype=torch.float64)
    for j in range(count):
        gen = torch.Generator(device="cpu").manual_seed(base_seed + 1000 * case + j)
        out[j] = torch.randn(2 * n, 2 * k, dtype=torch.float64, generator=gen) / math.sqrt(2 * n)
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=4096)
    p.add_argument("--k", type=int, default=48)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--case", type=int, default=5)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=2)
    a = p.parse_args()
    if not (REF / "symplectic_projection" / "dual_recommended_hvp.py").exists():
        print(json.dumps({"unavailable": f"reference package not installed under {REF}"}))
        return 0
    sys.path.insert(0, str(HERE))           # the cupy stand-in
    sys.path.insert(0, str(REF))            # the reference package
    import torch
    torch.zeros(1, device="cuda")           # the primary context the stand-in loads into
    import symplectic_projection as ref
    if Path(ref.__file__).resolve().parent != (REF / "symplectic_projection").resolve():
        raise RuntimeError(f"imported {ref.__file__}, not the reference under {REF}")
    from symplectic_projection import dual_recommended_hvp as D
    from symplectic_projection.gram_triangle_reflect import gram_add_
    from symplectic_projection.recovery_fused import recover_block
    ref.initialize_kernels()

    n, k, B = a.n, a.k, a.batch
    m = 2 * k
    T = targets(n, k, B, a.case)
    jm = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    jm[:k, k:] = torch.eye(k, dtype=torch.float64, device="cuda")
    jm[k:, :k] = -torch.eye(k, dtype=torch.float64, device="cuda")

    def feasibility(X):
        Xd = X.cuda()
        g = Xd[:, :n].mT @ Xd[:, n:]
        return float((torch.linalg.vector_norm(g - g.mT - jm, dim=(-2, -1)) / math.sqrt(m)).max())

    # CPU -> CPU through the public solve
    for _ in range(a.warmup):
        ref.solve(T)
    times = []
    for _ in range(a.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        X, omega, it = ref.solve(T)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    cpu_ms = 1e3 * min(times)
    rf_cpu = feasibility(X)
    iters = it.tolist()

    # device resident: the reference's own blocks, Gram kernels, dual_batch and recovery kernel
    blocks = []
    for start in range(0, n, D.ROW_CHUNK):
        stop = min(start + D.ROW_CHUNK, n)
        blocks.append((T[:, start:stop].contiguous().cuda(), T[:, n + start:n + stop].contiguous().cuda()))

    def device_solve():
        Cr = torch.zeros(B, m, m, dtype=torch.float64, device="cuda")
        Ci = torch.zeros_like(Cr)
        for A_, D_ in blocks:
            gram_add_(A_, D_, Cr, Ci)
        final = []
        D.dual_batch(Cr, Ci, final)
        P, Q = final
        return [recover_block(A_, D_, P, Q) for A_, D_ in blocks]

    for _ in range(a.warmup):
        device_solve()
    dev = []
    for _ in range(a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        parts = device_solve()
        e1.record()
        torch.cuda.synchronize()
        dev.append(e0.elapsed_time(e1))
    Xd = torch.cat([torch.cat([u for u, _ in parts], 1), torch.cat([v for _, v in parts], 1)], 1)
    dev_ms = min(dev)
    print(json.dumps({
        "impl": "reference GPU path (unmodified package, its own kernels via an NVRTC stand-in for CuPy)",
        "workload": f"{B} x ({2 * n} x {m}), n={n}, k={k}",
        "cpu_to_cpu": {"value": B / (cpu_ms * 1e-3), "unit": "solves/s", "ms_per_solve_call": cpu_ms,
                       "timing": "perf_counter between torch.cuda.synchronize, best of steps"},
        "device_resident": {"value": B / (dev_ms * 1e-3), "unit": "solves/s", "ms_per_batch": dev_ms,
                            "timing": "CUDA events on the default stream, best of steps"},
        "feasibility_max": {"cpu_to_cpu": rf_cpu, "device_resident": feasibility(Xd)},
        "newton_iterations": {"max": max(iters), "mean": sum(iters) / len(iters)},
        "steps": a.steps, "warmup": a.warmup}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
