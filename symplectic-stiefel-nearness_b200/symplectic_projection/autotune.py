"""Per-(n, k) autotuner of the solve's launch parameters (``ssn_set_tuning``).

The reference hard-codes its schedule (``ROW_CHUNK = 1024``,
src/symplectic_projection/dual_recommended_hvp.py:13; 16x16 Gram tiles,
gram_triangle_reflect.py:32-36).  Here four launch parameters of ``ssn_solve``
are searched per problem class (precision form, m = 2k, n, batch):

  gram_splits    row splits of the FP64 Gram (plain FP64 form);
  gram_chunks    row chunks of the INT8 Ozaki Gram (split form);
  recover_parts  row-tile parts of the Ozaki recovery (split form);
  cluster        CTAs per instance of the Newton kernels (1 or 2).

``tune`` times ``ssn_solve`` on seeded targets of the class for each candidate
value, one parameter at a time starting from the library's built-in rules
(coordinate descent, best of ``reps`` CUDA-event timings), and keeps a value
only when it beats the incumbent by more than ``min_gain``.  The winners go to
a JSON table (``tuning_b200.json`` beside this file) that the package installs
when it loads the native library.  A parameter only changes the schedule: the
tuned and built-in solves agree to the products' rounding.
"""
from __future__ import annotations

import json
from pathlib import Path

import torch

from . import _native as N

TABLE_PATH = Path(__file__).with_name("tuning_b200.json")
FIELDS = ("gram_splits", "gram_chunks", "recover_parts", "cluster")
PRECISION_CODES = {"fp64": 0, "split": 1}
BATCH_ANY = (1, 1 << 30)


def _entry_struct(e: dict) -> N.Tuning:
    t = N.Tuning()
    t.precision = PRECISION_CODES[e["precision"]]
    t.m = int(e["m"])
    t.n_min, t.n_max = int(e["n_min"]), int(e["n_max"])
    t.batch_min, t.batch_max = int(e["batch_min"]), int(e["batch_max"])
    for f in FIELDS:
        setattr(t, f, int(e.get(f, 0)))
    return t


def install(entries: list[dict]) -> None:
    """Replace the library's table with ``entries`` (dicts with the ssn_tuning fields)."""
    arr = (N.Tuning * max(1, len(entries)))(*[_entry_struct(e) for e in entries])
    N.check(N.load().ssn_set_tuning(arr, len(entries)), "ssn_set_tuning")


def installed() -> list[dict]:
    """The table the library holds now."""
    lib = N.load()
    count = lib.ssn_get_tuning(None, 0)
    arr = (N.Tuning * max(1, count))()
    lib.ssn_get_tuning(arr, count)
    names = {v: k for k, v in PRECISION_CODES.items()}
    out = []
    for t in arr[:count]:
        e = {"precision": names[t.precision], "m": t.m, "n_min": t.n_min, "n_max": t.n_max,
             "batch_min": t.batch_min, "batch_max": t.batch_max}
        e.update({f: getattr(t, f) for f in FIELDS})
        out.append(e)
    return out


def load(path: Path | str = TABLE_PATH) -> int:
    """Install the table stored at ``path`` (if it exists); returns the entry count."""
    path = Path(path)
    if not path.exists():
        return 0
    entries = json.loads(path.read_text())["entries"]
    install(entries)
    return len(entries)


def save(entries: list[dict], path: Path | str = TABLE_PATH, note: str = "") -> None:
    Path(path).write_text(json.dumps({"note": note, "entries": entries}, indent=1) + "\n")


def candidates(precision: str, n: int, m: int, batch: int) -> dict:
    """Values tried for each parameter (0 = the built-in rule)."""
    c = {"cluster": [0, 1] + ([2] if m > 32 else [])}
    if precision == "fp64":
        c["gram_splits"] = [0, 1, 2, 3, 4, 6, 8, 12, 16]
    else:
        c["gram_chunks"] = [0, 1, 2, 3, 4, 6, 8]
        c["recover_parts"] = [0, 1, 2, 4, 8, 16, 32]
    return c


def _time_solve(T: torch.Tensor, precision: str, entry: dict | None, reps: int) -> float:
    from .dual_recommended_hvp import solve_ex
    install([entry] if entry else [])
    solve_ex(T, precision=precision)                     # warm-up (workspace, first-touch)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        solve_ex(T, precision=precision)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune(n: int, k: int, batch: int, precision: str = "split", reps: int = 5, seed: int = 0,
         batch_range: tuple[int, int] | None = None, min_gain: float = 0.02) -> dict:
    """The best parameters for the class (precision, m = 2k, n, batch); returns its table entry.

    The entry covers exactly this n and m, and ``batch_range`` (default: exactly ``batch``).
    The table installed before the call is restored afterwards.
    """
    from .inputs import gaussian_targets
    saved = installed()
    m = 2 * k
    lo, hi = batch_range or (batch, batch)
    entry = {"precision": precision, "m": m, "n_min": n, "n_max": n, "batch_min": lo, "batch_max": hi}
    entry.update({f: 0 for f in FIELDS})
    try:
        T = gaussian_targets(n, k, batch, seed).cuda()
        base = best = _time_solve(T, precision, entry, reps)
        for field, values in candidates(precision, n, m, batch).items():
            for v in values:
                if v == entry[field]:
                    continue
                trial = dict(entry, **{field: v})
                t = _time_solve(T, precision, trial, reps)
                if t < best * (1.0 - min_gain):
                    best, entry = t, trial
        entry["tuned_ms"] = round(best, 4)
        entry["builtin_ms"] = round(base, 4)
    finally:
        install(saved)
    return entry


def ragged_classes(count: int = 384) -> list[tuple[int, int, int]]:
    """(n, k, group size) of every shape group of the ragged workload."""
    from collections import Counter
    from .inputs import ragged_shapes
    return sorted((n, k, c) for (n, k), c in Counter(ragged_shapes(count)).items())


def main(argv=None) -> None:
    """Tune the benchmark classes and write the table:

        python -m symplectic_projection.autotune [--out PATH] [--reps R]

    Classes: 64 targets at (n, k) = (2048, 16) and (4096, 48) in both precision
    forms (exact batch), and every (n, k) group of the 384-target ragged workload in
    both forms (any batch size).
    """
    import argparse
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(TABLE_PATH))
    p.add_argument("--reps", type=int, default=5)
    p.add_argument("--forms", default="split,fp64")
    args = p.parse_args(argv)
    forms = args.forms.split(",")
    entries = []
    for precision in forms:
        for n, k in ((2048, 16), (4096, 48)):
            e = tune(n, k, 64, precision, reps=args.reps)
            print(json.dumps(e), flush=True)
            entries.append(e)
    for precision in forms:
        for n, k, c in ragged_classes():
            e = tune(n, k, c, precision, reps=args.reps, batch_range=BATCH_ANY)
            print(json.dumps(e), flush=True)
            entries.append(e)
    # an entry that keeps every built-in rule changes nothing: leave it out
    kept = [e for e in entries if any(e[f] for f in FIELDS)]
    save(kept, args.out, note="ssn_solve launch parameters tuned on one B200 by "
                              "python -m symplectic_projection.autotune (tuned_ms / builtin_ms: best of "
                              f"{args.reps} timings of the class's solve)")
    print(f"{len(kept)} of {len(entries)} classes keep a tuned parameter -> {args.out}")


if __name__ == "__main__":
    main()
