"""The reference's timing protocol, run on this package's solver.

Follows the experiment harness of the reference for the methods that go
through ``solve`` (reproduce.py:13-34 for the protocol table,
src/symplectic_projection/experiment.py:69-97 call_method, :140-161 timed_call,
:164-176 schedule, :179-211 run_case, :219-262 summarize_results):

* six cases n in {2048, 4096} x k in {16, 32, 48}, 64 seeded targets each, run in
  three rounds with the reference's case orders and per-round target shuffles;
* "single" experiment: every target alone, ``solve(t.unsqueeze(0))``, after two
  warm-up calls;
* "batch" experiment: "dual_sequential" (the 64 targets as 64 single-target
  calls) and "dual" (one batched call), each after one warm-up, in the
  reference's alternating order;
* every call is timed CPU-in/CPU-out between device synchronisations and then
  validated: success means no exception and every instance within
  r_F <= 1e-8, r_G <= 1e-9, delta <= 1e-8.

The Gao and Jensen-Zimmermann baseline methods of the reference are not part of
this package.  Validation uses the device-side acceptance metrics of
``certify`` (the three quantities of the reference's ``inspect_output``,
experiment.py:105-137) instead of a CPU pass.
"""
from __future__ import annotations

import argparse
import json
import math
import random
import time
from pathlib import Path
from statistics import fmean

import torch

from .certify import THRESHOLDS, certify
from .dual_recommended_hvp import solve
from .inputs import gaussian_targets

# reproduce.py:13-34, restricted to this package's methods
PROTOCOL = {
    "cases": [dict(name=f"n{n}_k{k}", n=n, k=k) for n in (2048, 4096) for k in (16, 32, 48)],
    "round_orders": [
        ["n2048_k16", "n4096_k16", "n2048_k32", "n4096_k32", "n2048_k48", "n4096_k48"],
        ["n4096_k32", "n2048_k32", "n4096_k48", "n2048_k48", "n4096_k16", "n2048_k16"],
        ["n2048_k48", "n4096_k48", "n2048_k16", "n4096_k16", "n2048_k32", "n4096_k32"],
    ],
    "base_seed": 2026102100,
    "shuffle_seed_base": 202610210000,
    "targets_per_case": 64,
    "rounds": 3,
    "single_warmups": 2,
    "single_methods": ["dual"],
    "batch_methods": ["dual_sequential", "dual"],
    "thresholds": dict(THRESHOLDS),
}


def case_inputs(case, case_index, protocol):
    """Targets and seeds of a case (experiment.py:43-51: seed = base + 1000 case_index + j)."""
    count = protocol["targets_per_case"]
    seeds = [protocol["base_seed"] + 1000 * case_index + j for j in range(count)]
    return gaussian_targets(case["n"], case["k"], count, case_index, protocol["base_seed"]), seeds


def call_method(method, target, precision="fp64"):
    """(X, omega, iterations) on the host for one method (experiment.py:69-97)."""
    if method == "dual":
        x, omega, iterations = solve(target, precision=precision)
        return x, omega, iterations.tolist()
    if method == "dual_sequential":
        xs, omegas, its = [], [], []
        for t in target:
            x, omega, iteration = solve(t.unsqueeze(0), precision=precision)
            xs.append(x[0])
            omegas.append(omega[0])
            its.append(int(iteration[0]))
        return torch.stack(xs), torch.stack(omegas), its
    raise ValueError(f"unknown method {method!r}")


def numeric_pass(record, thresholds):
    """Every metric present, finite and within its threshold (experiment.py:100-102)."""
    return all(record.get(key) is not None and math.isfinite(record[key]) and abs(record[key]) <= bound
               for key, bound in thresholds.items())


def validate(target, x):
    """Per-instance acceptance records for a host batch, computed on the device."""
    cert = certify(target.to("cuda"), x.to("cuda"))
    records = []
    for index in range(len(target)):
        records.append(dict(index=index, **{key: float(cert[key][index]) for key in THRESHOLDS}))
    return records


def timed_call(method, target, protocol, precision="fp64"):
    """Time one call CPU-in/CPU-out between synchronisations, then validate (experiment.py:140-161)."""
    result = dict(milliseconds=None, exception=None, validation=[], iterations=[])
    output = None
    torch.cuda.synchronize()
    started = time.perf_counter_ns()
    try:
        output = call_method(method, target, precision)
    except Exception as exc:          # a cap or a bad input: recorded as a failed call, as the reference does
        result["exception"] = f"{type(exc).__name__}: {exc}"
    torch.cuda.synchronize()
    result["milliseconds"] = (time.perf_counter_ns() - started) / 1e6
    if output is not None:
        x, _, iterations = output
        result["iterations"] = iterations
        result["validation"] = validate(target, x)
    result["success"] = (result["exception"] is None and len(result["validation"]) == len(target)
                         and all(numeric_pass(r, protocol["thresholds"]) for r in result["validation"]))
    return result


def schedule(protocol, case_index, round_number):
    """(phase, experiment, method, position, warmup_index) in the reference's order (experiment.py:164-176)."""
    single, batch = protocol["single_methods"], protocol["batch_methods"]
    for repeat in range(protocol["single_warmups"]):
        for method in single:
            yield "warmup", "single", method, 0, repeat
    for position in range(protocol["targets_per_case"]):
        shift = (position + round_number - 1 + case_index) % len(single)
        for method in single[shift:] + single[:shift]:
            yield "measured", "single", method, position, None
    for method in batch:
        yield "warmup", "batch", method, None, 0
    for method in (batch[::-1] if (round_number - 1 + case_index) % 2 else batch):
        yield "measured", "batch", method, None, None


def run_case(protocol, name, round_number, precision="fp64", log=None):
    """All calls of one case in one round; returns the rows (experiment.py:179-211)."""
    case_index = next(i for i, case in enumerate(protocol["cases"]) if case["name"] == name)
    case = protocol["cases"][case_index]
    targets, _ = case_inputs(case, case_index, protocol)
    shuffle_seed = protocol["shuffle_seed_base"] + 100 * round_number + case_index
    item_order = list(range(protocol["targets_per_case"]))
    random.Random(shuffle_seed).shuffle(item_order)
    ordered = targets[item_order].contiguous()
    rows = []
    for phase, experiment, method, position, warmup_index in schedule(protocol, case_index, round_number):
        item = None if position is None else item_order[position]
        target = ordered if position is None else ordered[position:position + 1]
        result = timed_call(method, target, protocol, precision)
        row = dict(case=name, round=round_number, phase=phase, experiment=experiment, method=method,
                   item=item, warmup_index=warmup_index, **result)
        rows.append(row)
        if log is not None:
            log.write(json.dumps(row) + "\n")
    return rows


def summarize(rows, protocol):
    """Per case: mean and per-round mean milliseconds of every measured method, the
    sequential / batched speed-up and success counts (experiment.py:219-262)."""
    cases = []
    measured = [row for row in rows if row["phase"] == "measured"]
    for case in protocol["cases"]:
        mine = [row for row in measured if row["case"] == case["name"]]
        if not mine:
            continue
        rounds = sorted({row["round"] for row in mine})
        item = dict(case=case)
        for group, methods in (("single", protocol["single_methods"]), ("batch", protocol["batch_methods"])):
            item[group] = {}
            for method in methods:
                sel = [row for row in mine if row["experiment"] == group and row["method"] == method]
                item[group][method] = dict(
                    calls=len(sel), successful_calls=sum(row["success"] for row in sel),
                    all_calls_successful=all(row["success"] for row in sel),
                    milliseconds=dict(mean=fmean(row["milliseconds"] for row in sel)),
                    round_mean_ms=[fmean(row["milliseconds"] for row in sel if row["round"] == r) for r in rounds])
        seq, bat = item["batch"]["dual_sequential"], item["batch"]["dual"]
        item["batch"]["speedups"] = {"dual_sequential": (
            seq["milliseconds"]["mean"] / bat["milliseconds"]["mean"]
            if seq["all_calls_successful"] and bat["all_calls_successful"] else None)}
        item["batch"]["solves_per_s"] = protocol["targets_per_case"] / (bat["milliseconds"]["mean"] * 1e-3)
        cases.append(item)
    validations = [v for row in measured for v in row["validation"]]
    accuracy = dict(outputs=len(validations))
    for key in protocol["thresholds"]:
        vals = [v[key] for v in validations if v.get(key) is not None and math.isfinite(v[key])]
        accuracy["max_" + key] = max(vals, default=None)
    return dict(cases=cases, accuracy=accuracy,
                counts=dict(formal_calls=len(measured), formal_successes=sum(r["success"] for r in measured)),
                all_calls_successful=all(row["success"] for row in rows),
                failure_records=[dict(case=r["case"], round=r["round"], method=r["method"], item=r["item"],
                                      exception=r["exception"]) for r in rows if not r["success"]])


def run_protocol(protocol=PROTOCOL, rounds=None, cases=None, precision="fp64", output=None):
    """Every (round, case) task in the reference's order; returns the summary.  With
    ``output`` the raw rows go to output/raw.jsonl and the summary to output/summary.json."""
    rounds = rounds or protocol["rounds"]
    wanted = set(cases) if cases else None
    log = None
    if output is not None:
        output = Path(output)
        output.mkdir(parents=True, exist_ok=False)
        (output / "protocol.json").write_text(json.dumps(dict(protocol, precision=precision), indent=2) + "\n")
        log = (output / "raw.jsonl").open("w")
    rows = []
    try:
        for r, names in enumerate(protocol["round_orders"][:rounds], 1):
            for name in names:
                if wanted is None or name in wanted:
                    rows.extend(run_case(protocol, name, r, precision, log))
    finally:
        if log is not None:
            log.close()
    summary = summarize(rows, protocol)
    summary["precision"] = precision
    if output is not None:
        (output / "summary.json").write_text(json.dumps(summary, indent=2) + "\n")
    return summary


def main(argv=None):
    p = argparse.ArgumentParser(description="The reference's timing protocol on this package's solver.")
    p.add_argument("--output", type=Path, default=None, help="new directory for raw.jsonl and summary.json")
    p.add_argument("--rounds", type=int, default=PROTOCOL["rounds"])
    p.add_argument("--cases", nargs="*", default=None, help="case names, e.g. n4096_k48 (default: all six)")
    p.add_argument("--targets", type=int, default=PROTOCOL["targets_per_case"])
    p.add_argument("--precision", choices=["fp64", "split"], default="fp64")
    args = p.parse_args(argv)
    protocol = dict(PROTOCOL, targets_per_case=args.targets)
    summary = run_protocol(protocol, args.rounds, args.cases, args.precision, args.output)
    for item in summary["cases"]:
        b = item["batch"]
        print(json.dumps(dict(case=item["case"]["name"], single_ms=item["single"]["dual"]["milliseconds"]["mean"],
                              sequential_ms=b["dual_sequential"]["milliseconds"]["mean"],
                              batched_ms=b["dual"]["milliseconds"]["mean"], speedup=b["speedups"]["dual_sequential"],
                              batched_solves_per_s=b["solves_per_s"])))
    print(json.dumps(dict(all_calls_successful=summary["all_calls_successful"], accuracy=summary["accuracy"])))
    return 0 if summary["all_calls_successful"] else 1


if __name__ == "__main__":
    raise SystemExit(main())
