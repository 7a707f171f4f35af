"""Batched sedov jobs: many uneven meshes advanced together, one graph per
cycle (or per several cycles), with launch shapes picked by the autotuner
(lulesh_autotune) and remembered in a JSON file keyed by the batch's shape.

The job draw of the 64-job batch follows numpy.random.default_rng(seed):
edge s uniform in {10..48}, regions uniform in {5..20}, balance and cost
drawn from {1, 2, 4}, 200 iterations each.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

import lulesh_b200 as L

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_PATH = os.path.join(HERE, "tuning.json")


def config3_jobs(n: int = 64, seed: int = 0, its: int = 200) -> list:
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        s = int(rng.integers(10, 49))
        r = int(rng.integers(5, 21))
        b = int(rng.choice([1, 2, 4]))
        c = int(rng.choice([1, 2, 4]))
        jobs.append(L.JobSpec(s, r, b, c, its))
    return jobs


def signature(jobs: list, flags: int = 0) -> str:
    """Cache key: job count, total and largest element count (two significant
    digits), and the set flags.  Batches with the same key share a tuning."""
    elems = [j.nx ** 3 for j in jobs]

    def r2(v):
        return float(f"{v:.2g}")
    return f"jobs{len(jobs)}-elems{r2(sum(elems)):g}-max{r2(max(elems)):g}-flags{flags}"


def _load(path):
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tuned_batch(jobs: list, flags: int = 0, cache: str | None = TUNING_PATH,
                trial_cycles: int = 10, rounds: int = 2, device: int = -1):
    """Create the batch set and apply its tuning: from the cache when the
    batch's signature is there, else by running the autotuner (from the
    set's initial state, which it restores) and recording the result.
    Returns (set, tuning record)."""
    s = L.LuleshSet.batch(jobs, flags=flags, device=device)
    key = signature(jobs, flags)
    db = _load(cache) if cache else {}
    if key in db:
        s.set_tuning(**db[key]["best"])
        return s, dict(db[key], cached=True)
    t0 = time.perf_counter()
    rec = s.autotune(trial_cycles=trial_cycles, rounds=rounds)
    rec["tune_seconds"] = time.perf_counter() - t0
    rec["trial_cycles"] = trial_cycles
    rec["rounds"] = rounds
    if cache:
        db = _load(cache)
        db[key] = rec
        with open(cache, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
    return s, dict(rec, cached=False)


def run_batch_vs_plain(jobs: list, cache: str | None = TUNING_PATH) -> dict:
    """Config 3: the whole batch in one graph launch (lulesh_run_graph: a
    device-side loop over the tuned cycle) against each job run alone
    through the plain path; every job's Final Origin Energy must be equal
    in both."""
    import torch

    s, rec = tuned_batch(jobs, cache=cache)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    st = s.run_graph()
    e1.record(stream)
    torch.cuda.synchronize()
    batch_s = e0.elapsed_time(e1) / 1e3
    eb = [s.origin_energy(i) for i in range(len(jobs))]
    cycles = [s.state(i)["cycle"] for i in range(len(jobs))]
    s.close()
    plain_s, ep = 0.0, []
    for j in jobs:
        with L.LuleshSet(nx=j.nx, numReg=j.numReg, balance=j.balance, cost=j.cost,
                         its=j.its) as p:
            p.set_stream(stream.cuda_stream)
            torch.cuda.synchronize()
            e0.record(stream)
            p.run()
            e1.record(stream)
            torch.cuda.synchronize()
            plain_s += e0.elapsed_time(e1) / 1e3
            ep.append(p.origin_energy())
    zc = sum(j.nx ** 3 * c for j, c in zip(jobs, cycles))
    return {"jobs": len(jobs), "status": st, "zone_cycles": zc, "batch_s": batch_s,
            "plain_s": plain_s, "batch_zone_cycles_per_s": zc / batch_s,
            "plain_zone_cycles_per_s": zc / plain_s, "speedup": plain_s / batch_s,
            "energy_mismatches": sum(1 for a, b in zip(eb, ep) if a != b),
            "tuning": rec["best"], "tuning_cached": rec["cached"],
            "launches": "one graph launch for the whole batch run"}
