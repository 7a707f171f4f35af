"""Serving driver: a seeded Poisson stream of sedov jobs, served two ways.

served  continuous batching through lulesh_server_* (jobs admitted by HBM
        footprint, resident on the device, advanced together every step)
plain   the same stream, first come first served, one job at a time through
        the plain path (lulesh_create + lulesh_run + lulesh_destroy)

Job latency = completion time - arrival time (wall clock); throughput =
sum of the jobs' zone-cycles / (last completion - first arrival).  Both runs
check every job's Final Origin Energy against the other's.

At lambda = 50/s the served form keeps up with arrivals, so its throughput
over the makespan is bounded by the offered load.  Capacity is measured
separately: the served form replays the same jobs all queued at t = 0
(`saturated`), and the plain form's capacity is its zone-cycles over the
sum of its per-job service times (run time without queueing).
"""
from __future__ import annotations

import math
import time

import numpy as np

import lulesh_b200 as L


def make_stream(n_jobs: int = 2000, lam: float = 50.0, seed: int = 0,
                s_range=(8, 64), r_range=(5, 20), its_range=(100, 2000)) -> list[dict]:
    """numpy.random.default_rng(seed): exponential inter-arrival times of
    rate lam, edge s log-uniform in s_range, regions uniform in r_range,
    iteration budget uniform in its_range (balance 1, cost 1)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / lam, n_jobs)
    arrive = np.cumsum(gaps) - gaps[0]
    s = np.rint(np.exp(rng.uniform(math.log(s_range[0]), math.log(s_range[1]), n_jobs)))
    r = rng.integers(r_range[0], r_range[1] + 1, n_jobs)
    its = rng.integers(its_range[0], its_range[1] + 1, n_jobs)
    return [{"arrive": float(arrive[i]), "nx": int(s[i]), "numReg": int(r[i]), "balance": 1,
             "cost": 1, "its": int(its[i])} for i in range(n_jobs)]


def saturated(stream: list[dict]) -> list[dict]:
    """The same jobs, all arriving at t = 0."""
    return [dict(j, arrive=0.0) for j in stream]


def _spec(j):
    return L.JobSpec(j["nx"], j["numReg"], j["balance"], j["cost"], j["its"])


def _summary(stream, lat, done_at, cycles, t0):
    zc = sum(j["nx"] ** 3 * c for j, c in zip(stream, cycles))
    makespan = max(done_at) - t0
    lat = np.asarray(lat)
    return {"jobs": len(stream), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "makespan_s": makespan, "zone_cycles": zc, "zone_cycles_per_s": zc / makespan}


def run_served(stream, hbm_cap_bytes=150 * 10**9, max_jobs=4096, cycles_per_step=64,
               prepare_threads=8, device=0):
    """Serve `stream` through lulesh_server_*.  Admission is by device
    footprint under hbm_cap_bytes; max_jobs (slots) is set above the
    stream's size, so the footprint is what limits it."""
    srv = L.Server(hbm_cap_bytes=hbm_cap_bytes, max_jobs=max_jobs,
                   cycles_per_step=cycles_per_step, prepare_threads=prepare_threads,
                   device=device)
    n = len(stream)
    results = [None] * n
    id_of = {}
    nxt = 0
    t0 = srv.clock()
    got = 0
    while got < n:
        now = srv.clock() - t0
        while nxt < n and stream[nxt]["arrive"] <= now:
            id_of[srv.submit(_spec(stream[nxt]))] = nxt
            nxt += 1
        active, queued = srv.step()
        for r in srv.poll():
            results[id_of[r["id"]]] = r
            got += 1
        if active == 0 and queued == 0 and nxt < n:
            # idle: sleep until the next arrival
            time.sleep(max(0.0, min(0.002, stream[nxt]["arrive"] - (srv.clock() - t0))))
    srv.close()
    lat = [results[i]["t_done"] - (t0 + stream[i]["arrive"]) for i in range(n)]
    done_at = [r["t_done"] for r in results]
    out = _summary(stream, lat, done_at, [r["cycle"] for r in results], t0)
    out["status_ok"] = all(r["status"] == 0 for r in results)
    return out, [r["origin_energy"] for r in results]


def run_plain(stream, device=0):
    n = len(stream)
    t0 = time.perf_counter()
    lat, done_at, cycles, energy = [], [], [], []
    service = 0.0
    for j in stream:
        wait = j["arrive"] - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ts = time.perf_counter()
        with L.LuleshSet(nx=j["nx"], numReg=j["numReg"], balance=j["balance"], cost=j["cost"],
                         its=j["its"], device=device) as s:
            st = s.run()
            energy.append(s.origin_energy())
            cycles.append(s.state()["cycle"])
            if st != L.OK:
                raise RuntimeError(f"plain job failed with status {st}")
        t = time.perf_counter()
        service += t - ts
        done_at.append(t)
        lat.append(t - (t0 + j["arrive"]))
    out = _summary(stream, lat, done_at, cycles, t0)
    out["service_s"] = service
    out["capacity_zone_cycles_per_s"] = out["zone_cycles"] / service
    return out, energy


def capacity_repeats(stream, repeats: int = 3, every: int = 10, device: int = 0,
                     **kw) -> dict:
    """Capacity of both forms on the same jobs, repeated: every `every`-th
    job of the stream, all queued at t = 0, served `repeats` times and run
    job by job `repeats` times.  Plain capacity = zone-cycles / summed
    service time; served = zone-cycles / makespan.  The plain path's per-job
    create and destroy times vary from run to run, so the medians are the
    figures to compare."""
    sample = saturated(stream[::every])
    plain, served = [], []
    for _ in range(repeats):
        out, _ = run_plain(sample, device=device)
        plain.append(out["capacity_zone_cycles_per_s"])
        srv, _ = run_served(sample, device=device, **kw)
        served.append(srv["zone_cycles_per_s"])
    pm, sm = float(np.median(plain)), float(np.median(served))
    return {"jobs": len(sample), "every": every, "plain_repeats": plain,
            "served_repeats": served, "plain_median_zone_cycles_per_s": pm,
            "served_median_zone_cycles_per_s": sm, "capacity_ratio_median": sm / pm}


def compare(stream, plain_repeats: int = 3, capacity_every: int = 10, **kw) -> dict:
    """Served vs plain on the same stream: at the offered load (arrival
    times kept) and at capacity (served: all jobs queued at t = 0; plain:
    zone-cycles over the summed service times of its offered-load run), and
    the capacity of both forms again, `plain_repeats` times each, over a
    1-in-`capacity_every` sample (capacity_repeats)."""
    served, e_served = run_served(stream, **kw)
    sat, e_sat = run_served(saturated(stream), **kw)
    plain, e_plain = run_plain(stream, device=kw.get("device", 0))
    mism = sum(1 for a, b in zip(e_served, e_plain) if a != b)
    mism += sum(1 for a, b in zip(e_sat, e_plain) if a != b)
    out = {"served": served, "served_saturated": sat, "plain": plain,
           "throughput_ratio": served["zone_cycles_per_s"] / plain["zone_cycles_per_s"],
           "capacity_ratio_full_run": sat["zone_cycles_per_s"] /
           plain["capacity_zone_cycles_per_s"],
           "energy_mismatches": mism}
    out["capacity_ratio"] = out["capacity_ratio_full_run"]
    if plain_repeats > 0:
        out["capacity_sample"] = capacity_repeats(stream, plain_repeats, capacity_every, **kw)
    return out
