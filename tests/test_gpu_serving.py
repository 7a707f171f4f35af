"""Continuous batching (lulesh_server_*): jobs of different sizes join and
leave the resident batch between steps; each result equals the same job run
alone through lulesh_create + lulesh_run, bit for bit."""
import time

import pytest

pytestmark = pytest.mark.gpu


def _plain(lulesh, spec):
    with lulesh.LuleshSet(nx=spec.nx, numReg=spec.numReg, balance=spec.balance, cost=spec.cost,
                          its=spec.its) as s:
        st = s.run()
        return st, s.origin_energy(), s.state()["cycle"]


def _serve(lulesh, jobs, stagger=0, **cfg):
    out = {}
    with lulesh.Server(**cfg) as srv:
        ids = {}
        pending = list(enumerate(jobs))
        deadline = time.time() + 120
        while len(out) < len(jobs):
            assert time.time() < deadline, "server did not finish"
            # submit `stagger` new jobs per step (all at once when 0)
            take = len(pending) if stagger == 0 else min(stagger, len(pending))
            for _ in range(take):
                i, spec = pending.pop(0)
                ids[srv.submit(spec)] = i
            srv.step()
            for r in srv.poll():
                out[ids[r["id"]]] = r
    return out


def test_served_jobs_match_their_plain_runs(lulesh):
    jobs = [lulesh.JobSpec(nx, nr, b, c, its) for nx, nr, b, c, its in [
        (8, 11, 1, 1, 40), (14, 5, 2, 1, 25), (6, 20, 4, 4, 60), (11, 11, 1, 2, 33),
        (17, 9, 1, 1, 18), (9, 13, 2, 4, 47), (12, 7, 4, 1, 29)]]
    got = _serve(lulesh, jobs, stagger=2, hbm_cap_bytes=10**9, max_jobs=3, cycles_per_step=4,
                 prepare_threads=2)
    for i, spec in enumerate(jobs):
        st, e, cyc = _plain(lulesh, spec)
        r = got[i]
        assert r["status"] == st == lulesh.OK
        assert r["cycle"] == cyc == spec.its
        assert r["origin_energy"] == e, (i, r["origin_energy"], e)
        assert r["t_submit"] <= r["t_admit"] <= r["t_done"]


def test_memory_cap_admits_one_at_a_time(lulesh):
    """A cap that holds one job's footprint serialises admission, and every
    job still completes with its own answer."""
    jobs = [lulesh.JobSpec(10, its=12), lulesh.JobSpec(12, its=9), lulesh.JobSpec(10, its=15)]
    cap = max(lulesh.footprint_bytes([j]) for j in jobs) + 1024
    got = _serve(lulesh, jobs, hbm_cap_bytes=cap, max_jobs=8, cycles_per_step=3)
    for i, spec in enumerate(jobs):
        st, e, cyc = _plain(lulesh, spec)
        assert got[i]["origin_energy"] == e and got[i]["cycle"] == spec.its
    admits = sorted((got[i]["t_admit"], got[i]["t_done"]) for i in range(3))
    # with room for one job, each admission follows the previous retirement
    for (a0, d0), (a1, d1) in zip(admits, admits[1:]):
        assert a1 >= d0


def test_job_larger_than_cap_is_rejected(lulesh):
    with lulesh.Server(hbm_cap_bytes=10**6, max_jobs=2) as srv:
        with pytest.raises(lulesh.LuleshError) as ei:
            srv.submit(lulesh.JobSpec(40))
        assert ei.value.status == lulesh.OOM
