"""The seeded synthetic workloads the bench and the batch/serving modes run:
the 64-job batch (numpy default_rng(0): s ~ U{10..48}, r ~ U{5..20},
b, c in {1, 2, 4}, 200 cycles) and the 2,000-job stream (Poisson arrivals
at 50/s, s log-uniform in [8, 64], r ~ U[5, 20], its ~ U[100, 2000])."""
import math

import numpy as np

import batching
import serving


def test_batch_jobs_follow_their_spec():
    jobs = batching.config3_jobs()
    assert len(jobs) == 64
    assert all(10 <= j.nx <= 48 and 5 <= j.numReg <= 20 for j in jobs)
    assert all(j.balance in (1, 2, 4) and j.cost in (1, 2, 4) and j.its == 200 for j in jobs)
    # seeded: the same list every time, and a spread of sizes and settings
    again = batching.config3_jobs()
    assert [(j.nx, j.numReg, j.balance, j.cost) for j in jobs] == \
        [(j.nx, j.numReg, j.balance, j.cost) for j in again]
    assert len({j.nx for j in jobs}) > 20
    assert {j.balance for j in jobs} == {1, 2, 4} and {j.cost for j in jobs} == {1, 2, 4}


def test_stream_follows_its_spec():
    st = serving.make_stream()
    assert len(st) == 2000 and st == serving.make_stream()
    arrive = np.array([j["arrive"] for j in st])
    assert arrive[0] == 0.0 and np.all(np.diff(arrive) >= 0)
    # Poisson at 50/s: 1,999 gaps of mean 0.02 s (4 standard errors)
    gaps = np.diff(arrive)
    assert abs(gaps.mean() - 0.02) < 4 * 0.02 / math.sqrt(len(gaps))
    s = np.array([j["nx"] for j in st])
    assert s.min() >= 8 and s.max() <= 64
    # log-uniform: the median edge is near sqrt(8 * 64)
    assert abs(np.median(s) - math.sqrt(8 * 64)) < 2.5
    assert all(5 <= j["numReg"] <= 20 and 100 <= j["its"] <= 2000 for j in st)
    assert all(j["balance"] == 1 and j["cost"] == 1 for j in st)


def test_saturated_only_moves_arrivals():
    st = serving.make_stream(n_jobs=50)
    sat = serving.saturated(st)
    assert all(j["arrive"] == 0.0 for j in sat)
    assert [dict(j, arrive=0.0) for j in st] == sat
