"""Launch shapes and the autotuner: results never depend on the shape, the
tuner leaves the set's state as it found it, and tunings are cached as JSON."""
import json

import pytest

pytestmark = pytest.mark.gpu

JOBS = [(12, 7, 2, 2, 40), (20, 11, 1, 1, 40), (9, 5, 4, 1, 40), (16, 20, 1, 4, 40)]


def _batch(lulesh):
    return lulesh.LuleshSet.batch([lulesh.JobSpec(*j) for j in JOBS])


def _energies(s, n):
    return [s.origin_energy(i) for i in range(n)]


def test_every_shape_gives_identical_results(lulesh):
    with _batch(lulesh) as s:
        s.run()
        ref = _energies(s, len(JOBS))
    for eb in (64, 128, 256):
        for nb in (128, 256, 512):
            for order in (0, 1):
                with _batch(lulesh) as s:
                    s.set_tuning(eb, nb, order, 4)
                    assert s.tuning() == {"elem_block": eb, "node_block": nb, "order": order,
                                          "graph_cycles": 4}
                    s.run()
                    assert _energies(s, len(JOBS)) == ref, (eb, nb, order)


def test_autotune_restores_state_and_applies_winner(lulesh):
    with _batch(lulesh) as a:
        a.step(7)
        a.run()
        ref = _energies(a, len(JOBS))
    with _batch(lulesh) as s:
        s.step(7)
        s.sync()
        rec = s.autotune(trial_cycles=4, rounds=1)
        assert rec["best"] == s.tuning()
        assert len(rec["trials"]) >= 18 + 1
        assert all(t["ms_per_cycle"] > 0 for t in rec["trials"])
        assert s.state(0)["cycle"] == 7
        s.run()
        assert _energies(s, len(JOBS)) == ref


def test_invalid_shapes_rejected(lulesh):
    with _batch(lulesh) as s:
        for bad in ((96, 128, 0, 1), (128, 64, 0, 1), (128, 128, 2, 1), (128, 128, 0, 0)):
            with pytest.raises(lulesh.LuleshError):
                s.set_tuning(*bad)
    with lulesh.LuleshSet(nx=6, tp=2, its=5) as s:
        with pytest.raises(lulesh.LuleshError):
            s.set_tuning(64, 128, 0, 1)
        s.set_tuning(128, 128, 1, 2)  # order and cycles per launch are free
        assert s.run() == lulesh.OK


def test_tuning_cache_round_trip(lulesh, tmp_path):
    import batching

    jobs = [lulesh.JobSpec(*j) for j in JOBS]
    path = str(tmp_path / "tuning.json")
    s, rec = batching.tuned_batch(jobs, cache=path, trial_cycles=3, rounds=1)
    s.close()
    assert not rec["cached"]
    db = json.load(open(path))
    assert batching.signature(jobs) in db
    s2, rec2 = batching.tuned_batch(jobs, cache=path)
    assert rec2["cached"] and s2.tuning() == rec["best"]
    s2.close()
