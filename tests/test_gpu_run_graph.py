"""lulesh_run_graph: the whole run as one graph launch (WHILE conditional
node around the cycle) gives the results of the host-driven loop."""
import pytest

pytestmark = pytest.mark.gpu


def test_single_job_matches_host_loop(lulesh):
    for its in (-1, 77):
        with lulesh.LuleshSet(nx=16, its=its) as a, lulesh.LuleshSet(nx=16, its=its) as b:
            assert a.run() == b.run_graph() == lulesh.OK
            assert a.state() == b.state()
            assert (a.field("e") == b.field("e")).all()


def test_batch_in_one_launch(lulesh):
    jobs = [lulesh.JobSpec(n, r, bb, cc, its) for n, r, bb, cc, its in
            [(9, 7, 2, 2, 120), (14, 11, 1, 1, -1), (5, 20, 4, 1, 60), (20, 5, 1, 4, 200)]]
    with lulesh.LuleshSet.batch(jobs) as a, lulesh.LuleshSet.batch(jobs) as b:
        a.run()
        assert b.run_graph() == lulesh.OK
        for j in range(len(jobs)):
            assert a.state(j) == b.state(j)
            assert a.origin_energy(j) == b.origin_energy(j)


def test_subdomains_and_staged(lulesh):
    for flags in (0, lulesh.FLAG_COMM_STAGED):
        with lulesh.LuleshSet(nx=6, tp=2, its=40, flags=flags) as a, \
                lulesh.LuleshSet(nx=6, tp=2, its=40, flags=flags) as b:
            a.run()
            b.run_graph()
            assert a.origin_energy() == b.origin_energy()


def test_cycle_cap_bounds_the_loop(lulesh):
    with lulesh.LuleshSet(nx=12, its=-1) as s:
        assert s.run_graph(max_cycles=25) == lulesh.OK
        st = s.state()
        assert st["cycle"] == 25 and not st["done"]
        s.run_graph(max_cycles=10)  # continues from where it stopped
        assert s.state()["cycle"] == 35


def test_errors_end_the_loop(lulesh):
    with lulesh.LuleshSet(nx=8, its=-1) as s:
        s.step(3)
        v = s.field("v")
        v[5] = -1.0
        s.set_field("v", v)
        assert s.run_graph() == lulesh.VOLUME_ERROR
        assert s.state()["done"]
