"""One problem over several parts (the multi-GPU path) on the CPU.

The parts here are oracle parts (tests/oracle_parts.py): the CPU oracle's
subdomains in place of the GPU kernels.  What runs is the product's
exchange layer -- the message plan (lulesh_halo_plan, host code shared with
the GPU build's pack/unpack tables), the cycle order of distributed.Engine,
and its transports: LocalTransport (all parts in one process) and
HostTransport over torch.distributed gloo ranks (2 and 8 processes).  The
decomposed run must give the single-domain values bit for bit: the same
check the GPU tests make on one device.  Failure detection is made on the
host: a rank that leaves before an exchange ends the others' exchange with
an error instead of a hang.
"""
import os
import sys
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import REPO

import distributed as D
import oracle
from oracle_parts import OraclePart, compare_with_single

TESTS = os.path.dirname(os.path.abspath(__file__))


def _single(nx_global, cycles):
    o = oracle.Oracle(nx_global)
    for _ in range(cycles):
        assert o.step() == 0
    return o


def test_plan_pairs_are_symmetric_in_size():
    """Every message has the same plan on both sides (one function), and the
    per-kind sizes match the layer geometry: a face of nx^2 elements x 4
    corners x 3 components, an edge nx x 2 x 3, a corner 3."""
    nx = 5
    E = nx ** 3
    Ep = (E + 31) // 32 * 32
    for nparts in (2, 4, 8):
        for a in range(nparts):
            for b in D.peers(2, nparts, a):
                r1, f1, i1 = D.plan(nx, 2, nparts, a, b, D.L.HALO_CORNERS)
                assert len(r1) > 0
                assert set(np.unique(f1)) == {13, 14, 15}
                assert np.all((i1 >= 0) & (i1 < 8 * Ep))
    # 8 parts: one subdomain each; rank 0 -> rank 1 (face), 3 (edge), 7 (corner)
    assert len(D.plan(nx, 2, 8, 0, 1, D.L.HALO_CORNERS)[0]) == nx * nx * 4 * 3
    assert len(D.plan(nx, 2, 8, 0, 3, D.L.HALO_CORNERS)[0]) == nx * 2 * 3
    assert len(D.plan(nx, 2, 8, 0, 7, D.L.HALO_CORNERS)[0]) == 3
    # positions/velocities travel only toward the minus side
    assert len(D.plan(nx, 2, 8, 0, 1, D.L.HALO_POSVEL)[0]) == 0
    assert len(D.plan(nx, 2, 8, 1, 0, D.L.HALO_POSVEL)[0]) == (nx + 1) ** 2 * 6
    # monotonic-Q ghosts: faces only
    assert len(D.plan(nx, 2, 8, 0, 3, D.L.HALO_MONOQ)[0]) == 0
    assert len(D.plan(nx, 2, 8, 0, 1, D.L.HALO_MONOQ)[0]) == nx * nx * 3


@pytest.mark.parametrize("sync_posvel", [False, True])
@pytest.mark.parametrize("nparts", [1, 2, 4, 8])
def test_local_parts_match_single_domain(nparts, sync_posvel):
    """With or without the POSVEL exchange (the engine leaves it out by
    default: each part computes its shared nodes as their owner does)."""
    nx, cycles = 4, 25
    parts = [OraclePart(nx, 2, nparts, p) for p in range(nparts)]
    eng = D.Engine(parts, D.LocalTransport(), sync_posvel=sync_posvel)
    eng.setup()
    eng.run(cycles)
    single = _single(2 * nx, cycles)
    for p in parts:
        assert compare_with_single(p, single) == []
    origin = parts[0].doms[0]
    assert origin.origin_energy() == single.origin_energy()
    assert origin.scalar("cycle") == cycles
    assert origin.scalar("time") == single.scalar("time")


def test_nodal_mass_exchange_matches_single_domain():
    nx = 5
    parts = [OraclePart(nx, 2, 4, p) for p in range(4)]
    D.Engine(parts, D.LocalTransport()).setup()
    single = oracle.Oracle(2 * nx)
    assert all(compare_with_single(p, single) == [] for p in parts)


def _gloo_worker(rank, world, port, nx, cycles, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (TESTS, os.path.join(REPO, "cuda-ipc-benchmarks_b200"), os.path.join(REPO, "oracle")):
        sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    import distributed as Dm
    from oracle_parts import OraclePart as OP, compare_with_single as cmp

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        part = OP(nx, 2, world, rank)
        eng = Dm.Engine([part], Dm.HostTransport(dist, timeout_s=10.0))
        eng.setup()
        if mode == "leave" and rank == world - 1:
            os._exit(3)  # this rank never takes part in the cycle's exchanges
        t0 = time.time()
        try:
            eng.run(cycles)
        except Exception as e:  # noqa: BLE001
            q.put((rank, "error", f"{type(e).__name__}: {e}"[:200], time.time() - t0))
            q.close()
            q.join_thread()  # the result must leave before the process does
            os._exit(0)
        import oracle as om

        single = om.Oracle(2 * nx)
        for _ in range(cycles):
            single.step()
        bad = cmp(part, single)
        e0 = part.doms[0].origin_energy() if 0 in part.doms else None
        q.put((rank, "ok", bad, e0 == single.origin_energy() if e0 is not None else None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # noqa: BLE001
        q.put((rank, "error", f"{type(e).__name__}: {e}"[:200], 0.0))


def _run_gloo(world, nx, cycles, mode="run", timeout=240):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() * 7 + world * 13 + nx) % 3000
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, nx, cycles, mode, q))
             for r in range(world)]
    for p in procs:
        p.start()
    n_expected = world - 1 if mode == "leave" else world
    out = [q.get(timeout=timeout) for _ in range(n_expected)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda t: t[0])


@pytest.mark.parametrize("world,nx", [(2, 4), (8, 6)])
def test_gloo_ranks_match_single_domain(world, nx):
    """2 ranks at -s 8 and 8 ranks at -s 12 (2x2x2 subdomains of -s 4 / 6),
    halos through the host transport over gloo."""
    res = _run_gloo(world, nx, cycles=20)
    assert [r[1] for r in res] == ["ok"] * world, res
    assert all(r[2] == [] for r in res), res
    assert res[0][3] is True  # rank 0 holds the origin: energy bit for bit


def test_rank_that_leaves_ends_the_exchange_with_an_error():
    """The last rank exits after set-up without taking part in the first
    cycle's exchange: the other rank's bounded wait (10 s) raises instead of
    hanging."""
    res = _run_gloo(2, 4, cycles=5, mode="leave")
    assert len(res) == 1
    rank, kind, msg, waited = res[0]
    assert rank == 0 and kind == "error", res
    assert waited < 60.0
