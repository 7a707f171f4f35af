"""GPU parity: the CUDA step (through the C ABI) against the CPU oracle.

Tolerances.  The oracle evaluates the reference's expressions without FMA
contraction; the GPU build contracts multiply-adds like the reference CUDA
build does.  Fields therefore agree to rounding level after one cycle
(rtol 1e-12) and drift slowly; the parity gate is Final Origin Energy
within 1e-9 relative.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

pytestmark = pytest.mark.gpu

E_TOL = 1e-9  # Final Origin Energy, relative (the parity bound)

ELEM_FIELDS = ["e", "p", "q", "v", "ss", "delv", "vdov", "arealg", "ql", "qq", "vnew",
               "delx_xi", "delx_eta", "delx_zeta"]
NODE_FIELDS = ["x", "y", "z", "xd", "yd", "zd", "xdd", "ydd", "zdd", "fx", "fy", "fz"]


def _close(a, b, rtol):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return np.allclose(a, b, rtol=rtol, atol=rtol * scale)


def _compare_state(gs, orc, rtol, fields=ELEM_FIELDS + NODE_FIELDS):
    bad = []
    for f in fields:
        g = gs.field(f)
        o = orc.field(f)[: g.size]
        if not _close(g, o, rtol):
            d = np.max(np.abs(g - o)) / max(np.max(np.abs(o)), 1e-300)
            bad.append(f"{f}: max scaled diff {d:.3e}")
    return bad


@pytest.mark.parametrize("nx,cycles,rtol", [(4, 1, 1e-12), (8, 1, 1e-12), (8, 25, 1e-10)])
def test_fields_match_oracle(lulesh, oracle_mod, nx, cycles, rtol):
    with lulesh.LuleshSet(nx=nx, its=cycles, flags=lulesh.FLAG_MATERIALIZE) as gs:
        orc = oracle_mod.Oracle(nx)
        for _ in range(cycles):
            assert orc.step() == 0
        assert gs.run() == lulesh.OK
        st = gs.state()
        assert st["cycle"] == cycles and st["done"] == 1
        assert rel(st["time"], orc.scalar("time")) < 1e-12
        assert rel(st["deltatime"], orc.scalar("deltatime")) < 1e-12
        bad = _compare_state(gs, orc, rtol)
        assert not bad, bad
        # corner forces of the last cycle
        for f in ("fx_elem", "fy_elem", "fz_elem"):
            assert _close(gs.field(f), orc.field(f), rtol), f


@pytest.mark.parametrize("nx", [1, 2, 3, 5])
def test_small_meshes_full_run(lulesh, oracle_mod, nx):
    """Edge sizes: a single element (every face on a boundary) up to -s 5,
    run to t = 0.01; same cycle count, time and energies as the oracle."""
    with lulesh.LuleshSet(nx=nx, its=-1) as gs:
        orc = oracle_mod.Oracle(nx)
        ost, ocyc = orc.run()
        assert gs.run() == ost == lulesh.OK
        st = gs.state()
        assert st["cycle"] == ocyc and st["done"] == 1
        assert rel(st["time"], orc.scalar("time")) < 1e-12
        assert rel(gs.origin_energy(), orc.origin_energy()) < E_TOL
        bad = _compare_state(gs, orc, 1e-9, ["e", "p", "q", "v", "x", "xd"])
        assert not bad, bad


def test_setup_matches_oracle(lulesh, oracle_mod):
    """Everything NewDomain builds (lulesh.cu:750-1221) is laid out as the
    reference lays it out: bit-exact for index data and the initial state."""
    with lulesh.LuleshSet(nx=7, numReg=9, balance=2, cost=3) as gs:
        orc = oracle_mod.Oracle(7, numReg=9, balance=2, cost=3)
        for f in ["nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
                  "nodeElemCount", "nodeElemStart", "nodeElemCornerList", "symmX", "symmY",
                  "symmZ", "matElemlist", "regCSR", "regReps", "regNumList", "regElemlist",
                  "regSorted"]:
            assert np.array_equal(gs.field(f), orc.field(f)), f
        for f in ["x", "y", "z", "volo", "elemMass", "nodalMass", "e", "v"]:
            assert np.array_equal(gs.field(f), orc.field(f)), f


def test_config1_energy(lulesh, oracle_mod):
    """LULESH sedov -s 30 -i 100 -r 11 -b 1 -c 1 (the CPU/GPU parity config)."""
    with lulesh.LuleshSet(nx=30, its=100) as gs:
        assert gs.run() == lulesh.OK
        e_gpu = gs.origin_energy()
        sym_gpu = gs.symmetry()
    orc = oracle_mod.Oracle(30)
    st, n = orc.run(100)
    assert st == 0 and n == 100
    assert rel(e_gpu, orc.origin_energy()) < E_TOL
    with open(os.path.join(GOLDEN, "omp_reference.json")) as f:
        gold = json.load(f)["runs"]["-s 30 -i 100"]
    assert rel(e_gpu, gold["energy"]) < E_TOL
    # symmetry check of plane 0: same order of magnitude as the references
    assert sym_gpu[2] < 1e-10


def test_determinism(lulesh):
    """No float atomics anywhere: two runs are bit-identical."""
    outs = []
    for _ in range(2):
        with lulesh.LuleshSet(nx=12, its=40) as gs:
            assert gs.run() == lulesh.OK
            outs.append((gs.field("e"), gs.field("x"), gs.field("xd")))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_region_flags_do_not_change_results(lulesh):
    """The EOS rep loop is pure (lulesh.cu:4045-4083): -r/-b/-c change cost
    only, never the answer."""
    res = []
    for nr, b, c in [(11, 1, 1), (20, 4, 4), (1, 1, 1)]:
        with lulesh.LuleshSet(nx=10, numReg=nr, balance=b, cost=c, its=30) as gs:
            assert gs.run() == lulesh.OK
            res.append(gs.field("e"))
    assert np.array_equal(res[0], res[1]) and np.array_equal(res[0], res[2])


@pytest.mark.parametrize("tp,nx", [(2, 6), (2, 9), (3, 4), (4, 5)])
def test_subdomains_bitwise_equal_single_domain(lulesh, tp, nx):
    """tp^3 in-device subdomains of -s nx reproduce the single -s tp*nx
    domain exactly, every node and element field of every subdomain:
    corner forces are gathered across subdomain faces in the undecomposed
    corner order and nodal mass is summed in global order, so both copies of
    a shared node are computed alike and need no PosVel copy."""
    cycles = 200
    node = ["x", "y", "z", "xd", "yd", "zd"]
    elem = ["e", "p", "q", "v", "ss"]
    G = tp * nx
    with lulesh.LuleshSet(nx=G, its=cycles) as single:
        assert single.run() == lulesh.OK
        ref_n = {f: single.field(f).reshape(G + 1, G + 1, G + 1) for f in node}
        ref_e = {f: single.field(f).reshape(G, G, G) for f in elem}
    with lulesh.LuleshSet(nx=nx, tp=tp, its=cycles) as sub:
        assert sub.run() == lulesh.OK
        for r in range(tp ** 3):
            c, w, p = r % tp, (r // tp) % tp, r // (tp * tp)
            for f in elem:
                got = sub.field(f, domain=r)[:nx ** 3].reshape(nx, nx, nx)
                want = ref_e[f][p * nx:(p + 1) * nx, w * nx:(w + 1) * nx, c * nx:(c + 1) * nx]
                assert np.array_equal(got, want), (r, f)
            for f in node:
                got = sub.field(f, domain=r).reshape(nx + 1, nx + 1, nx + 1)
                want = ref_n[f][p * nx:(p + 1) * nx + 1, w * nx:(w + 1) * nx + 1,
                                c * nx:(c + 1) * nx + 1]
                assert np.array_equal(got, want), (r, f)


def test_subdomains_staged_comm_matches(lulesh):
    """The reference's CommSend/CommSBN/CommSyncPosVel/CommMonoQ sequence over
    per-rank receive buffers agrees with the single domain to the 1e-9
    gate (the SBN sums associate differently at shared edges/corners)."""
    tp, nx, cycles = 2, 8, 40
    with lulesh.LuleshSet(nx=tp * nx, its=cycles) as single:
        assert single.run() == lulesh.OK
        e1 = single.origin_energy()
    with lulesh.LuleshSet(nx=nx, tp=tp, its=cycles, flags=lulesh.FLAG_COMM_STAGED) as sub:
        assert sub.run() == lulesh.OK
        e2 = sub.origin_energy()
    assert rel(e2, e1) < E_TOL


def test_batch_jobs_match_their_own_runs(lulesh):
    """Independent jobs of different sizes advance together; each equals its
    own single-job run bit for bit."""
    jobs = [lulesh.JobSpec(6, 5, 1, 1, 20), lulesh.JobSpec(11, 20, 4, 2, 35),
            lulesh.JobSpec(9, 11, 2, 4, 10), lulesh.JobSpec(14, 7, 1, 1, 25)]
    with lulesh.LuleshSet.batch(jobs) as b:
        assert b.run() == lulesh.OK
        got = [b.origin_energy(j) for j in range(len(jobs))]
        cyc = [b.state(j)["cycle"] for j in range(len(jobs))]
    for j, spec in enumerate(jobs):
        with lulesh.LuleshSet(nx=spec.nx, numReg=spec.numReg, balance=spec.balance,
                              cost=spec.cost, its=spec.its) as s:
            assert s.run() == lulesh.OK
            assert got[j] == s.origin_energy()
            assert cyc[j] == spec.its


def test_volume_error_status(lulesh):
    """A negative element volume ends the job with VolumeError (-1) and the
    offending element, as checkErrors does (lulesh.cu:2879-2892)."""
    with lulesh.LuleshSet(nx=6, its=10) as gs:
        v = gs.field("v")
        v[17] = -1.0
        gs.set_field("v", v)
        st = gs.run()
        assert st == lulesh.VOLUME_ERROR
        s = gs.state()
        assert s["status"] == lulesh.VOLUME_ERROR and s["bad_elem"] == 17
        assert s["cycle"] == 1


def test_qstop_error_status(lulesh):
    """q above qstop ends the job with QStopError (-2).  p = -q keeps the
    element's stress (-p-q) at zero so no volume inverts first (checkErrors
    tests the volume flag before the q flag)."""
    with lulesh.LuleshSet(nx=6, its=10) as gs:
        q = gs.field("q")
        p = gs.field("p")
        q[5] = 2.0e12
        p[5] = -2.0e12
        gs.set_field("q", q)
        gs.set_field("p", p)
        assert gs.run() == lulesh.QSTOP_ERROR
        s = gs.state()
        assert s["bad_elem"] == 5


def test_host_driven_cycle_matches_graph_run(lulesh):
    """lulesh_host_cycle (host passes the time state in, reads it back) gives
    the same trajectory as the device-resident loop."""
    with lulesh.LuleshSet(nx=10, its=15) as a:
        assert a.run() == lulesh.OK
        ea = a.origin_energy()
    with lulesh.LuleshSet(nx=10, its=15) as b:
        st, out = b.host_cycle(None)
        for _ in range(14):
            st, out = b.host_cycle(out)
            assert st == lulesh.OK
        assert out.cycle == 15
        assert b.origin_energy() == ea


def test_host_driven_cycle_takes_the_hosts_time_state(lulesh):
    """The time state the host passes in is the one the cycle starts from:
    moving the clock forward changes the trajectory, and the record handed
    back is the device's after the cycle.  Plain steps and host cycles mix."""
    with lulesh.LuleshSet(nx=10, its=-1) as a, lulesh.LuleshSet(nx=10, its=-1) as b:
        a.step(3)
        b.step(3)
        _, oa = a.host_cycle(None)
        _, ob = b.host_cycle(None)
        assert (oa.time, oa.deltatime, oa.cycle) == (ob.time, ob.deltatime, ob.cycle) == (
            oa.time, oa.deltatime, 4)
        _, oa = a.host_cycle(oa)
        moved = lulesh.JobState()
        ctypes_fields = [f for f, _ in lulesh.JobState._fields_]
        for f in ctypes_fields:
            setattr(moved, f, getattr(ob, f))
        moved.time = ob.time + 1.0e-4
        _, ob = b.host_cycle(moved)
        assert ob.cycle == oa.cycle == 5
        assert ob.time > oa.time
        st_a, st_b = a.state(), b.state()
        assert st_a["time"] == oa.time and st_b["time"] == ob.time
        assert st_a["deltatime"] == oa.deltatime and st_b["deltatime"] == ob.deltatime


def test_profile_phases(lulesh):
    with lulesh.LuleshSet(nx=20, its=-1) as gs:
        ph = gs.profile_phases(3)
        assert set(ph) >= {"force", "nodal", "kinematics", "eos"}
        assert all(v >= 0 for v in ph.values())
