"""The multi-GPU path on one GPU: every part of the problem in this process.

Each part is a set from lulesh_create_part with its proxies, packs and
unpacks its halo messages through the C ABI, and the messages move by device
copies (distributed.LocalTransport) in place of NCCL.  The parts share one
stream, so nothing waits on another kernel.  The decomposed run must equal
the single-domain run (and the in-device 2x2x2 set) bit for bit.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ELEM = ["e", "p", "q", "v", "ss", "volo", "elemMass", "arealg", "vdov"]
NODE = ["x", "y", "z", "xd", "yd", "zd", "nodalMass"]


def _region(nx, tp, r):
    c, w, p = r % tp, (r // tp) % tp, r // (tp * tp)
    G = nx * tp
    ie, ine = np.arange(nx), np.arange(nx + 1)
    ge = (((p * nx + ie[:, None, None]) * G + (w * nx + ie[None, :, None])) * G
          + (c * nx + ie[None, None, :])).ravel()
    gn = (((p * nx + ine[:, None, None]) * (G + 1) + (w * nx + ine[None, :, None])) * (G + 1)
          + (c * nx + ine[None, None, :])).ravel()
    return ge, gn


@pytest.mark.parametrize("nparts,sync_posvel", [(2, False), (4, False), (8, False), (2, True),
                                                (8, True)])
def test_parts_on_one_gpu_match_single_domain(lulesh, nparts, sync_posvel):
    torch = pytest.importorskip("torch")
    import distributed as D

    nx, tp, cycles = 6, 2, 30
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [D.GpuPart(nx, tp, nparts, p, device=0, stream=stream) for p in range(nparts)]
        eng = D.Engine(parts, D.LocalTransport(), sync_posvel=sync_posvel)
        eng.setup()
        eng.run(cycles)
    torch.cuda.synchronize()
    with lulesh.LuleshSet(nx=nx * tp, its=-1, device=0) as single:
        single.step(cycles)
        ref = {f: single.field(f) for f in ELEM + NODE}
        e_ref = single.origin_energy()
        st_ref = single.state()
    assert parts[0].set.origin_energy() == e_ref
    for p in parts:
        st = p.set.state()
        assert st["cycle"] == cycles and st["status"] == 0
        assert st["time"] == st_ref["time"] and st["deltatime"] == st_ref["deltatime"]
        for d in range(p.set.num_domains):
            rank = [q for q in range(tp ** 3) if D.part_of(q, tp, nparts) == p.part][d]
            ge, gn = _region(nx, tp, rank)
            for f in ELEM:
                assert np.array_equal(p.set.field(f, d)[:nx ** 3], ref[f][ge]), (p.part, rank, f)
            for f in NODE:
                assert np.array_equal(p.set.field(f, d), ref[f][gn]), (p.part, rank, f)
    for p in parts:
        p.close()


def test_part_without_origin_refuses_origin_energy_and_step(lulesh):
    torch = pytest.importorskip("torch")
    import distributed as D

    stream = torch.cuda.Stream()
    p = D.GpuPart(4, 2, 2, 1, device=0, stream=stream)
    with pytest.raises(lulesh.LuleshError):
        p.set.origin_energy()
    with pytest.raises(lulesh.LuleshError):
        p.set.step(1)  # a part of several GPUs advances through the exchange
    with pytest.raises(lulesh.LuleshError):
        p.phase(lulesh.PHASE_FORCE)  # MASS exchange and finish_setup first
    p.close()


@pytest.mark.parametrize("tp", [2, 3])
def test_device_nodal_mass_equals_host_builder(lulesh, tp):
    """Subdomain sets sum each node's mass over the whole problem on the
    device (the init-time nodalMass exchange as a gather); the host builder
    (LULESH_FLAG_HOST_SETUP) computes the same sum in the same order."""
    nx = 5
    with lulesh.LuleshSet(nx=nx, tp=tp, its=-1, device=0) as dev, \
            lulesh.LuleshSet(nx=nx, tp=tp, its=-1, flags=lulesh.FLAG_HOST_SETUP,
                             device=0) as host:
        for d in range(tp ** 3):
            for f in ("nodalMass", "volo", "elemMass", "x", "y", "z", "e"):
                assert np.array_equal(dev.field(f, d), host.field(f, d)), (d, f)
        dev.step(20)
        host.step(20)
        assert dev.origin_energy() == host.origin_energy()


def test_bounded_flag_wait_times_out_and_the_context_survives(lulesh):
    """A wait on a flag that nothing sets gives up after its limit, stops the
    set's job with LULESH_TIMEOUT, and the device keeps working."""
    torch = pytest.importorskip("torch")
    lib = lulesh.load_library()
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    with lulesh.LuleshSet(nx=4, its=-1, device=0) as s:
        st = lib.lulesh_wait_flag(s.h, ctypes.c_void_p(flag.data_ptr()), 1, 200.0)
        assert st == lulesh.OK
        s.sync()
        assert s.state()["status"] == lulesh.TIMEOUT
        assert s.state()["done"] == 1
    flag.fill_(1)
    with lulesh.LuleshSet(nx=4, its=5, device=0) as s:
        assert lib.lulesh_wait_flag(s.h, ctypes.c_void_p(flag.data_ptr()), 1, 200.0) == 0
        s.sync()
        assert s.state()["status"] == lulesh.OK
        assert s.run() == lulesh.OK  # the context is usable
        assert s.state()["cycle"] == 5


def _two_proc_worker(rank, port, nx, cycles, q):
    import datetime
    import os
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "cuda-ipc-benchmarks_b200"))
    try:
        import torch
        import torch.distributed as dist

        import distributed as D

        torch.cuda.set_device(0)
        dist.init_process_group("gloo", rank=rank, world_size=2,
                                timeout=datetime.timedelta(seconds=60))
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        part = D.GpuPart(nx, 2, 2, rank, device=0, stream=stream)
        eng = D.Engine([part], D.HostTransport(dist, timeout_s=60.0))
        dist.barrier()
        eng.setup()
        eng.run(cycles)
        torch.cuda.synchronize()
        fields = {d: {f: part.set.field(f, d) for f in ELEM + NODE}
                  for d in range(part.set.num_domains)}
        st = part.set.state()
        e0 = part.set.origin_energy() if rank == 0 else None
        part.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok", fields, st, e0))
    except Exception as e:  # noqa: BLE001
        q.put((rank, "error", repr(e)[:400], None, None))


def test_two_processes_on_one_gpu_match_single_domain(lulesh):
    """Two processes, each with its own GpuPart on this GPU, exchange their
    halo messages and dt through the host transport over gloo: the hosts
    wait on each other, no kernel waits on another.  The decomposed run
    equals the single domain bit for bit."""
    import os

    import torch.multiprocessing as mp

    nx, cycles = 6, 25
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 2000
    procs = [ctx.Process(target=_two_proc_worker, args=(r, port, nx, cycles, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    assert [r[1] for r in res] == ["ok", "ok"], res
    with lulesh.LuleshSet(nx=nx * 2, its=-1, device=0) as single:
        single.step(cycles)
        ref = {f: single.field(f) for f in ELEM + NODE}
        e_ref = single.origin_energy()
    assert res[0][4] == e_ref
    import distributed as D
    for rank, _, fields, st, _ in res:
        assert st["cycle"] == cycles and st["status"] == 0
        ranks = [q2 for q2 in range(8) if D.part_of(q2, 2, 2) == rank]
        for d, f_d in fields.items():
            ge, gn = _region(nx, 2, ranks[d])
            for f in ELEM:
                assert np.array_equal(f_d[f][:nx ** 3], ref[f][ge]), (rank, d, f)
            for f in NODE:
                assert np.array_equal(f_d[f], ref[f][gn]), (rank, d, f)


@pytest.mark.parametrize("nparts,sync_posvel", [(2, False), (8, False), (8, True)])
def test_direct_transport_parts_on_one_gpu(lulesh, nparts, sync_posvel):
    """The direct transport with every part in this process: each put kernel
    stores its message into the receiver's mailbox and raises the flag
    before the receiver's take kernel runs (one stream), so no wait spins.
    The run equals the single domain bit for bit."""
    torch = pytest.importorskip("torch")
    import distributed as D

    nx, tp, cycles = 6, 2, 30
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [D.GpuPart(nx, tp, nparts, p, device=0, stream=stream) for p in range(nparts)]
        eng = D.Engine(parts, D.DirectTransport(), sync_posvel=sync_posvel)
        eng.setup()
        eng.run(cycles)
    torch.cuda.synchronize()
    with lulesh.LuleshSet(nx=nx * tp, its=-1, device=0) as single:
        single.step(cycles)
        ref = {f: single.field(f) for f in ELEM + NODE}
        e_ref = single.origin_energy()
    assert parts[0].set.origin_energy() == e_ref
    for p in parts:
        assert p.set.state()["status"] == 0 and p.set.state()["cycle"] == cycles
        ranks = [q for q in range(tp ** 3) if D.part_of(q, tp, nparts) == p.part]
        for d in range(p.set.num_domains):
            ge, gn = _region(nx, tp, ranks[d])
            for f in ELEM:
                assert np.array_equal(p.set.field(f, d)[:nx ** 3], ref[f][ge]), (p.part, f)
            for f in NODE:
                assert np.array_equal(p.set.field(f, d), ref[f][gn]), (p.part, f)
    for p in parts:
        p.close()


def test_direct_transport_take_that_never_arrives_times_out(lulesh):
    """A take waiting for a sequence number no put has raised gives up after
    its limit: the job stops with LULESH_TIMEOUT, nothing is scattered, and
    the device keeps working."""
    torch = pytest.importorskip("torch")
    import distributed as D

    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [D.GpuPart(4, 2, 2, p, device=0, stream=stream) for p in range(2)]
        tr = D.DirectTransport(timeout_ms=200.0)
        eng = D.Engine(parts, tr)
        eng.setup()
        eng.run(2)
        lib = lulesh.load_library()
        p = parts[1]
        assert lib.lulesh_halo_take(p.h, lulesh.HALO_CORNERS, 0, 999, 200.0) == lulesh.OK
    torch.cuda.synchronize()
    st = parts[1].set.state()
    assert st["status"] == lulesh.TIMEOUT and st["done"] == 1
    assert parts[0].set.state()["status"] == lulesh.OK
    for p in parts:
        p.close()
    with lulesh.LuleshSet(nx=4, its=3, device=0) as s:
        assert s.run() == lulesh.OK
