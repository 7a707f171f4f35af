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


@pytest.mark.parametrize("nparts", [2, 4, 8])
def test_parts_on_one_gpu_match_single_domain(lulesh, nparts):
    torch = pytest.importorskip("torch")
    import distributed as D

    nx, tp, cycles = 6, 2, 30
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [D.GpuPart(nx, tp, nparts, p, device=0, stream=stream) for p in range(nparts)]
        eng = D.Engine(parts, D.LocalTransport())
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
