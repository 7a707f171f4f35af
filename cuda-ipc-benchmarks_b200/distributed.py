"""One LULESH problem over several GPUs: the reference's multi-rank run.

The reference runs one MPI rank per GPU, each with one subdomain of a cube
decomposition (InitMeshDecomp, LULESH/cuda/src/lulesh.cu:4606-4668), and
moves halos between ranks three times per cycle (CommSBN of the nodal
forces, CommSyncPosVel, CommMonoQ; lulesh.cu:2897-2921, 3061-3094,
4165-4190) plus one MIN reduction of dt (lulesh.cu:1423-1429), through one
of its comm backends (LULESH/cuda/README.md:18-113).

Here each process drives one GPU's *part*: a set of consecutive subdomains
(lulesh_create_part) plus proxies of the neighbours that live on other
parts.  What crosses between parts is planned by lulesh_halo_plan: corner
forces instead of partial nodal sums, so every node still adds its corners
in corner order over the whole mesh and a decomposed run gives the
single-domain results bit for bit (the in-device 2x2x2 run does the same).

Pieces:
  GpuPart          one GPU's part: the set, its device message buffers, and
                   the phase / pack / unpack / dt calls of the C ABI
  NcclTransport    torch.distributed over NCCL: grouped send/recv of the
                   device buffers, all_reduce(MIN) of the dt record; one
                   part per process
  HostTransport    the same over a host backend (gloo): device -> host,
                   send/recv and all_reduce on the host, host -> device
  LocalTransport   every part in this process (device copies); lets one GPU
                   run the whole multi-part path
  DirectTransport  peer stores: each message is written by the sender's kernel
                   straight into the receiver's mailbox (CUDA IPC across
                   processes), with an arrival flag the receiver's kernel
                   waits on for a bounded time
  Engine           the cycle: phases, the three exchanges, the dt reduction

A rank that fails or never arrives makes the others' next exchange end with
an error after the process group's timeout (no device-side waiting is
involved: the transports block on the host).
"""
from __future__ import annotations

import ctypes

import numpy as np

import lulesh_b200 as L

KINDS = (L.HALO_CORNERS, L.HALO_POSVEL, L.HALO_MONOQ, L.HALO_MASS)
CYCLE_KINDS = (L.HALO_CORNERS, L.HALO_POSVEL, L.HALO_MONOQ)


# ---------------------------------------------------------------------------
# the plan (host only)

def part_of(rank: int, tp: int, nparts: int) -> int:
    """Part holding subdomain `rank` (rank * nparts // tp^3)."""
    return int(L.load_library().lulesh_part_of(rank, tp, nparts))


def peers(tp: int, nparts: int, part: int) -> list[int]:
    lib = L.load_library()
    buf = (ctypes.c_int * 64)()
    n = lib.lulesh_halo_peers(tp, nparts, part, buf, 64)
    if n < 0:
        raise ValueError(f"lulesh_halo_peers({tp}, {nparts}, {part}) = {n}")
    return [buf[i] for i in range(n)]


def plan(nx: int, tp: int, nparts: int, src: int, dst: int, kind: int):
    """The message of `kind` from part src to part dst: arrays (rank, field
    id, index), item i being field[i] of subdomain rank[i] at index[i]."""
    lib = L.load_library()
    n = lib.lulesh_halo_plan(nx, tp, nparts, src, dst, kind, None, None, None, 0)
    if n < 0:
        raise ValueError(f"lulesh_halo_plan: status {n}")
    r = np.empty(n, np.int32)
    f = np.empty(n, np.int32)
    i = np.empty(n, np.int64)
    lib.lulesh_halo_plan(nx, tp, nparts, src, dst, kind,
                         r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                         f.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                         i.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), n)
    return r, f, i


def weak_scaling_edge(nparts: int, tp: int = 2, elems_per_part: float = 1e6) -> int:
    """Subdomain edge giving each of nparts GPUs about elems_per_part."""
    return max(1, int(round((elems_per_part * nparts / tp ** 3) ** (1.0 / 3.0))))


# ---------------------------------------------------------------------------
# one GPU's part

class GpuPart:
    """The part of a tp^3 problem (subdomains of edge nx) that one GPU holds.
    All of its work goes to `stream` (default: torch's current stream, which
    must not be the legacy default stream), the stream torch.distributed
    orders its NCCL calls after."""

    def __init__(self, nx: int, tp: int, nparts: int, part: int, numReg: int = 11,
                 balance: int = 1, cost: int = 1, its: int = -1, device: int | None = None,
                 stream=None):
        import torch

        self.torch = torch
        self.lib = L.load_library()
        self.nx, self.tp, self.nparts, self.part = nx, tp, nparts, part
        dev = torch.cuda.current_device() if device is None else device
        h = ctypes.c_void_p()
        job = L.JobSpec(nx, numReg, balance, cost, its).c()
        L._check(self.lib, self.lib.lulesh_create_part(ctypes.byref(job), tp, nparts, part, 0,
                                                       dev, ctypes.byref(h)),
                 "lulesh_create_part")
        self.set = L.LuleshSet(_handle=h)
        self.h = h
        self.stream = stream if stream is not None else torch.cuda.current_stream(dev)
        if self.stream.cuda_stream == 0:
            raise ValueError("GpuPart needs a stream other than the legacy default stream")
        self.set.set_stream(self.stream.cuda_stream)
        self.peers = peers(tp, nparts, part)
        self.send, self.recv = {}, {}
        for k in KINDS:
            self.send[k], self.recv[k] = {}, {}
            for q in self.peers:
                ns = int(self.lib.lulesh_halo_count(h, k, q, 1))
                nr = int(self.lib.lulesh_halo_count(h, k, q, 0))
                if ns < 0 or nr < 0:
                    raise L.LuleshError(min(ns, nr), "lulesh_halo_count")
                self.send[k][q] = torch.zeros(ns, dtype=torch.float64, device=dev)
                self.recv[k][q] = torch.zeros(nr, dtype=torch.float64, device=dev)
        self.dt = torch.zeros(4, dtype=torch.int64, device=dev)

    def _ck(self, st, what):
        L._check(self.lib, st, what)

    def phase(self, ph: int) -> None:
        self._ck(self.lib.lulesh_part_phase(self.h, ph), "lulesh_part_phase")

    def pack(self, kind: int) -> None:
        for q, b in self.send[kind].items():
            if b.numel():
                self._ck(self.lib.lulesh_halo_pack(self.h, kind, q, b.data_ptr()),
                         "lulesh_halo_pack")

    def unpack(self, kind: int) -> None:
        for q, b in self.recv[kind].items():
            if b.numel():
                self._ck(self.lib.lulesh_halo_unpack(self.h, kind, q, b.data_ptr()),
                         "lulesh_halo_unpack")

    def dt_pack(self):
        self._ck(self.lib.lulesh_part_dt_pack(self.h, self.dt.data_ptr()), "lulesh_part_dt_pack")
        return self.dt

    def dt_unpack(self, buf) -> None:
        self._ck(self.lib.lulesh_part_dt_unpack(self.h, buf.data_ptr()), "lulesh_part_dt_unpack")

    def finish_setup(self) -> None:
        self._ck(self.lib.lulesh_part_finish_setup(self.h), "lulesh_part_finish_setup")

    def halo_doubles(self, kinds=CYCLE_KINDS) -> int:
        """Doubles this part sends per cycle."""
        return sum(b.numel() for k in kinds for b in self.send[k].values())

    def close(self) -> None:
        if getattr(self, "set", None) is not None:
            self.set.close()
            self.set = None


# ---------------------------------------------------------------------------
# transports

class LocalTransport:
    """Every part lives in this process: a message is a copy from the
    sender's buffer into the receiver's (on the current stream)."""

    name = "local"

    def exchange(self, kind, parts) -> None:
        by_part = {p.part: p for p in parts}
        for p in parts:
            for q, buf in p.send[kind].items():
                if buf.numel():
                    by_part[q].recv[kind][p.part].copy_(buf)

    def allreduce_min(self, bufs) -> None:
        m = bufs[0].clone()
        for b in bufs[1:]:
            m = m.minimum(b)
        for b in bufs:
            b.copy_(m)


class NcclTransport:
    """One part per process; torch.distributed with the NCCL backend
    (process rank = part).  Grouped send/recv of the device buffers, then
    all_reduce(MIN) of the dt record, both ordered after the work already
    on the current stream."""

    name = "nccl"

    def __init__(self, dist):
        self.dist = dist

    def exchange(self, kind, parts) -> None:
        (p,) = parts
        d = self.dist
        ops = []
        for q in p.peers:
            if p.send[kind][q].numel():
                ops.append(d.P2POp(d.isend, p.send[kind][q], q))
            if p.recv[kind][q].numel():
                ops.append(d.P2POp(d.irecv, p.recv[kind][q], q))
        if ops:
            for r in d.batch_isend_irecv(ops):
                r.wait()

    def allreduce_min(self, bufs) -> None:
        (b,) = bufs
        self.dist.all_reduce(b, op=self.dist.ReduceOp.MIN)


class HostTransport:
    """One part per process over a host backend (gloo): each message is
    copied to the host, sent, received, and copied to the device.  Every
    wait is bounded by timeout_s: a peer that never sends (it failed, or
    left) ends the exchange with an exception instead of a hang."""

    name = "host"

    def __init__(self, dist, timeout_s: float = 120.0):
        import datetime

        self.dist = dist
        self.timeout = datetime.timedelta(seconds=timeout_s)

    def exchange(self, kind, parts) -> None:
        (p,) = parts
        d = self.dist
        reqs, inbox = [], {}
        for q in p.peers:
            if p.send[kind][q].numel():
                reqs.append(d.isend(p.send[kind][q].cpu(), q))
            if p.recv[kind][q].numel():
                inbox[q] = p.recv[kind][q].new_empty(p.recv[kind][q].shape, device="cpu")
                reqs.append(d.irecv(inbox[q], q))
        for r in reqs:
            r.wait(self.timeout)
        for q, t in inbox.items():
            p.recv[kind][q].copy_(t)

    def allreduce_min(self, bufs) -> None:
        (b,) = bufs
        c = b.cpu()
        self.dist.all_reduce(c, op=self.dist.ReduceOp.MIN)
        b.copy_(c)


class DirectTransport:
    """Peer stores (the reference's remote-pack IPC backend, with its tokens
    in device memory): a sender's kernel writes each message straight into
    the receiver's mailbox over peer memory and raises an arrival flag; the
    receiver's kernel waits for the flag (at most timeout_ms, then the job
    stops with LULESH_TIMEOUT) and scatters the message into its proxies.
    No staging buffer and no copy engine between the kernels.

    dist=None: every part is in this process (the mailboxes are plain device
    pointers).  Otherwise one part per process: the mailboxes are exported
    as CUDA IPC handles and exchanged with all_gather_object, and the dt
    record is reduced with all_reduce(MIN) over `dist` (NCCL); that
    reduction is also what makes reusing a mailbox next cycle safe."""

    name = "direct"
    handles_packing = True

    def __init__(self, dist=None, timeout_ms: float = 5000.0):
        self.dist = dist
        self.timeout_ms = timeout_ms
        self.seq = {k: 0 for k in KINDS}
        self.connected = False

    def _connect(self, parts) -> None:
        lib = L.load_library()
        if self.dist is None:
            ptr = {}
            for p in parts:
                v = ctypes.c_void_p()
                L._check(lib, lib.lulesh_part_mailbox(p.h, ctypes.byref(v), None, None),
                         "lulesh_part_mailbox")
                ptr[p.part] = v.value
            for p in parts:
                for q in p.peers:
                    L._check(lib, lib.lulesh_part_set_peer_mailbox(p.h, q, ctypes.c_void_p(ptr[q]),
                                                                  None),
                             "lulesh_part_set_peer_mailbox")
        else:
            (p,) = parts
            h = ctypes.create_string_buffer(64)
            L._check(lib, lib.lulesh_part_mailbox(p.h, None, None, h), "lulesh_part_mailbox")
            handles = [None] * self.dist.get_world_size()
            self.dist.all_gather_object(handles, h.raw)
            for q in p.peers:
                hq = ctypes.create_string_buffer(handles[q], 64)
                L._check(lib, lib.lulesh_part_set_peer_mailbox(p.h, q, None, hq),
                         "lulesh_part_set_peer_mailbox")
        self.connected = True

    def exchange(self, kind, parts) -> None:
        if not self.connected:
            self._connect(parts)
        lib = L.load_library()
        self.seq[kind] += 1
        seq = self.seq[kind]
        for p in parts:
            for q in p.peers:
                if p.send[kind][q].numel():
                    L._check(lib, lib.lulesh_halo_put(p.h, kind, q, seq), "lulesh_halo_put")
        for p in parts:
            for q in p.peers:
                if p.recv[kind][q].numel():
                    L._check(lib, lib.lulesh_halo_take(p.h, kind, q, seq, self.timeout_ms),
                             "lulesh_halo_take")

    def allreduce_min(self, bufs) -> None:
        if self.dist is None:
            LocalTransport().allreduce_min(bufs)
        else:
            (b,) = bufs
            self.dist.all_reduce(b, op=self.dist.ReduceOp.MIN)


# ---------------------------------------------------------------------------
# the cycle

class Engine:
    """Drives the parts of this process through set-up and cycles.  The
    order is that of LagrangeLeapFrog (lulesh.cu:4438-4452) with each halo
    exchange where the reference calls its comm backend.

    sync_posvel: also exchange the POSVEL messages and copy them into the
    receivers' max-side node faces (CommSyncPosVel).  Off by default: each
    part receives every corner force its nodes need (CORNERS) and the
    global node masses (MASS), sums them in the single-domain order, and so
    computes the shared nodes exactly as their +side owner does; the copy
    would write the values already there.  The reference needs it because
    its ranks add partial sums in their own orders."""

    def __init__(self, parts, transport, sync_posvel: bool = False):
        self.parts = list(parts)
        self.transport = transport
        self.sync_posvel = sync_posvel

    @property
    def cycle_kinds(self):
        """The message kinds exchanged every cycle."""
        if self.sync_posvel:
            return CYCLE_KINDS
        return tuple(k for k in CYCLE_KINDS if k != L.HALO_POSVEL)

    def exchange(self, kind: int) -> None:
        if getattr(self.transport, "handles_packing", False):
            self.transport.exchange(kind, self.parts)  # kernels store into peers directly
            return
        for p in self.parts:
            p.pack(kind)
        self.transport.exchange(kind, self.parts)
        for p in self.parts:
            p.unpack(kind)

    def setup(self) -> None:
        """The init-time nodal mass exchange (lulesh.cu:4811-4831)."""
        self.exchange(L.HALO_MASS)
        for p in self.parts:
            p.finish_setup()

    def _phase(self, *phases) -> None:
        for p in self.parts:
            for ph in phases:
                p.phase(ph)

    def cycle(self) -> None:
        self._phase(L.PHASE_TIME_INCREMENT, L.PHASE_FORCE)
        self.exchange(L.HALO_CORNERS)        # CommSend + CommSBN of the forces
        self._phase(L.PHASE_NODAL)
        if self.sync_posvel:
            self.exchange(L.HALO_POSVEL)     # CommSyncPosVel
            self._phase(L.PHASE_POSVEL_SYNC)
        self._phase(L.PHASE_KINEMATICS)
        self.exchange(L.HALO_MONOQ)          # CommMonoQ
        self._phase(L.PHASE_MONOQ_GHOST, L.PHASE_EOS)
        bufs = [p.dt_pack() for p in self.parts]
        self.transport.allreduce_min(bufs)   # MPI_Allreduce(MIN) of dt
        for p, b in zip(self.parts, bufs):
            p.dt_unpack(b)

    def run(self, ncycles: int) -> None:
        for _ in range(ncycles):
            self.cycle()

    def launches_per_cycle(self) -> int:
        """Kernels one cycle launches on each part (phases, packs, unpacks,
        dt pack/unpack; transport kernels not counted)."""
        p = self.parts[0]
        n = (7 if self.sync_posvel else 6) + 2
        for k in self.cycle_kinds:
            n += sum(1 for b in p.send[k].values() if b.numel())
            n += sum(1 for b in p.recv[k].values() if b.numel())
        return n


# ---------------------------------------------------------------------------
# the N-GPU bench leg

def bench_decomposed(warmup: int, steps: int, dist, transport: str = "nccl",
                     clock=None) -> dict:
    """Each process (one per GPU) runs its part of a 2x2x2 (or larger cube)
    decomposition sized so every GPU holds about 1e6 elements; device time
    of `steps` cycles after `warmup`, max over ranks.  Then `steps` more
    cycles driven from the host with each cycle's reduced dt record read
    back to the host (32 bytes), timed on the host clock, max over ranks:
    the end-to-end figure.  `clock` (start()/stop(), rank 0) samples the
    GPU clocks over the device-timed cycles."""
    import time

    import torch

    world, rank = dist.get_world_size(), dist.get_rank()
    tp = 2
    while tp ** 3 < world:
        tp += 1
    nx = weak_scaling_edge(world, tp)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    part = GpuPart(nx, tp, world, rank, stream=stream)
    tr = {"nccl": NcclTransport, "host": HostTransport,
          "direct": DirectTransport}[transport](dist)
    dist.barrier()
    eng = Engine([part], tr)
    eng.setup()
    eng.run(warmup)
    torch.cuda.synchronize()
    dist.barrier()
    if clock is not None:
        clock.start()
        time.sleep(0.3)  # the sampler is running before the timed cycles
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    eng.run(steps)
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = clock.stop() if clock is not None else None
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    ms = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    st = part.set.state()
    energy = part.set.origin_energy() if part_of(0, tp, world) == rank else None
    # end to end: the host drives every cycle and reads its result back
    dist.barrier()
    tw = time.perf_counter()
    for _ in range(steps):
        eng.cycle()
        part.dt.cpu()
    e2e_s = torch.tensor([time.perf_counter() - tw], dtype=torch.float64, device=dev)
    dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    out = {"ms_max_over_ranks": float(ms.item()), "sub_nx": nx, "tp": tp,
           "e2e_s_max_over_ranks": float(e2e_s.item()), "e2e_d2h_bytes_per_step": 8 * 4,
           "clocks": clocks,
           "global_nx": nx * tp, "zones_total": (nx * tp) ** 3, "transport": tr.name,
           "energy": energy, "cycle": st["cycle"], "status": st["status"],
           "launches_per_cycle": eng.launches_per_cycle(),
           "halo_bytes_per_cycle": 8 * part.halo_doubles(eng.cycle_kinds)}
    part.close()
    return out


def _main(argv=None) -> int:
    """`python distributed.py --parts 8 --nx 32 --cycles 10`: every part of a
    tp^3 problem on this process's GPU (LocalTransport, one stream), then
    the origin energy next to the single-domain run's of the same mesh."""
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--parts", type=int, default=8)
    ap.add_argument("--tp", type=int, default=2)
    ap.add_argument("--nx", type=int, default=32, help="subdomain edge")
    ap.add_argument("--cycles", type=int, default=10)
    ap.add_argument("--transport", default="local", choices=["local", "direct"])
    a = ap.parse_args(argv)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [GpuPart(a.nx, a.tp, a.parts, p, stream=stream) for p in range(a.parts)]
        eng = Engine(parts, LocalTransport() if a.transport == "local" else DirectTransport())
        eng.setup()
        eng.run(a.cycles)
    torch.cuda.synchronize()
    e = parts[0].set.origin_energy()
    with L.LuleshSet(nx=a.nx * a.tp, its=a.cycles) as single:
        single.run()
        e1 = single.origin_energy()
    print(json.dumps({"parts": a.parts, "tp": a.tp, "nx": a.nx, "cycles": a.cycles,
                      "origin_energy": e, "single_domain": e1, "equal": e == e1}))
    for p in parts:
        p.close()
    return 0 if e == e1 else 1


if __name__ == "__main__":
    raise SystemExit(_main())
