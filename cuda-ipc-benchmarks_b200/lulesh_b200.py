"""ctypes binding of liblulesh_b200.so (include/lulesh_b200.h).

The binding is a thin layer over the C ABI: every call goes to the CUDA
library built in this directory, and a missing library raises instead of
falling back to anything else.  Names follow the reference's Domain fields
(LULESH/cuda/src/lulesh.h:40-298) and its command line (-s -r -b -c -i).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblulesh_b200.so")

OK = 0
VOLUME_ERROR = -1
QSTOP_ERROR = -2
FILE_ERROR = -3
CUDA_ERROR = -4
INVALID_ARG = -5
OOM = -6
TIMEOUT = -7
NO_DEVICE = -8
BOUNDS_ERROR = -9  # -DLULESH_CHECKED builds only

FLAG_MATERIALIZE = 0x1
FLAG_COMM_STAGED = 0x2
FLAG_MIXED = 0x4
FLAG_HOST_SETUP = 0x8

MAX_NX = 645  # LULESH_MAX_NX

MSG_COMM_SBN = 1024
MSG_SYNC_POS_VEL = 2048
MSG_MONOQ = 3072

FIELD_IDS = {
    "x": 0, "y": 1, "z": 2, "xd": 3, "yd": 4, "zd": 5, "fx": 6, "fy": 7,
    "fz": 8, "nodalMass": 9, "delv_xi": 10, "delv_eta": 11, "delv_zeta": 12,
    "fx_elem": 13, "fy_elem": 14, "fz_elem": 15, "volo": 16,
}
FIELD_NAMES = {v: k for k, v in FIELD_IDS.items()}

# halo message kinds of a problem split over GPUs (lulesh_halo_plan)
HALO_CORNERS, HALO_POSVEL, HALO_MONOQ, HALO_MASS = 0, 1, 2, 3
# phases of a part's cycle (lulesh_part_phase)
PHASE_TIME_INCREMENT, PHASE_FORCE, PHASE_NODAL, PHASE_POSVEL_SYNC = 0, 1, 2, 3
PHASE_KINEMATICS, PHASE_MONOQ_GHOST, PHASE_EOS = 4, 5, 6

INT_FIELDS = {
    "nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
    "matElemlist", "regNumList", "regElemlist", "nodeElemCount",
    "nodeElemStart", "nodeElemCornerList", "symmX", "symmY", "symmZ", "regCSR",
    "regReps", "regSorted", "eosOrder",
}

# every symbol include/lulesh_b200.h declares
EXPORTED = [
    "lulesh_create", "lulesh_create_batch", "lulesh_create_from_mesh", "lulesh_destroy",
    "lulesh_footprint_bytes", "lulesh_set_stream", "lulesh_lagrange_leapfrog",
    "lulesh_step", "lulesh_run", "lulesh_host_cycle", "lulesh_sync",
    "lulesh_num_jobs", "lulesh_num_domains", "lulesh_job_state_get",
    "lulesh_origin_energy", "lulesh_symmetry", "lulesh_field_bytes",
    "lulesh_get_field", "lulesh_set_field", "lulesh_domain_view_get",
    "lulesh_write_solution", "lulesh_status_string", "lulesh_last_error",
    "lulesh_comm_recv", "lulesh_comm_send", "lulesh_comm_sbn",
    "lulesh_comm_sync_posvel", "lulesh_comm_monoq", "lulesh_comm_recv_offset",
    "lulesh_profile_phases", "lulesh_phase_name", "lulesh_volume_force_noalloc",
    "lulesh_server_create", "lulesh_server_destroy", "lulesh_server_submit",
    "lulesh_server_step", "lulesh_server_poll", "lulesh_server_clock",
    "lulesh_set_graph_cycles", "lulesh_get_tuning", "lulesh_set_tuning",
    "lulesh_autotune", "lulesh_checkpoint_bytes", "lulesh_checkpoint_save",
    "lulesh_checkpoint_load", "lulesh_run_graph",
    "lulesh_part_of", "lulesh_halo_peers", "lulesh_halo_plan", "lulesh_create_part",
    "lulesh_part_finish_setup", "lulesh_halo_count", "lulesh_halo_pack", "lulesh_halo_unpack",
    "lulesh_part_phase", "lulesh_part_dt_pack", "lulesh_part_dt_unpack", "lulesh_wait_flag",
    "lulesh_measure_fp64_peak", "lulesh_part_mailbox", "lulesh_part_set_peer_mailbox",
    "lulesh_halo_put", "lulesh_halo_take",
]
# the host-only planning functions, also exported by liblulesh_host.so
HOST_PLAN_SIGS = {
    "lulesh_part_of": (ctypes.c_int, [ctypes.c_int] * 3),
    "lulesh_halo_peers": (ctypes.c_int, [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int),
                                                              ctypes.c_int]),
    "lulesh_halo_plan": (ctypes.c_longlong,
                         [ctypes.c_int] * 6 + [ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_longlong),
                                               ctypes.c_longlong]),
}


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_cap_bytes", ctypes.c_size_t), ("max_jobs", ctypes.c_int),
                ("cycles_per_step", ctypes.c_int), ("prepare_threads", ctypes.c_int),
                ("device", ctypes.c_int)]


class ServerResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_longlong), ("status", ctypes.c_int), ("cycle", ctypes.c_int),
                ("bad_elem", ctypes.c_int), ("origin_energy", ctypes.c_double),
                ("time", ctypes.c_double), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("elem_block", ctypes.c_int), ("node_block", ctypes.c_int),
                ("order", ctypes.c_int), ("graph_cycles", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(ctypes.Structure):
    _fields_ = [("tuning", Tuning), ("ms_per_cycle", ctypes.c_double)]


class Job(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("numReg", ctypes.c_int),
                ("balance", ctypes.c_int), ("cost", ctypes.c_int),
                ("its", ctypes.c_int)]


class JobState(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("bad_elem", ctypes.c_int),
                ("cycle", ctypes.c_int), ("done", ctypes.c_int),
                ("time", ctypes.c_double), ("deltatime", ctypes.c_double),
                ("dtcourant", ctypes.c_double), ("dthydro", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class LuleshError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load the CUDA library; raises FileNotFoundError if it was not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} is missing: build it with `make -C {HERE}` (nvcc, sm_100a)")
    lib = ctypes.CDLL(p)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "lulesh_create": (ip, [ctypes.POINTER(Job), ip, ip, ip, ctypes.POINTER(vp)]),
        "lulesh_create_batch": (ip, [ctypes.POINTER(Job), ip, ip, ip, ctypes.POINTER(vp)]),
        "lulesh_create_from_mesh": (ip, [ctypes.c_char_p, ctypes.POINTER(Job), ip, ip,
                                         ctypes.POINTER(vp)]),
        "lulesh_destroy": (ip, [vp]),
        "lulesh_footprint_bytes": (ctypes.c_size_t, [ctypes.POINTER(Job), ip, ip]),
        "lulesh_set_stream": (ip, [vp, vp]),
        "lulesh_lagrange_leapfrog": (ip, [vp]),
        "lulesh_step": (ip, [vp, ip]),
        "lulesh_run": (ip, [vp, ip]),
        "lulesh_host_cycle": (ip, [vp, ctypes.POINTER(JobState), ctypes.POINTER(JobState)]),
        "lulesh_sync": (ip, [vp]),
        "lulesh_num_jobs": (ip, [vp]),
        "lulesh_num_domains": (ip, [vp]),
        "lulesh_job_state_get": (ip, [vp, ip, ctypes.POINTER(JobState)]),
        "lulesh_origin_energy": (ip, [vp, ip, ctypes.POINTER(dp)]),
        "lulesh_symmetry": (ip, [vp, ip, ctypes.POINTER(dp), ctypes.POINTER(dp),
                                 ctypes.POINTER(dp)]),
        "lulesh_field_bytes": (ip, [vp, ip, ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t)]),
        "lulesh_get_field": (ip, [vp, ip, ctypes.c_char_p, vp, ctypes.c_size_t]),
        "lulesh_set_field": (ip, [vp, ip, ctypes.c_char_p, vp, ctypes.c_size_t]),
        "lulesh_domain_view_get": (ip, [vp, ip, vp]),
        "lulesh_write_solution": (ip, [vp, ip, ctypes.c_char_p]),
        "lulesh_status_string": (ctypes.c_char_p, [ip]),
        "lulesh_last_error": (ctypes.c_char_p, []),
        "lulesh_comm_recv": (ip, [vp, ip, ip, ip, ip, ip, ip, ip, ip]),
        "lulesh_comm_send": (ip, [vp, ip, ip, ip, ctypes.POINTER(ip), ip, ip, ip, ip, ip]),
        "lulesh_comm_sbn": (ip, [vp, ip, ip, ctypes.POINTER(ip)]),
        "lulesh_comm_sync_posvel": (ip, [vp, ip]),
        "lulesh_comm_monoq": (ip, [vp, ip]),
        "lulesh_comm_recv_offset": (ctypes.c_long, [vp, ip, ip, ip, ip, ip, ip, ip]),
        "lulesh_profile_phases": (ip, [vp, ip, ctypes.POINTER(dp), ctypes.POINTER(ip)]),
        "lulesh_phase_name": (ctypes.c_char_p, [ip]),
        "lulesh_volume_force_noalloc": (ip, [ip] + [vp] * 12 + [dp] + [vp] * 5),
        "lulesh_server_create": (ip, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
        "lulesh_server_destroy": (ip, [vp]),
        "lulesh_server_submit": (ip, [vp, ctypes.POINTER(Job), ctypes.POINTER(ctypes.c_longlong)]),
        "lulesh_server_step": (ip, [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]),
        "lulesh_server_poll": (ip, [vp, ctypes.POINTER(ServerResult), ip, ctypes.POINTER(ip)]),
        "lulesh_server_clock": (dp, []),
        "lulesh_set_graph_cycles": (ip, [vp, ip]),
        "lulesh_get_tuning": (ip, [vp, ctypes.POINTER(Tuning)]),
        "lulesh_set_tuning": (ip, [vp, ctypes.POINTER(Tuning)]),
        "lulesh_autotune": (ip, [vp, ip, ip, ctypes.POINTER(Tuning), ctypes.POINTER(TuneTrial),
                                 ip, ctypes.POINTER(ip)]),
        "lulesh_checkpoint_bytes": (ctypes.c_size_t, [vp]),
        "lulesh_checkpoint_save": (ip, [vp, vp, ctypes.c_size_t]),
        "lulesh_checkpoint_load": (ip, [vp, vp, ctypes.c_size_t]),
        "lulesh_run_graph": (ip, [vp, ctypes.c_longlong]),
        "lulesh_create_part": (ip, [ctypes.POINTER(Job), ip, ip, ip, ip, ip, ctypes.POINTER(vp)]),
        "lulesh_part_finish_setup": (ip, [vp]),
        "lulesh_halo_count": (ctypes.c_longlong, [vp, ip, ip, ip]),
        "lulesh_halo_pack": (ip, [vp, ip, ip, vp]),
        "lulesh_halo_unpack": (ip, [vp, ip, ip, vp]),
        "lulesh_part_phase": (ip, [vp, ip]),
        "lulesh_part_dt_pack": (ip, [vp, vp]),
        "lulesh_part_dt_unpack": (ip, [vp, vp]),
        "lulesh_wait_flag": (ip, [vp, vp, ctypes.c_uint, dp]),
        "lulesh_measure_fp64_peak": (ip, [ip, ctypes.POINTER(dp)]),
        "lulesh_part_mailbox": (ip, [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t), vp]),
        "lulesh_part_set_peer_mailbox": (ip, [vp, ip, vp, vp]),
        "lulesh_halo_put": (ip, [vp, ip, ip, ctypes.c_uint]),
        "lulesh_halo_take": (ip, [vp, ip, ip, ctypes.c_uint, dp]),
    }
    sig.update(HOST_PLAN_SIGS)
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _check(lib, st: int, what: str) -> int:
    if st != OK:
        detail = lib.lulesh_last_error().decode(errors="replace")
        name = lib.lulesh_status_string(st).decode()
        raise LuleshError(st, f"{what}: {name} {detail}".strip())
    return st


@dataclass
class JobSpec:
    nx: int
    numReg: int = 11
    balance: int = 1
    cost: int = 1
    its: int = -1

    def c(self) -> Job:
        return Job(self.nx, self.numReg, self.balance, self.cost, self.its)


def measure_fp64_peak(device: int = -1) -> float:
    """Measured FP64 FMA operations per second of the GPU
    (lulesh_measure_fp64_peak)."""
    lib = load_library()
    v = ctypes.c_double()
    _check(lib, lib.lulesh_measure_fp64_peak(device, ctypes.byref(v)), "lulesh_measure_fp64_peak")
    return v.value


def footprint_bytes(jobs: list[JobSpec], tp: int = 1) -> int:
    lib = load_library()
    arr = (Job * len(jobs))(*[j.c() for j in jobs])
    return int(lib.lulesh_footprint_bytes(arr, len(jobs), tp))


class LuleshSet:
    """One set of domains resident on one GPU (single domain, tp^3
    subdomains, or a batch of independent jobs)."""

    def __init__(self, nx: int = 30, tp: int = 1, numReg: int = 11, balance: int = 1,
                 cost: int = 1, its: int = -1, flags: int = 0, device: int = -1,
                 _handle=None):
        self.lib = load_library()
        if _handle is not None:
            self.h = _handle
        else:
            h = ctypes.c_void_p()
            job = JobSpec(nx, numReg, balance, cost, its).c()
            _check(self.lib, self.lib.lulesh_create(ctypes.byref(job), tp, flags, device,
                                                    ctypes.byref(h)), "lulesh_create")
            self.h = h
        self.tp = tp

    @classmethod
    def batch(cls, jobs: list[JobSpec], flags: int = 0, device: int = -1) -> "LuleshSet":
        lib = load_library()
        arr = (Job * len(jobs))(*[j.c() for j in jobs])
        h = ctypes.c_void_p()
        _check(lib, lib.lulesh_create_batch(arr, len(jobs), flags, device, ctypes.byref(h)),
               "lulesh_create_batch")
        return cls(_handle=h)

    @classmethod
    def from_mesh(cls, path: str, numReg: int = 11, balance: int = 1, cost: int = 1,
                  its: int = -1, flags: int = 0, device: int = -1) -> "LuleshSet":
        """One unstructured domain read from an lmesh file (the reference's
        `-u file.lmesh`); FILE_ERROR for a missing or malformed file."""
        lib = load_library()
        job = JobSpec(1, numReg, balance, cost, its).c()
        h = ctypes.c_void_p()
        _check(lib, lib.lulesh_create_from_mesh(str(path).encode(), ctypes.byref(job), flags,
                                                device, ctypes.byref(h)),
               "lulesh_create_from_mesh")
        return cls(_handle=h)

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.lulesh_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- stepping
    def step(self, ncycles: int = 1) -> None:
        _check(self.lib, self.lib.lulesh_step(self.h, ncycles), "lulesh_step")

    def run(self, check_every: int = 64) -> int:
        """Run to completion; returns the status (VolumeError/QStopError are
        returned, not raised, as the reference exits with them)."""
        st = self.lib.lulesh_run(self.h, check_every)
        if st not in (OK, VOLUME_ERROR, QSTOP_ERROR):
            _check(self.lib, st, "lulesh_run")
        return st

    def run_graph(self, max_cycles: int = 0) -> int:
        """Run to completion in one graph launch (a device-side loop over
        cycles); status as run()."""
        st = self.lib.lulesh_run_graph(self.h, max_cycles)
        if st not in (OK, VOLUME_ERROR, QSTOP_ERROR):
            _check(self.lib, st, "lulesh_run_graph")
        return st

    def sync(self) -> None:
        _check(self.lib, self.lib.lulesh_sync(self.h), "lulesh_sync")

    def set_graph_cycles(self, k: int) -> None:
        _check(self.lib, self.lib.lulesh_set_graph_cycles(self.h, k), "lulesh_set_graph_cycles")

    def tuning(self) -> dict:
        t = Tuning()
        _check(self.lib, self.lib.lulesh_get_tuning(self.h, ctypes.byref(t)), "lulesh_get_tuning")
        return t.as_dict()

    def set_tuning(self, elem_block: int = 128, node_block: int = 128, order: int = 0,
                   graph_cycles: int = 1) -> None:
        t = Tuning(elem_block, node_block, order, graph_cycles)
        _check(self.lib, self.lib.lulesh_set_tuning(self.h, ctypes.byref(t)), "lulesh_set_tuning")

    def autotune(self, trial_cycles: int = 10, rounds: int = 2) -> dict:
        """Time the candidate launch shapes from the current state (which is
        restored afterwards) and apply the fastest; returns the winner and
        every trial."""
        best = Tuning()
        trials = (TuneTrial * 64)()
        n = ctypes.c_int(0)
        _check(self.lib, self.lib.lulesh_autotune(self.h, trial_cycles, rounds, ctypes.byref(best),
                                                  trials, 64, ctypes.byref(n)), "lulesh_autotune")
        return {"best": best.as_dict(),
                "trials": [dict(trials[i].tuning.as_dict(), ms_per_cycle=trials[i].ms_per_cycle)
                           for i in range(n.value)]}

    def checkpoint(self) -> bytes:
        """The set's whole state (header + device arrays + time state)."""
        n = int(self.lib.lulesh_checkpoint_bytes(self.h))
        buf = ctypes.create_string_buffer(n)
        _check(self.lib, self.lib.lulesh_checkpoint_save(self.h, buf, n), "lulesh_checkpoint_save")
        return buf.raw

    def restore(self, ckpt: bytes) -> None:
        """Load a checkpoint taken from a set with the same jobs, tp and flags."""
        buf = ctypes.create_string_buffer(ckpt, len(ckpt))
        _check(self.lib, self.lib.lulesh_checkpoint_load(self.h, buf, len(ckpt)),
               "lulesh_checkpoint_load")

    def profile_phases(self, ncycles: int) -> dict:
        """Average ms per phase over `ncycles` separately launched cycles."""
        out = (ctypes.c_double * 12)()
        n = ctypes.c_int()
        _check(self.lib, self.lib.lulesh_profile_phases(self.h, ncycles, out, ctypes.byref(n)),
               "lulesh_profile_phases")
        return {self.lib.lulesh_phase_name(k).decode(): out[k] for k in range(n.value)}

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(self.lib, self.lib.lulesh_set_stream(self.h, stream_ptr), "lulesh_set_stream")

    def host_cycle(self, state_in: JobState | None = None) -> tuple[int, JobState]:
        out = JobState()
        st = self.lib.lulesh_host_cycle(self.h, ctypes.byref(state_in) if state_in else None,
                                        ctypes.byref(out))
        if st not in (OK, VOLUME_ERROR, QSTOP_ERROR):
            _check(self.lib, st, "lulesh_host_cycle")
        return st, out

    # -- results
    @property
    def num_jobs(self) -> int:
        return self.lib.lulesh_num_jobs(self.h)

    @property
    def num_domains(self) -> int:
        return self.lib.lulesh_num_domains(self.h)

    def state(self, job: int = 0) -> dict:
        s = JobState()
        _check(self.lib, self.lib.lulesh_job_state_get(self.h, job, ctypes.byref(s)),
               "lulesh_job_state_get")
        return s.as_dict()

    def origin_energy(self, job: int = 0) -> float:
        v = ctypes.c_double()
        _check(self.lib, self.lib.lulesh_origin_energy(self.h, job, ctypes.byref(v)),
               "lulesh_origin_energy")
        return v.value

    def symmetry(self, job: int = 0) -> tuple[float, float, float]:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib, self.lib.lulesh_symmetry(self.h, job, ctypes.byref(a), ctypes.byref(b),
                                                  ctypes.byref(c)), "lulesh_symmetry")
        return a.value, b.value, c.value

    def field(self, name: str, domain: int = 0) -> np.ndarray:
        nb = ctypes.c_size_t()
        _check(self.lib, self.lib.lulesh_field_bytes(self.h, domain, name.encode(),
                                                     ctypes.byref(nb)), "lulesh_field_bytes")
        dt = np.int32 if name in INT_FIELDS else np.float64
        out = np.empty(nb.value // np.dtype(dt).itemsize, dtype=dt)
        _check(self.lib, self.lib.lulesh_get_field(self.h, domain, name.encode(),
                                                   out.ctypes.data_as(ctypes.c_void_p),
                                                   nb.value), "lulesh_get_field")
        return out

    def set_field(self, name: str, values: np.ndarray, domain: int = 0) -> None:
        dt = np.int32 if name in INT_FIELDS else np.float64
        arr = np.ascontiguousarray(values, dtype=dt)
        _check(self.lib, self.lib.lulesh_set_field(self.h, domain, name.encode(),
                                                   arr.ctypes.data_as(ctypes.c_void_p),
                                                   arr.nbytes), "lulesh_set_field")

    def write_solution(self, path: str, domain: int = 0) -> None:
        _check(self.lib, self.lib.lulesh_write_solution(self.h, domain, path.encode()),
               "lulesh_write_solution")

    # -- comm backend (rank = subdomain index, -1 = all)
    def comm_recv(self, rank, msg, xfer, dx, dy, dz, do_recv, plane_only):
        _check(self.lib, self.lib.lulesh_comm_recv(self.h, rank, msg, xfer, dx, dy, dz,
                                                   int(do_recv), int(plane_only)), "CommRecv")

    def comm_send(self, rank, msg, fields, dx, dy, dz, do_send, plane_only):
        ids = (ctypes.c_int * len(fields))(*[FIELD_IDS[f] for f in fields])
        _check(self.lib, self.lib.lulesh_comm_send(self.h, rank, msg, len(fields), ids, dx, dy,
                                                   dz, int(do_send), int(plane_only)),
               "CommSend")

    def comm_sbn(self, rank, fields):
        ids = (ctypes.c_int * len(fields))(*[FIELD_IDS[f] for f in fields])
        _check(self.lib, self.lib.lulesh_comm_sbn(self.h, rank, len(fields), ids), "CommSBN")

    def comm_sync_posvel(self, rank):
        _check(self.lib, self.lib.lulesh_comm_sync_posvel(self.h, rank), "CommSyncPosVel")

    def comm_monoq(self, rank):
        _check(self.lib, self.lib.lulesh_comm_monoq(self.h, rank), "CommMonoQ")

    def comm_recv_offset(self, recv_rank, dc, dr, dp, xfer, do_recv, plane_only) -> int:
        return int(self.lib.lulesh_comm_recv_offset(self.h, recv_rank, dc, dr, dp, xfer,
                                                    int(do_recv), int(plane_only)))


class Server:
    """Continuous-batching server (lulesh_server_*): submit jobs, call step()
    repeatedly, poll() finished results."""

    def __init__(self, hbm_cap_bytes: int = 150 * 10**9, max_jobs: int = 256,
                 cycles_per_step: int = 8, prepare_threads: int = 4, device: int = -1):
        self.lib = load_library()
        cfg = ServerConfig(hbm_cap_bytes, max_jobs, cycles_per_step, prepare_threads, device)
        h = ctypes.c_void_p()
        _check(self.lib, self.lib.lulesh_server_create(ctypes.byref(cfg), ctypes.byref(h)),
               "lulesh_server_create")
        self.h = h

    def submit(self, job: JobSpec) -> int:
        jid = ctypes.c_longlong()
        c = job.c()
        _check(self.lib, self.lib.lulesh_server_submit(self.h, ctypes.byref(c), ctypes.byref(jid)),
               "lulesh_server_submit")
        return jid.value

    def step(self) -> tuple[int, int]:
        a, q = ctypes.c_int(), ctypes.c_int()
        _check(self.lib, self.lib.lulesh_server_step(self.h, ctypes.byref(a), ctypes.byref(q)),
               "lulesh_server_step")
        return a.value, q.value

    def poll(self, max_results: int = 1024) -> list[dict]:
        buf = (ServerResult * max_results)()
        n = ctypes.c_int()
        _check(self.lib, self.lib.lulesh_server_poll(self.h, buf, max_results, ctypes.byref(n)),
               "lulesh_server_poll")
        return [buf[i].as_dict() for i in range(n.value)]

    def clock(self) -> float:
        return float(self.lib.lulesh_server_clock())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.lulesh_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
