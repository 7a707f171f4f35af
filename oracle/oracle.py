"""ctypes binding of oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle is the checker: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use it to compute the reference answer on the CPU.  It
restates the reference CUDA single-domain step (LULESH/cuda/src/lulesh.cu)
in plain C; see lulesh_oracle.c for the line-by-line citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_OMP = os.path.join(HERE, "_ref", "lulesh_omp")
REF_CUDA = os.path.join(HERE, "_ref", "lulesh_ref_cuda")

INT_FIELDS = {
    "nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
    "nodeElemCount", "nodeElemStart", "nodeElemCornerList", "symmX", "symmY",
    "symmZ", "matElemlist", "regElemSize", "regCSR", "regReps", "regNumList",
    "regElemlist", "regSorted",
}

_lib = None

MIRROR_FIELDS = ("x", "y", "z", "xd", "yd", "zd", "fx_elem", "fy_elem", "fz_elem",
                 "delv_xi", "delv_eta", "delv_zeta", "volo")


class OracleMirror(ctypes.Structure):
    """A neighbour's arrays for decomposed stepping (lulesh_oracle.h)."""
    _fields_ = [(f, ctypes.POINTER(ctypes.c_double)) for f in MIRROR_FIELDS]


def build() -> None:
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                   stdout=subprocess.DEVNULL)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.oracle_create.restype = vp
    lib.oracle_create.argtypes = [ip] * 9
    lib.oracle_create_lmesh.restype = vp
    lib.oracle_create_lmesh.argtypes = [ctypes.c_char_p, ip, ip, ip]
    lib.oracle_destroy.argtypes = [vp]
    lib.oracle_step.restype = ip
    lib.oracle_step.argtypes = [vp]
    lib.oracle_run.restype = ip
    lib.oracle_run.argtypes = [vp, ip, ctypes.POINTER(ip)]
    lib.oracle_real_field.restype = ctypes.POINTER(dp)
    lib.oracle_real_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ip)]
    lib.oracle_int_field.restype = ctypes.POINTER(ip)
    lib.oracle_int_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ip)]
    lib.oracle_scalar.restype = dp
    lib.oracle_scalar.argtypes = [vp, ctypes.c_char_p]
    lib.oracle_set_deltatime.argtypes = [vp, dp]
    lib.oracle_origin_energy.restype = dp
    lib.oracle_origin_energy.argtypes = [vp]
    lib.oracle_symmetry.argtypes = [vp] + [ctypes.POINTER(dp)] * 3
    lib.oracle_set_mirror.argtypes = [vp, ip, ctypes.POINTER(OracleMirror)]
    lib.oracle_phase.restype = ip
    lib.oracle_phase.argtypes = [vp, ip]
    lib.oracle_nodal_mass_decomposed.argtypes = [vp]
    lib.oracle_set_dt_minima.argtypes = [vp, dp, dp]
    _lib = lib
    return lib


class Oracle:
    """One reference domain on the CPU."""

    def __init__(self, nx: int, numReg: int = 11, balance: int = 1, cost: int = 1,
                 tp: int = 1, col: int = 0, row: int = 0, plane: int = 0, rank: int = 0):
        self.lib = load()
        self.h = self.lib.oracle_create(nx, numReg, balance, cost, tp, col, row, plane, rank)
        if not self.h:
            raise ValueError("oracle_create rejected the arguments")
        self.nx = nx

    @classmethod
    def from_lmesh(cls, path: str, numReg: int = 11, balance: int = 1,
                   cost: int = 1) -> "Oracle":
        """The -u branch of NewDomain (lulesh.cu:855-1052) on an lmesh file."""
        o = cls.__new__(cls)
        o.lib = load()
        o.h = o.lib.oracle_create_lmesh(str(path).encode(), numReg, balance, cost)
        if not o.h:
            raise ValueError(f"oracle_create_lmesh could not read {path}")
        o.nx = 0
        return o

    def close(self) -> None:
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> int:
        return self.lib.oracle_step(self.h)

    def run(self, its: int = -1) -> tuple[int, int]:
        n = ctypes.c_int()
        st = self.lib.oracle_run(self.h, its, ctypes.byref(n))
        return st, n.value

    def field(self, name: str) -> np.ndarray:
        n = ctypes.c_int()
        if name in INT_FIELDS:
            p = self.lib.oracle_int_field(self.h, name.encode(), ctypes.byref(n))
            dt = np.int32
        else:
            p = self.lib.oracle_real_field(self.h, name.encode(), ctypes.byref(n))
            dt = np.float64
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,)).astype(dt, copy=True)

    def set_real_field(self, name: str, values: np.ndarray) -> None:
        n = ctypes.c_int()
        p = self.lib.oracle_real_field(self.h, name.encode(), ctypes.byref(n))
        arr = np.ctypeslib.as_array(p, shape=(n.value,))
        arr[:] = values

    def view(self, name: str) -> np.ndarray:
        """The oracle's own array (no copy): writes go into the domain."""
        n = ctypes.c_int()
        p = self.lib.oracle_real_field(self.h, name.encode(), ctypes.byref(n))
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(n.value,))

    # -- decomposed stepping (a subdomain whose neighbours are read through
    #    mirrors; lulesh_oracle.h)
    def set_mirror(self, direction: int, arrays: dict | None) -> None:
        """arrays: name -> float64 numpy array (kept alive by the caller)."""
        if arrays is None:
            self.lib.oracle_set_mirror(self.h, direction, None)
            return
        m = OracleMirror(*[arrays[f].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                           for f in MIRROR_FIELDS])
        self.lib.oracle_set_mirror(self.h, direction, ctypes.byref(m))

    def phase(self, ph: int) -> int:
        return self.lib.oracle_phase(self.h, ph)

    def nodal_mass_decomposed(self) -> None:
        self.lib.oracle_nodal_mass_decomposed(self.h)

    def set_dt_minima(self, dtcourant: float, dthydro: float) -> None:
        self.lib.oracle_set_dt_minima(self.h, dtcourant, dthydro)

    def set_deltatime(self, dt: float) -> None:
        self.lib.oracle_set_deltatime(self.h, dt)

    def scalar(self, name: str) -> float:
        return self.lib.oracle_scalar(self.h, name.encode())

    def origin_energy(self) -> float:
        return self.lib.oracle_origin_energy(self.h)

    def symmetry(self) -> tuple[float, float, float]:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.lib.oracle_symmetry(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value


def parse_report(text: str) -> dict:
    """Parse the reference's final report (VerifyAndWriteFinalOutput)."""
    out = {}
    for line in text.splitlines():
        t = line.split()
        if "Final Origin Energy" in line:
            out["energy"] = float(t[4])
        elif line.strip().startswith("MaxAbsDiff"):
            out["max_abs"] = float(t[2])
        elif line.strip().startswith("TotalAbsDiff"):
            out["total_abs"] = float(t[2])
        elif line.strip().startswith("MaxRelDiff"):
            out["max_rel"] = float(t[2])
        elif line.strip().startswith("Iteration count"):
            out["cycles"] = int(t[3])
        elif line.startswith("Elapsed time"):
            out["elapsed"] = float(t[3])
        elif line.startswith("Grind time"):
            out["grind"] = float(t[4])
    return out
