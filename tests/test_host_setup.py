"""Host-side setup logic of the product, checked on the CPU (no GPU).

The product builds every Domain array on the host (csrc/host_setup.cpp,
restating NewDomain, lulesh.cu:750-1221) and uploads it.  liblulesh_host.so
exposes that code without CUDA; here it is compared with the oracle's own
setup, bit for bit, including ghost indexing of decomposed ranks and the
glibc-rand region sets.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import PKG

LIB = os.path.join(PKG, "liblulesh_host.so")


@pytest.fixture(scope="module")
def host():
    if not os.path.exists(LIB):
        import subprocess

        subprocess.run(["make", "-C", PKG, "liblulesh_host.so"], check=True)
    lib = ctypes.CDLL(LIB)
    lib.lulesh_host_rand.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.lulesh_host_domain_field.restype = ctypes.c_long
    lib.lulesh_host_domain_field.argtypes = [ctypes.c_int] * 10 + [ctypes.c_char_p,
                                                                  ctypes.c_void_p, ctypes.c_long]
    return lib


def _field(host, name, nx, tp=1, col=0, row=0, plane=0, rank=0, nr=11, b=1, c=1, gm=0):
    n = host.lulesh_host_domain_field(nx, tp, col, row, plane, rank, nr, b, c, gm,
                                      name.encode(), None, 0)
    assert n >= 0, name
    from oracle import INT_FIELDS

    dt = np.int32 if name in INT_FIELDS else np.float64
    out = np.empty(n, dtype=dt)
    host.lulesh_host_domain_field(nx, tp, col, row, plane, rank, nr, b, c, gm, name.encode(),
                                  out.ctypes.data_as(ctypes.c_void_p), n)
    return out


@pytest.mark.parametrize("seed", [0, 1, 7, 12345])
def test_glibc_rand_restatement(host, seed):
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    want = [libc.rand() for _ in range(2000)]
    got = (ctypes.c_int * 2000)()
    host.lulesh_host_rand(seed, 2000, got)
    assert list(got) == want


FIELDS = ["nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
          "nodeElemCount", "nodeElemStart", "nodeElemCornerList", "symmX", "symmY", "symmZ",
          "matElemlist", "regElemSize", "regCSR", "regReps", "regNumList", "regElemlist",
          "regSorted", "x", "y", "z", "volo", "elemMass", "nodalMass", "e"]


@pytest.mark.parametrize("nx,tp,loc,rank,nr,b,c", [
    (6, 1, (0, 0, 0), 0, 11, 1, 1),
    (5, 1, (0, 0, 0), 0, 20, 4, 4),
    (4, 2, (1, 0, 1), 5, 11, 1, 1),
    (3, 3, (1, 1, 1), 13, 7, 2, 3),
    (4, 3, (2, 0, 1), 11, 11, 1, 1),
    (1, 1, (0, 0, 0), 0, 1, 1, 1),
])
def test_setup_matches_oracle(host, oracle_mod, nx, tp, loc, rank, nr, b, c):
    col, row, plane = loc
    o = oracle_mod.Oracle(nx, numReg=nr, balance=b, cost=c, tp=tp, col=col, row=row,
                          plane=plane, rank=rank)
    for f in FIELDS:
        got = _field(host, f, nx, tp, col, row, plane, rank, nr, b, c)
        want = o.field(f)
        assert np.array_equal(got, want), f
    dt = np.empty(1)
    host.lulesh_host_domain_field(nx, tp, col, row, plane, rank, nr, b, c, 0, b"deltatime",
                                  dt.ctypes.data_as(ctypes.c_void_p), 1)
    assert dt[0] == o.scalar("initial_deltatime")


def test_global_nodal_mass_equals_undecomposed(host):
    """With global-order summation a subdomain's nodal masses equal the
    matching nodes of the undecomposed mesh bit for bit."""
    nx, tp = 4, 2
    full = _field(host, "nodalMass", nx * tp).reshape(nx * tp + 1, nx * tp + 1, nx * tp + 1)
    for r in range(tp ** 3):
        c, w, p = r % tp, (r // tp) % tp, r // (tp * tp)
        sub = _field(host, "nodalMass", nx, tp, c, w, p, r, gm=1).reshape(nx + 1, nx + 1, nx + 1)
        ref = full[p * nx:(p + 1) * nx + 1, w * nx:(w + 1) * nx + 1, c * nx:(c + 1) * nx + 1]
        assert np.array_equal(sub, ref), r
