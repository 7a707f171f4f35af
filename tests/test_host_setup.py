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


def _face_links(z, nx, tp, col, row, plane, ghost):
    """The rule the EOS kernel evaluates in place of elemBC/lxim..lzetap
    (kernels.cu elem_face_links)."""
    ix, iy, iz = z % nx, (z // nx) % nx, z // (nx * nx)
    bc = 0
    l = [z - 1, z + 1, z - nx, z + nx, z - nx * nx, z + nx * nx]  # xm xp em ep zm zp
    last = tp - 1
    if iz == 0:
        if plane == 0:
            bc |= 0x01000
        else:
            bc |= 0x04000; l[4] = ghost[0] + iy * nx + ix
    if iz == nx - 1:
        if plane == last:
            bc |= 0x10000
        else:
            bc |= 0x20000; l[5] = ghost[1] + iy * nx + ix
    if iy == 0:
        if row == 0:
            bc |= 0x00040
        else:
            bc |= 0x00100; l[2] = ghost[2] + iz * nx + ix
    if iy == nx - 1:
        if row == last:
            bc |= 0x00400
        else:
            bc |= 0x00800; l[3] = ghost[3] + iz * nx + ix
    if ix == 0:
        if col == 0:
            bc |= 0x00001
        else:
            bc |= 0x00004; l[0] = ghost[4] + iz * nx + iy
    if ix == nx - 1:
        if col == last:
            bc |= 0x00010
        else:
            bc |= 0x00020; l[1] = ghost[5] + iz * nx + iy
    return bc, l


@pytest.mark.parametrize("nx,tp,loc", [(5, 1, (0, 0, 0)), (4, 2, (1, 0, 1)), (3, 3, (1, 1, 1)),
                                       (4, 3, (0, 2, 1)), (1, 2, (1, 1, 1))])
def test_face_link_rule_matches_connectivity(oracle_mod, nx, tp, loc):
    """Where the limiter reads a neighbour (masks other than SYMM/FREE), the
    arithmetic rule gives exactly the SetupConnectivityBC index."""
    col, row, plane = loc
    o = oracle_mod.Oracle(nx, tp=tp, col=col, row=row, plane=plane)
    bcs = o.field("elemBC")
    names = ["lxim", "lxip", "letam", "letap", "lzetam", "lzetap"]
    arrs = [o.field(n) for n in names]
    E = nx ** 3
    present = [plane > 0, plane < tp - 1, row > 0, row < tp - 1, col > 0, col < tp - 1]
    ghost, p = [], E
    for f in range(6):
        ghost.append(p if present[f] else -1)
        p += nx * nx if present[f] else 0
    # (mask of the face, symm bit, free bit) per neighbour slot
    faces = [(0x7, 0x1, 0x2), (0x38, 0x8, 0x10), (0x1C0, 0x40, 0x80), (0xE00, 0x200, 0x400),
             (0x7000, 0x1000, 0x2000), (0x38000, 0x8000, 0x10000)]
    for z in range(E):
        bc, l = _face_links(z, nx, tp, col, row, plane, ghost)
        assert bc == bcs[z], z
        for s, (mask, symm, free) in enumerate(faces):
            if (bc & mask) not in (symm, free):
                assert l[s] == arrs[s][z], (z, names[s])


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


@pytest.mark.parametrize("nx", [1, 2, 3, 7, 12])
def test_closed_form_corner_csr(host, nx):
    """The closed forms the device setup kernel uses for nodeElemStart,
    nodeElemCount and nodeElemCornerList (setup.cu) reproduce the host
    builder's prefix-sum CSR (lulesh.cu:1054-1106)."""
    en, Ep = nx + 1, ((nx ** 3 + 31) // 32) * 32
    start = _field(host, "nodeElemStart", nx)
    count = _field(host, "nodeElemCount", nx)
    corners = _field(host, "nodeElemCornerList", nx)

    def adj(p):
        return (p > 0) + (p < nx)

    def below(k):
        return 0 if k == 0 else 2 * k - 1
    A = 2 * nx
    got = np.full_like(corners, -1)
    for n in range(en ** 3):
        px, t = n % en, n // en
        py, pz = t % en, t // en
        s = below(pz) * A * A + adj(pz) * below(py) * A + adj(pz) * adj(py) * below(px)
        assert s == start[n] and adj(px) * adj(py) * adj(pz) == count[n]
        r = 0
        for j in range(8):
            ex, ey, ez = px - ((0x66 >> j) & 1), py - ((0xCC >> j) & 1), pz - ((0xF0 >> j) & 1)
            if 0 <= ex < nx and 0 <= ey < nx and 0 <= ez < nx:
                got[s + r] = Ep * j + (ez * nx + ey) * nx + ex
                r += 1
    assert np.array_equal(got, corners)


def _light(host, name, nx, nr, b, c, dtype=np.int32):
    n = host.lulesh_host_light_field(nx, nr, b, c, name.encode(), None, 0)
    assert n >= 0, name
    out = np.empty(n, dtype=dtype)
    host.lulesh_host_light_field(nx, nr, b, c, name.encode(),
                                 out.ctypes.data_as(ctypes.c_void_p), n)
    return out


@pytest.mark.parametrize("nx,nr,b,c", [(1, 11, 1, 1), (2, 5, 2, 1), (7, 11, 1, 1),
                                       (13, 1, 1, 1), (16, 20, 4, 4), (30, 11, 1, 1),
                                       (45, 11, 1, 1), (48, 17, 2, 2)])
def test_region_runs_expand_to_the_host_builders_arrays(host, nx, nr, b, c):
    """Single domains built with their geometry on the device keep the
    region sets as runs, and the device writes regNumList, regElemlist and
    the EOS order from them, element by element (setup.cu k_region_sets).
    The same per-element function, run here on the host over every element,
    gives the full host builder's arrays (pinned to the oracle above), and
    the per-region and per-class tables built from the runs are equal too."""
    host.lulesh_host_light_field.restype = ctypes.c_long
    host.lulesh_host_light_field.argtypes = [ctypes.c_int] * 4 + [ctypes.c_char_p,
                                                                 ctypes.c_void_p, ctypes.c_long]
    E = nx ** 3
    for f in ("regNumList", "regElemlist", "eosOrder", "regElemSize", "regCSR", "regReps",
              "regSorted", "eosClassEnd", "eosClassRep"):
        got = _light(host, f, nx, nr, b, c)
        n = host.lulesh_host_domain_field(nx, 1, 0, 0, 0, 0, nr, b, c, 0, f.encode(), None, 0)
        want = np.empty(n, dtype=np.int32)
        host.lulesh_host_domain_field(nx, 1, 0, 0, 0, 0, nr, b, c, 0, f.encode(),
                                      want.ctypes.data_as(ctypes.c_void_p), n)
        assert got.size > 0 and np.array_equal(got, want), f
    # every element written once in each list (the expansion starts from -1)
    for f in ("regElemlist", "eosOrder"):
        assert np.array_equal(np.sort(_light(host, f, nx, nr, b, c)), np.arange(E)), f
    # about one run per 38 elements is what travels to the device
    nruns = _light(host, "nruns", nx, nr, b, c, dtype=np.int64)[0]
    assert 1 <= nruns <= E
    if nr > 1 and E >= 20000:
        assert nruns < E / 20


def test_region_runs_are_checked_before_they_reach_the_device(host):
    """setup_regions_on_device refuses a run table whose expansion would
    write outside the three per-element arrays (region_runs_valid); the
    tables the light builder draws pass, tampered ones do not."""
    host.lulesh_host_light_field.restype = ctypes.c_long
    host.lulesh_host_light_field.argtypes = [ctypes.c_int] * 4 + [ctypes.c_char_p,
                                                                 ctypes.c_void_p, ctypes.c_long]
    host.lulesh_host_region_runs_valid.restype = ctypes.c_int
    host.lulesh_host_region_runs_valid.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]

    def valid(t, E):
        t = np.ascontiguousarray(t, dtype=np.int32)
        return host.lulesh_host_region_runs_valid(t.ctypes.data_as(ctypes.c_void_p),
                                                  t.shape[0], E) == 1

    for nx, nr in [(1, 11), (2, 1), (9, 5), (20, 11), (33, 20)]:
        t = _light(host, "runs", nx, nr, 1, 1).reshape(-1, 4)
        E = nx ** 3
        assert valid(t, E), (nx, nr)
        if t.shape[0] < 2:
            continue
        bad = t.copy(); bad[0, 0] = 1                      # does not start at element 0
        assert not valid(bad, E)
        bad = t.copy(); bad[1, 0] = bad[0, 0]              # empty run
        assert not valid(bad, E)
        bad = t.copy(); bad[-1, 0] = E                     # a run past the last element
        assert not valid(bad, E)
        bad = t.copy(); bad[-1, 2] = E                     # regElemlist write past the end
        assert not valid(bad, E)
        bad = t.copy(); bad[0, 3] = -1                     # EOS-order write before the start
        assert not valid(bad, E)
        assert not valid(t, t.shape[0] - 1)                # more runs than elements
    assert not valid(np.zeros((0, 4)), 8)                  # no runs at all
