"""The lmesh writer/reader (the reference's -u input format, lulesh.cu:855-1052):
the cube it writes is the -s mesh of the oracle's BuildMesh restatement, and
files round-trip exactly."""
import os

import numpy as np
import pytest

import lmesh


@pytest.mark.parametrize("nx", [1, 3, 7])
def test_box_is_the_structured_mesh(oracle_mod, nx):
    m = lmesh.box(nx)
    o = oracle_mod.Oracle(nx)
    try:
        E, N = m.num_elem, m.num_node
        Ep = int(o.scalar("padded_numElem"))
        nl = o.field("nodelist").reshape(8, Ep)[:, :E].T
        assert (m.nodelist == nl).all()
        for k, name in enumerate(["lxim", "lxip", "letam", "letap", "lzetam", "lzetap"]):
            assert (m.links[:, k] == o.field(name)[:E]).all(), name
        for k, c in enumerate("xyz"):
            assert (m.xyz[:, k] == o.field(c)[:N]).all()
        for k, name in enumerate(["symmX", "symmY", "symmZ"]):
            n = int(o.scalar("numSymm" + "XYZ"[k]))
            assert sorted(o.field(name)[:n]) == list(m.symm[k])
    finally:
        o.close()


def test_round_trip(tmp_path):
    m = lmesh.box(4)
    p = tmp_path / "b.lmesh"
    lmesh.write(p, m)
    r = lmesh.read(p)
    assert (r.xyz == m.xyz).all()
    assert (r.nodelist == m.nodelist).all() and (r.links == m.links).all()
    assert all((a == b).all() for a, b in zip(r.symm, m.symm))
    assert (r.free == m.free).all()


def test_renumber_keeps_geometry():
    m = lmesh.box(3)
    rng = np.random.default_rng(7)
    npm = rng.permutation(m.num_node)
    epm = rng.permutation(m.num_elem)
    r = lmesh.renumber(m, npm, epm)
    # element epm[z] has the coordinates of element z, corner by corner
    assert (r.xyz[r.nodelist[epm]] == m.xyz[m.nodelist]).all()
    # face neighbours map the same way
    assert (r.links[epm] == epm[m.links]).all()
    assert sorted(r.free) == sorted(npm[m.free])


def test_oracle_reads_the_box_as_its_structured_mesh(oracle_mod, tmp_path):
    """The oracle's lmesh reader (the -u branch of NewDomain) builds the same
    tables from lmesh.box(nx) as its -s builder."""
    p = tmp_path / "b6.lmesh"
    lmesh.write(p, lmesh.box(6))
    s, u = oracle_mod.Oracle(6), oracle_mod.Oracle.from_lmesh(str(p))
    try:
        for f in ["nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
                  "nodeElemStart", "nodeElemCornerList", "regElemlist", "regReps"]:
            a, b = s.field(f), u.field(f)
            n = min(len(a), len(b))
            assert (a[:n] == b[:n]).all(), f
        for f in ["x", "y", "z", "volo", "elemMass", "nodalMass"]:
            assert (s.field(f) == u.field(f)).all(), f
        # the deposit: 3.948746e7 at the octant corner (element 0 here)
        assert u.field("e")[0] == 3.948746e7 and (u.field("e")[1:] == 0).all()
    finally:
        s.close()
        u.close()


def test_oracle_rejects_malformed_files(oracle_mod, tmp_path):
    m = lmesh.box(2)
    m.nodelist[1, 2] = 10 ** 6
    p = tmp_path / "bad.lmesh"
    lmesh.write(p, m)
    with pytest.raises(ValueError):
        oracle_mod.Oracle.from_lmesh(str(p))
    with pytest.raises(ValueError):
        oracle_mod.Oracle.from_lmesh(str(tmp_path / "absent.lmesh"))


LMESH_FIELDS = ["nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap", "elemBC",
                "nodeElemCount", "nodeElemStart", "nodeElemCornerList", "symmX", "symmY",
                "symmZ", "matElemlist", "regElemSize", "regCSR", "regReps", "regNumList",
                "regElemlist", "regSorted", "x", "y", "z", "volo", "elemMass", "nodalMass",
                "e"]


def _host_lmesh(path, name):
    import ctypes

    from conftest import PKG
    from oracle import INT_FIELDS

    lib = ctypes.CDLL(os.path.join(PKG, "liblulesh_host.so"))
    f = lib.lulesh_host_lmesh_field
    f.restype = ctypes.c_long
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                  ctypes.c_void_p, ctypes.c_long]
    n = f(str(path).encode(), 11, 1, 1, name.encode(), None, 0)
    assert n >= 0, (name, n)
    ints = INT_FIELDS | {"octant", "nodeCornerEll", "nodeBC"}
    dt = np.int32 if name in ints else np.float64
    out = np.empty(n, dtype=dt)
    f(str(path).encode(), 11, 1, 1, name.encode(), out.ctypes.data_as(ctypes.c_void_p), n)
    return out


def _meshes(tmp_path):
    m = lmesh.box(9)
    rng = np.random.default_rng(5)
    p = tmp_path / "warped.lmesh"
    lmesh.write(p, lmesh.renumber(lmesh.warp(m), rng.permutation(m.num_node),
                                  rng.permutation(m.num_elem)))
    out = [p]
    ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref", "meshes", "sedov15oct.lmesh")
    if os.path.exists(ref):
        out.append(ref)
    return out


def test_product_reader_matches_the_oracle(oracle_mod, tmp_path):
    """The product's lmesh reader (lulesh_create_from_mesh, C++) and the
    oracle's (C) build the same domain bit for bit: connectivity, boundary
    masks with the *_FREE free surface, corner lists, regions, geometry,
    masses, the octant-corner deposit and the initial dt."""
    for path in _meshes(tmp_path):
        o = oracle_mod.Oracle.from_lmesh(str(path))
        try:
            for f in LMESH_FIELDS:
                a, b = _host_lmesh(path, f), o.field(f)
                assert a.shape == b.shape and np.array_equal(a, b), (path, f)
            assert _host_lmesh(path, "deltatime")[0] == o.scalar("deltatime")
            oct_ = int(_host_lmesh(path, "octant")[0])
            assert o.field("e")[oct_] == 3.948746e7
        finally:
            o.close()


def test_product_reader_rejects_malformed_files(tmp_path):
    import ctypes

    from conftest import PKG

    lib = ctypes.CDLL(os.path.join(PKG, "liblulesh_host.so"))
    f = lib.lulesh_host_lmesh_field
    f.restype = ctypes.c_long
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                  ctypes.c_void_p, ctypes.c_long]
    m = lmesh.box(2)
    m.links[3, 4] = m.num_elem
    p = tmp_path / "bad.lmesh"
    lmesh.write(p, m)
    assert f(str(p).encode(), 11, 1, 1, b"x", None, 0) == -2
    assert f(str(tmp_path / "none.lmesh").encode(), 11, 1, 1, b"x", None, 0) == -2


def test_slot_major_runs_only_up_to_8_corners(tmp_path):
    """The reader lays the corner runs out slot-major (slot j of node i at
    j * N + i, -1 past the run) when no node has more than 8 corners, and
    leaves them out otherwise."""
    p = tmp_path / "b4.lmesh"
    m = lmesh.box(4)
    lmesh.write(p, m)
    ell = _host_lmesh(p, "nodeCornerEll").reshape(8, m.num_node)
    start, count = _host_lmesh(p, "nodeElemStart"), _host_lmesh(p, "nodeElemCount")
    runs = _host_lmesh(p, "nodeElemCornerList")
    for n in range(m.num_node):
        want = list(runs[start[n]:start[n] + count[n]]) + [-1] * (8 - count[n])
        assert list(ell[:, n]) == want
    q = tmp_path / "dup.lmesh"
    lmesh.write(q, lmesh.LMesh(m.xyz, np.concatenate([m.nodelist, m.nodelist[:1]]),
                               np.concatenate([m.links, m.links[:1]]), m.symm, m.free))
    assert _host_lmesh(q, "nodeCornerEll").size == 0
