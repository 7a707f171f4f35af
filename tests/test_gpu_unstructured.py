"""Unstructured input (the reference's `-u file.lmesh`, lulesh.cu:855-1052):
the kernels read the mesh's own nodelist, corner lists, face links and
boundary sets.

Parity is anchored on the structured path: the -s 45 cube written as an
lmesh file runs bit for bit like `-s 45` (the deposit 3.948746e7 is the
-s 45 value), a node renumbering changes nothing but labels, and an
element renumbering changes only the order of the nodal force sums."""
import os

import numpy as np
import pytest

import lmesh

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MESHES = os.path.join(REPO, "oracle", "_ref", "meshes")

ELEM_FIELDS = ["e", "p", "q", "v", "ss", "delv", "arealg"]
NODE_FIELDS = ["x", "y", "z", "xd", "yd", "zd"]


@pytest.fixture(scope="module")
def box45(tmp_path_factory):
    p = tmp_path_factory.mktemp("lmesh") / "box45.lmesh"
    lmesh.write(p, lmesh.box(45))
    return str(p)


def _fields(s, E, N):
    out = {f: s.field(f)[:E] for f in ELEM_FIELDS}
    out.update({f: s.field(f)[:N] for f in NODE_FIELDS})
    return out


def test_mesh_tables_match_the_structured_build(lulesh, box45):
    """The reader's tables equal the -s host build's (BuildMesh, the face
    links, SetupBoundaryConditions and the corner lists)."""
    with lulesh.LuleshSet(nx=45, its=1, flags=lulesh.FLAG_HOST_SETUP) as s, \
            lulesh.LuleshSet.from_mesh(box45, its=1) as u:
        for name in ["nodelist", "lxim", "lxip", "letam", "letap", "lzetam", "lzetap",
                     "elemBC", "nodeElemCount", "nodeElemStart", "nodeElemCornerList",
                     "regNumList", "regElemlist", "regReps", "regSorted", "regCSR"]:
            a, b = s.field(name), u.field(name)
            n = min(len(a), len(b))
            assert (a[:n] == b[:n]).all(), name
        for name in ["x", "y", "z", "volo", "elemMass", "nodalMass", "e"]:
            assert (s.field(name) == u.field(name)).all(), name
        assert s.state() == u.state()


@pytest.mark.parametrize("its", [60, -1])
def test_cube_runs_like_structured(lulesh, box45, its):
    with lulesh.LuleshSet(nx=45, its=its) as s, lulesh.LuleshSet.from_mesh(box45, its=its) as u:
        assert s.run() == lulesh.OK
        assert u.run() == lulesh.OK
        assert s.state() == u.state()
        assert s.origin_energy() == u.origin_energy()
        E, N = 45 ** 3, 46 ** 3
        a, b = _fields(s, E, N), _fields(u, E, N)
        for f in a:
            assert (a[f] == b[f]).all(), f


def test_run_graph_matches_host_loop(lulesh, box45):
    with lulesh.LuleshSet.from_mesh(box45, its=90) as a, \
            lulesh.LuleshSet.from_mesh(box45, its=90) as b:
        assert a.run_graph() == lulesh.OK
        assert b.run() == lulesh.OK
        assert a.state() == b.state()
        assert (a.field("e") == b.field("e")).all()


def _run_pair(lulesh, tmp_path, nx, its, node_perm, elem_perm):
    m = lmesh.box(nx)
    p0, p1 = tmp_path / "id.lmesh", tmp_path / "perm.lmesh"
    lmesh.write(p0, m)
    lmesh.write(p1, lmesh.renumber(m, node_perm, elem_perm))
    with lulesh.LuleshSet.from_mesh(str(p0), its=its) as a, \
            lulesh.LuleshSet.from_mesh(str(p1), its=its) as b:
        assert a.run() == lulesh.OK and b.run() == lulesh.OK
        E, N = m.num_elem, m.num_node
        return a.state(), b.state(), _fields(a, E, N), _fields(b, E, N), \
            a.origin_energy(), b.origin_energy()


def test_node_renumbering_is_exact(lulesh, tmp_path):
    nx = 20
    npm = np.random.default_rng(1).permutation((nx + 1) ** 3)
    sa, sb, fa, fb, ea, eb = _run_pair(lulesh, tmp_path, nx, 150, npm, None)
    assert sa == sb and ea == eb
    for f in ELEM_FIELDS:
        assert (fa[f] == fb[f]).all(), f
    for f in NODE_FIELDS:
        assert (fb[f][npm] == fa[f]).all(), f


def test_element_renumbering(lulesh, tmp_path):
    """Element labels change the order of each node's corner sum
    (AddNodeForcesFromElems, lulesh.cu:1715-1751) and of the nodal mass
    accumulation, so values agree to rounding: 1e-9 relative on energy."""
    nx = 20
    rng = np.random.default_rng(2)
    npm = rng.permutation((nx + 1) ** 3)
    epm = rng.permutation(nx ** 3)
    sa, sb, fa, fb, ea, eb = _run_pair(lulesh, tmp_path, nx, 150, npm, epm)
    assert sa["cycle"] == sb["cycle"]
    assert abs(ea - eb) <= 1e-9 * abs(ea)
    e_a, e_b = fa["e"], fb["e"][epm]
    assert np.abs(e_a - e_b).max() <= 1e-9 * np.abs(e_a).max()
    x_a, x_b = fa["x"], fb["x"][npm]
    assert np.abs(x_a - x_b).max() <= 1e-12


def duplicated(m, elems):
    """The mesh with copies of the listed elements appended: the copies share
    their originals' nodes and face links, so those nodes gain corners (a
    node of a duplicated interior element has up to 16).  Physically it is
    a denser material there; arithmetically it is a valid mesh, and it takes
    the nodal kernel off its at-most-8-corners path."""
    elems = np.asarray(elems, dtype=np.int64)
    return lmesh.LMesh(m.xyz.copy(), np.concatenate([m.nodelist, m.nodelist[elems]]),
                       np.concatenate([m.links, m.links[elems]]), m.symm, m.free)


def _compare(s, o, fields, E, N, rtol, atol=1e-14):
    """Max difference relative to the field's largest magnitude; a field
    that is still ~0 everywhere (delv after one cycle: the last bit of a
    relative volume of 1) is held to `atol` instead."""
    bad = []
    for f in fields:
        n = E if f in ELEM_FIELDS else N
        g, r = s.field(f)[:n], o.field(f)[:n]
        diff = float(np.max(np.abs(g - r)))
        scale = float(max(np.max(np.abs(r)), np.max(np.abs(g))))
        if diff > rtol * scale and diff > atol:
            bad.append(f"{f}: {diff:.3e} of {scale:.3e}")
    return bad


@pytest.mark.parametrize("mesh", ["warped", "sedov15oct", "dup_one", "dup_all"])
def test_matches_oracle(lulesh, oracle_mod, tmp_path, mesh):
    """Against the CPU oracle's reading of the same file: a curvilinear,
    renumbered -s 10 box (generated here), the reference's own octant mesh
    when its copy is present, and boxes with duplicated elements whose nodes
    have more than 8 corners (one duplicate: the staged corner-run path; all
    duplicated: runs too long to stage, read from the list).  One cycle to
    rounding level, then the full run to t = 0.01: same cycle count, origin
    energy within 1e-9."""
    if mesh == "dup_one":
        path = str(tmp_path / "dup_one.lmesh")
        lmesh.write(path, duplicated(lmesh.box(8), [200]))
    elif mesh == "dup_all":
        m = lmesh.box(6)
        path = str(tmp_path / "dup_all.lmesh")
        lmesh.write(path, duplicated(m, np.arange(m.num_elem)))
    elif mesh == "warped":
        m = lmesh.box(10)
        rng = np.random.default_rng(3)
        path = str(tmp_path / "warped.lmesh")
        lmesh.write(path, lmesh.renumber(lmesh.warp(m), rng.permutation(m.num_node),
                                         rng.permutation(m.num_elem)))
    else:
        path = os.path.join(MESHES, "sedov15oct.lmesh")
        if not os.path.exists(path):
            pytest.skip("reference mesh copy absent")
    m = lmesh.read(path)
    E, N = m.num_elem, m.num_node
    o = oracle_mod.Oracle.from_lmesh(path)
    try:
        with lulesh.LuleshSet.from_mesh(path, its=1) as s:
            assert s.run() == lulesh.OK
            assert o.step() == 0
            bad = _compare(s, o, ELEM_FIELDS + NODE_FIELDS, E, N, 1e-12)
            assert not bad, bad
        o.close()
        o = oracle_mod.Oracle.from_lmesh(path)
        ost, ocyc = o.run()
        with lulesh.LuleshSet.from_mesh(path) as s:
            assert s.run() == ost == lulesh.OK
            st = s.state()
            assert st["cycle"] == ocyc
            e_g, e_o = s.origin_energy(), o.origin_energy()
            assert abs(e_g - e_o) <= 1e-9 * abs(e_o), (e_g, e_o)
            bad = _compare(s, o, ["e", "p", "v", "x", "y", "z", "xd"], E, N, 1e-8)
            assert not bad, bad
    finally:
        o.close()


def test_reference_octant_mesh(lulesh):
    """The reference's own sedov15oct.lmesh (when its copy is present) runs
    to t = 0.01 with a finite, positive origin energy."""
    path = os.path.join(MESHES, "sedov15oct.lmesh")
    if not os.path.exists(path):
        pytest.skip("reference mesh copy absent")
    m = lmesh.read(path)
    with lulesh.LuleshSet.from_mesh(path) as s:
        assert s.run() == lulesh.OK
        st = s.state()
        assert st["done"] and st["time"] >= 1e-2 * (1 - 1e-12)
        e0 = s.origin_energy()
        assert np.isfinite(e0) and e0 > 0
        e = s.field("e")[:m.num_elem]
        assert np.isfinite(e).all()


def test_bad_inputs(lulesh, tmp_path):
    with pytest.raises(lulesh.LuleshError) as ei:
        lulesh.LuleshSet.from_mesh(str(tmp_path / "absent.lmesh"))
    assert ei.value.status == lulesh.FILE_ERROR

    m = lmesh.box(3)
    good = tmp_path / "g.lmesh"
    lmesh.write(good, m)
    text = good.read_text()
    trunc = tmp_path / "t.lmesh"
    trunc.write_text(text[: len(text) // 2])
    bad_node = tmp_path / "n.lmesh"
    m2 = lmesh.box(3)
    m2.nodelist[5, 3] = m2.num_node + 10
    lmesh.write(bad_node, m2)
    bad_link = tmp_path / "l.lmesh"
    m3 = lmesh.box(3)
    m3.links[2, 1] = -4
    lmesh.write(bad_link, m3)
    for p in (trunc, bad_node, bad_link):
        with pytest.raises(lulesh.LuleshError) as ei:
            lulesh.LuleshSet.from_mesh(str(p))
        assert ei.value.status == lulesh.FILE_ERROR, p

    for flags in (lulesh.FLAG_COMM_STAGED, lulesh.FLAG_MIXED):
        with pytest.raises(lulesh.LuleshError) as ei:
            lulesh.LuleshSet.from_mesh(str(good), flags=flags)
        assert ei.value.status == lulesh.INVALID_ARG
    with lulesh.LuleshSet.from_mesh(str(good), its=5) as s:
        with pytest.raises(lulesh.LuleshError):
            s.symmetry()
