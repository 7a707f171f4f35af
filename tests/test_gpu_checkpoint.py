"""Checkpoint / restore of a set's whole state (lulesh_checkpoint_*)."""
import pytest

pytestmark = pytest.mark.gpu


def test_restore_continues_bit_for_bit(lulesh):
    with lulesh.LuleshSet(nx=24, its=-1) as a:
        a.step(20)
        ck = a.checkpoint()
        a.step(30)
        a.sync()
        ref = (a.origin_energy(), a.state()["cycle"], a.field("e"))
    with lulesh.LuleshSet(nx=24, its=-1) as b:
        b.step(3)  # a different state first: the load replaces all of it
        b.restore(ck)
        assert b.state()["cycle"] == 20
        b.step(30)
        b.sync()
        assert (b.origin_energy(), b.state()["cycle"]) == ref[:2]
        assert (b.field("e") == ref[2]).all()


def test_batch_and_subdomain_checkpoints(lulesh):
    jobs = [lulesh.JobSpec(10, 7, 2, 2, 60), lulesh.JobSpec(14, 11, 1, 1, 60)]
    with lulesh.LuleshSet.batch(jobs) as a:
        a.step(10)
        ck = a.checkpoint()
        a.run()
        ref = [a.origin_energy(i) for i in range(2)]
    with lulesh.LuleshSet.batch(jobs) as b:
        b.restore(ck)
        b.run()
        assert [b.origin_energy(i) for i in range(2)] == ref
    with lulesh.LuleshSet(nx=6, tp=2, its=40) as a:
        a.step(15)
        ck = a.checkpoint()
        a.run()
        e = a.origin_energy()
    with lulesh.LuleshSet(nx=6, tp=2, its=40) as b:
        b.restore(ck)
        b.run()
        assert b.origin_energy() == e


def test_checkpoint_of_another_set_is_refused(lulesh):
    with lulesh.LuleshSet(nx=12, its=-1) as a:
        ck = a.checkpoint()
    for kw in ({"nx": 13}, {"nx": 12, "numReg": 5}, {"nx": 12, "flags": lulesh.FLAG_MIXED}):
        with lulesh.LuleshSet(its=-1, **kw) as b:
            with pytest.raises(lulesh.LuleshError):
                b.restore(ck)
    with lulesh.LuleshSet(nx=12, its=-1) as b:
        with pytest.raises(lulesh.LuleshError):
            b.restore(ck[: len(ck) // 2])
        with pytest.raises(lulesh.LuleshError):
            b.restore(b"x" * len(ck))


def test_checkpoint_of_another_mesh_file_is_refused(lulesh, tmp_path):
    """Two lmesh files with the same element and node counts but different
    geometry: a checkpoint of one loads into a set of the same file and is
    refused by a set of the other."""
    import lmesh

    a_path, b_path = tmp_path / "a.lmesh", tmp_path / "b.lmesh"
    lmesh.write(a_path, lmesh.box(6))
    lmesh.write(b_path, lmesh.warp(lmesh.box(6)))
    with lulesh.LuleshSet.from_mesh(str(a_path), its=-1) as a:
        a.step(3)
        ck = a.checkpoint()
    with lulesh.LuleshSet.from_mesh(str(a_path), its=-1) as same:
        same.restore(ck)
        assert same.state()["cycle"] == 3
    with lulesh.LuleshSet.from_mesh(str(b_path), its=-1) as other:
        with pytest.raises(lulesh.LuleshError):
            other.restore(ck)
