"""Single-domain geometry built on the device (setup.cu) against the host
builder (LULESH_FLAG_HOST_SETUP, the NewDomain restatement): every Domain
array equal bit for bit, before the first cycle and after a run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["e", "p", "q", "ql", "qq", "v", "volo", "delv", "vdov", "arealg", "ss", "elemMass",
          "x", "y", "z", "xd", "yd", "zd", "nodalMass", "fx_elem", "nodelist", "lxim", "lxip",
          "letam", "letap", "lzetam", "lzetap", "elemBC", "matElemlist", "regNumList",
          "regElemlist", "eosOrder", "nodeElemCount", "nodeElemStart", "nodeElemCornerList", "symmX",
          "symmY", "symmZ", "regCSR", "regReps", "regSorted"]


def _same(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("nx,nr,b,c", [(1, 11, 1, 1), (2, 5, 2, 1), (7, 11, 1, 1),
                                       (30, 20, 4, 4), (45, 11, 1, 1)])
def test_device_setup_equals_host_setup(lulesh, nx, nr, b, c):
    kw = dict(nx=nx, numReg=nr, balance=b, cost=c, its=25)
    with lulesh.LuleshSet(**kw) as dev, \
            lulesh.LuleshSet(flags=lulesh.FLAG_HOST_SETUP, **kw) as host:
        for name in FIELDS:
            assert _same(dev.field(name), host.field(name)), name
        assert dev.state()["deltatime"] == host.state()["deltatime"]
        assert dev.run() == host.run() == lulesh.OK
        assert dev.origin_energy() == host.origin_energy()
        assert np.array_equal(dev.field("e"), host.field("e"))


def test_batch_uses_device_setup_with_same_results(lulesh):
    jobs = [lulesh.JobSpec(n, r, bb, cc, 30) for n, r, bb, cc in
            [(9, 7, 2, 2), (16, 11, 1, 1), (5, 20, 4, 1)]]
    with lulesh.LuleshSet.batch(jobs) as dev, \
            lulesh.LuleshSet.batch(jobs, flags=lulesh.FLAG_HOST_SETUP) as host:
        for d in range(3):
            for name in ("x", "volo", "nodalMass", "nodeElemCornerList", "regNumList",
                         "regElemlist", "eosOrder"):
                assert _same(dev.field(name, d), host.field(name, d)), (d, name)
        dev.run()
        host.run()
        assert [dev.origin_energy(i) for i in range(3)] == [host.origin_energy(i) for i in range(3)]
