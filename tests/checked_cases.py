"""Runs the checked-build cases of test_gpu_checked.py in one process, with
the library named on the command line, and prints one JSON line of results.
(Not collected by pytest: no test_ prefix.)"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "cuda-ipc-benchmarks_b200"))

import numpy as np  # noqa: E402

import lmesh  # noqa: E402
import lulesh_b200 as L  # noqa: E402


def _digest(s, ndom):
    h = hashlib.sha1()
    for d in range(ndom):
        for f in ("e", "p", "q", "v", "x", "xd"):
            h.update(s.field(f, domain=d).tobytes())
    return h.hexdigest()


def run(tmpdir):
    out = {}

    def record(name, s, ndom=1, njobs=1):
        st = s.run()
        out[name] = {"status": st, "states": [s.state(j) for j in range(njobs)],
                     "digest": _digest(s, ndom)}

    for nx, its in ((1, -1), (5, -1), (12, 40)):
        with L.LuleshSet(nx=nx, its=its) as s:
            record(f"single_{nx}", s)
    with L.LuleshSet(nx=12, its=40, flags=L.FLAG_MIXED) as s:
        record("mixed", s)
    for flags, name in ((0, "fused"), (L.FLAG_COMM_STAGED, "staged")):
        with L.LuleshSet(nx=6, tp=2, its=30, flags=flags) as s:
            record(f"subdomains_{name}", s, ndom=8)
    jobs = [L.JobSpec(6, 5, 1, 1, 25), L.JobSpec(11, 20, 4, 2, 25), L.JobSpec(9, 11, 2, 4, 25)]
    with L.LuleshSet.batch(jobs) as s:
        record("batch", s, ndom=3, njobs=3)
    m = lmesh.box(6)
    path = os.path.join(tmpdir, "warped6.lmesh")
    lmesh.write(path, lmesh.warp(m))
    with L.LuleshSet.from_mesh(path) as s:
        record("unstructured", s)
    # nodes with more than 8 corners (duplicated elements): the staged and
    # the list-reading corner-run paths of the unstructured nodal kernel
    for name, nx, dup in (("dup_one", 8, [200]), ("dup_all", 6, None)):
        b = lmesh.box(nx)
        idx = list(range(b.num_elem)) if dup is None else dup
        d = lmesh.LMesh(b.xyz, np.concatenate([b.nodelist, b.nodelist[idx]]),
                        np.concatenate([b.links, b.links[idx]]), b.symm, b.free)
        path = os.path.join(tmpdir, name + ".lmesh")
        lmesh.write(path, d)
        with L.LuleshSet.from_mesh(path) as s:
            record(name, s)
    return out


if __name__ == "__main__":
    L._lib = L.load_library(sys.argv[1])
    print("RESULT " + json.dumps(run(sys.argv[2])), flush=True)
