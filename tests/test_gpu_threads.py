"""Sets are thread-compatible: one set per host thread, several threads at
once (ctypes releases the GIL during each call).  Staged subdomain sets
build their message tables concurrently; results equal sequential runs."""
import threading

import pytest

pytestmark = pytest.mark.gpu


def _job(lulesh, nx, flags, out, key):
    with lulesh.LuleshSet(nx=nx, tp=2, its=30, flags=flags) as s:
        s.run()
        out[key] = s.origin_energy()


def test_staged_sets_on_concurrent_threads(lulesh):
    cases = [(6, lulesh.FLAG_COMM_STAGED), (7, lulesh.FLAG_COMM_STAGED), (6, 0), (8, 0)]
    seq = {}
    for i, (nx, fl) in enumerate(cases):
        _job(lulesh, nx, fl, seq, i)
    par = {}
    threads = [threading.Thread(target=_job, args=(lulesh, nx, fl, par, i))
               for i, (nx, fl) in enumerate(cases)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert par == seq
