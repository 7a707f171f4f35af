"""The checked build stands in for a memory checker.

liblulesh_b200_checked.so is the library compiled with -DLULESH_CHECKED=1:
every index the FP64 cycle kernels compute or load (node indices, corner
indices, corner-list runs, EOS slots, face links) is range-checked first; an
index out of range would be replaced by 0 and end the job with
LULESH_BOUNDS_ERROR.  The checked build runs every kind of FP64 set (single
domains from one element up, fused and staged subdomains, a batch, an
unstructured mesh) to its end: no index may be out of range, and every
result must equal the normal build's bit for bit."""
import json
import os
import subprocess
import sys

import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CHECKED = os.path.join(PKG, "liblulesh_b200_checked.so")
NORMAL = os.path.join(PKG, "liblulesh_b200.so")


def _run(lib, tmp):
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_cases.py"), lib, str(tmp)],
                       capture_output=True, text=True, timeout=600)
    line = [x for x in r.stdout.splitlines() if x.startswith("RESULT ")]
    assert r.returncode == 0 and line, r.stderr[-3000:]
    return json.loads(line[0][7:])


def test_checked_build_runs_clean_and_identical(lulesh, tmp_path):
    if not os.path.exists(CHECKED):
        pytest.fail("liblulesh_b200_checked.so is missing: make -C cuda-ipc-benchmarks_b200")
    checked = _run(CHECKED, tmp_path)
    normal = _run(NORMAL, tmp_path)
    assert checked.keys() == normal.keys()
    for name in checked:
        c, n = checked[name], normal[name]
        assert c["status"] == lulesh.OK, (name, c["status"])
        assert all(st["status"] == lulesh.OK and st["done"] for st in c["states"]), name
        assert c["states"] == n["states"], name
        assert c["digest"] == n["digest"], name
