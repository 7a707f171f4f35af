"""bench.py's reference arm on the host cores: one JSON line in the
contract's shape, timed on the reference's own omp build (when it was built
here), and the argument checks that keep a run valid."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(REPO, "bench.py")
OMP = os.path.join(REPO, "oracle", "_ref", "lulesh_omp")


def _bench(*args):
    return subprocess.run([sys.executable, BENCH, *args], capture_output=True, text=True,
                          timeout=600, cwd=REPO)


@pytest.mark.skipif(not os.path.exists(OMP), reason="reference omp build absent")
def test_reference_arm_line():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "config", "cpu_baseline",
              "e2e"):
        assert k in d, k
    assert d["unit"] == "zone-cycles/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "workload" in d["config"]


def test_too_few_warmup_steps_are_refused():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "2")
    assert r.returncode != 0 and "warmup" in r.stderr
