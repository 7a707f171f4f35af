"""bench.py's N-GPU path, run as the driver runs it (torch.distributed.run,
one process per rank), with two ranks on this one GPU and the host
transport: the ranks' hosts exchange the halo messages over gloo, no kernel
waits on another.  It checks the JSON line of the decomposed problem (2x2x2
subdomains split over the ranks) and its energy against the single domain
of the same mesh, read at the end of the device-timed cycles (the
host-driven end-to-end cycles run after it)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu


def test_two_rank_decomposed_bench_line(lulesh):
    port = 29900 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--gpus", "2", "--steps", "3", "--warmup", "3", "--transport", "host"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["steps"] == 3 and d["scaling"] == "weak"
    assert d["config"]["tp"] == 2 and d["config"]["transport"] == "host"
    nx = d["config"]["nx"]
    assert d["config"]["zones"] == (2 * nx) ** 3 and d["value"] > 0
    # end to end: host-driven cycles with each cycle's dt record read back
    assert d["e2e"]["value"] > 0 and d["e2e"]["value"] != d["value"]
    assert d["e2e"]["d2h_bytes_per_step"] == 32
    assert "sm_mhz" in d["clocks"]
    with lulesh.LuleshSet(nx=2 * nx, its=-1, device=0) as single:
        single.step(6)
        assert d["origin_energy"] == single.origin_energy()
