"""The lulesh_b200 command line as the reference's harnesses drive and parse
it: the CUDA form (-s N x ITERS), the harness form (-s N 0 ITERS), the omp
flags, and the report fields the sbatch scripts read with awk
(run_lulesh.sbatch:83-85, run_lulesh_lifecycle.sbatch:96-103)."""
import os
import re
import subprocess

import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu

EXE = os.path.join(PKG, "lulesh_b200")


def _run(*args, cwd=None):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=120, cwd=cwd)


def _awk(out, pattern, field):
    """awk '/pattern/{print $field}': every matching line's field."""
    return [line.split()[field - 1] for line in out.splitlines() if pattern in line]


@pytest.mark.parametrize("args", [["-s", "12", "x", "40"], ["-s", "12", "0", "40"],
                                  ["-s", "12", "-i", "40"]])
def test_report_fields_parse_like_the_harness(lulesh, args, tmp_path):
    r = _run(*args, "--no-xyz", cwd=tmp_path) if args[2] == "-i" else _run(*args, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    energy = _awk(r.stdout, "Final Origin Energy", 5)
    elapsed = _awk(r.stdout, "Elapsed time", 4)
    fom = _awk(r.stdout, "FOM", 3)
    assert len(energy) == len(elapsed) == len(fom) == 1, r.stdout
    assert int(_awk(r.stdout, "Iteration count", 4)[0]) == 40
    with lulesh.LuleshSet(nx=12, its=40) as s:
        s.run()
        e = s.origin_energy()
    assert energy[0] == f"{e:12.6e}".strip()
    full = float(re.search(r"Origin energy, 17 digits = (\S+)", r.stdout).group(1))
    assert full == e
    float(elapsed[0]), float(fom[0])
    assert ("xyz.asc" in os.listdir(tmp_path)) == (args[2] != "-i")


def test_subdomain_run_prints_lifecycle_lines(tmp_path):
    r = _run("-s", "8", "-t", "2", "-i", "20", "--no-xyz", cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    for name in ("COMM_SETUP", "WIN_ALLOCATE", "PEER_QUERY", "COMM_FREE", "APP_TOTAL"):
        m = re.search(rf"PHASE_{name}_ms\s+([0-9.]+)", r.stdout)
        assert m, name
    assert _awk(r.stdout, "MPI tasks", 4) == ["8"]


def test_errors_map_to_reference_exit_codes(tmp_path):
    # exit(LFileError) with LFileError = -3 (lulesh.h:22-26): status 253
    assert _run("-u", "mesh.lmesh", cwd=tmp_path).returncode == (-3) & 0xFF
    r = _run("-s", "8", "--bogus", cwd=tmp_path)
    assert r.returncode != 0 and "Unknown command line argument" in r.stdout
    r = _run("-s", "646", "-i", "1", "--no-xyz", cwd=tmp_path)  # above LULESH_MAX_NX
    assert r.returncode != 0
    r = _run("-s", "8", "-i", "5", "-q", "--no-xyz", cwd=tmp_path)
    assert r.returncode == 0 and r.stdout == ""


def test_unstructured_form(tmp_path):
    """-u FILE x ITERS: the reference's unstructured report (problem size =
    element count, no plane-0 block), and the -s 45 cube as an lmesh file
    gives the -s 45 energy."""
    import lmesh

    p = tmp_path / "box45.lmesh"
    lmesh.write(p, lmesh.box(45))
    u = _run("-u", str(p), "x", "100", cwd=tmp_path)
    s = _run("-s", "45", "x", "100", cwd=tmp_path)
    assert u.returncode == 0 and s.returncode == 0, u.stdout + u.stderr
    assert "Problem size=91125" in u.stdout
    assert not _awk(u.stdout, "Final Origin Energy", 5)
    full = [re.search(r"Origin energy, 17 digits = (\S+)", r.stdout).group(1) for r in (u, s)]
    assert full[0] == full[1]
    assert len(_awk(u.stdout, "FOM", 3)) == 1


def test_one_launch_gives_the_same_run(tmp_path):
    """--one-launch (the device-side loop) and the default per-cycle graph
    launches print the same energy and iteration count."""
    outs = [_run("-s", "12", "-i", "40", "--no-xyz", *extra, cwd=tmp_path)
            for extra in ([], ["--one-launch"])]
    for r in outs:
        assert r.returncode == 0, r.stdout + r.stderr
    full = [re.search(r"Origin energy, 17 digits = (\S+)", r.stdout).group(1) for r in outs]
    assert full[0] == full[1]
    assert _awk(outs[0].stdout, "Iteration count", 4) == _awk(outs[1].stdout, "Iteration count", 4)


def _read_xyz(path):
    """xyz.asc as write_solution writes it (lulesh.cu:4584-4603): per node a
    "%10d" index line, then x, y and z on lines of their own."""
    with open(path) as f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    assert len(lines) % 4 == 0
    idx = [int(lines[k]) for k in range(0, len(lines), 4)]
    xyz = [[float(lines[k + c]) for c in (1, 2, 3)] for k in range(0, len(lines), 4)]
    return lines, idx, xyz


def test_xyz_solution_file_content(tmp_path, oracle_mod):
    """`lulesh_b200 -s 10 x 20` writes the node coordinates of cycle 20 in
    the reference's format: 10-wide index lines and %.10f values, equal to
    the oracle's coordinates to the printed precision; and the same file the
    reference CUDA build writes (its 17-digit print hook) to 1e-9."""
    r = _run("-s", "10", "x", "20", cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines, idx, xyz = _read_xyz(tmp_path / "xyz.asc")
    nn = 11 ** 3
    assert idx == list(range(nn))
    assert all(len(lines[k]) == 10 for k in range(0, len(lines), 4))
    assert all(re.fullmatch(r"-?\d+\.\d{10}", lines[k + c])
               for k in range(0, len(lines), 4) for c in (1, 2, 3))
    o = oracle_mod.Oracle(10)
    st, n = o.run(20)
    assert st == 0 and n == 20
    ref = list(zip(o.field("x"), o.field("y"), o.field("z")))
    for got, want in zip(xyz, ref):
        for g, w in zip(got, want):
            assert abs(g - w) <= 5.000001e-11
    ref_bin = os.path.join(os.path.dirname(PKG), "oracle", "_ref", "lulesh_ref_cuda")
    if os.path.exists(ref_bin):
        rd = tmp_path / "ref"
        rd.mkdir()
        rr = subprocess.run([ref_bin, "-s", "10", "x", "20"], capture_output=True, text=True,
                            timeout=300, cwd=rd)
        assert rr.returncode == 0, rr.stdout + rr.stderr
        _, ridx, rxyz = _read_xyz(rd / "xyz.asc")
        assert ridx == idx
        for got, want in zip(xyz, rxyz):
            for g, w in zip(got, want):
                assert abs(g - w) <= 5.000001e-11 + 1e-9 * abs(w)
