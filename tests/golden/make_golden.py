"""Generate tests/golden/omp_reference.json from the reference's own OpenMP
CPU build (oracle/_ref/lulesh_omp, compiled from LULESH/omp_4.0 by
oracle/Makefile with the 17-digit print hook).  Run in the build container:

    make -C oracle ref && python tests/golden/make_golden.py

The omp build crashes with one thread (LULESH/omp_4.0/lulesh.cc:585), so it
runs with OMP_NUM_THREADS=4.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
from oracle import REF_OMP, parse_report  # noqa: E402

CASES = [
    ["-s", "5", "-i", "10"],
    ["-s", "10", "-i", "5"],
    ["-s", "10", "-i", "50"],
    ["-s", "12", "-i", "200"],
    ["-s", "15", "-i", "60"],
    ["-s", "30", "-i", "20"],
    ["-s", "30", "-i", "100"],
    ["-s", "30", "-i", "100", "-r", "20", "-b", "4", "-c", "4"],
    ["-s", "8", "-i", "400"],
]


def main():
    env = dict(os.environ, OMP_NUM_THREADS="4")
    runs = {}
    for args in CASES:
        out = subprocess.run([REF_OMP, *args], env=env, capture_output=True, text=True,
                             check=True).stdout
        r = parse_report(out)
        r.pop("elapsed", None)
        r.pop("grind", None)
        runs[" ".join(args)] = r
    doc = {
        "source": "reference LULESH/omp_4.0 built by oracle/Makefile (g++ -O3 -fopenmp "
                  "-DUSE_GPU=0 -DUSE_MPI=0), OMP_NUM_THREADS=4, 17-digit print hook",
        "runs": runs,
    }
    with open(os.path.join(HERE, "omp_reference.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print(json.dumps(doc, indent=1))


if __name__ == "__main__":
    main()
