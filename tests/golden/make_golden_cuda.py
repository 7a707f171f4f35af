"""Generate tests/golden/cuda_reference.json from the reference's own CUDA
single-domain build (oracle/_ref/lulesh_ref_cuda, compiled from
LULESH/cuda/src by oracle/Makefile for sm_100a with the 17-digit print hook).
It needs a B200, so it runs on a GPU machine with the built tree:

    make -C oracle ref                         # in the build container
    python tests/golden/make_golden_cuda.py [out.json]   # on the GPU machine

The reference CUDA command line is `lulesh -s N x ITERS` (lulesh.cu:4754-4770;
argv[4] is the iteration cap, -1 runs to the stop time); it fixes
-r 11 -b 1 -c 1 (lulesh.cu:4803-4805).
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
from oracle import REF_CUDA, parse_report  # noqa: E402

# (edge, iterations); -1 = run to the stop time t = 1e-2
CASES = [
    (10, 50),
    (30, 100),
    (30, -1),      # config 1 size, full run
    (45, 300),
    (64, 100),
    (90, 200),     # the published -s 45 x 8 ranks case as one domain
    (100, 500),    # config 2
    (120, 1000),   # config 4 FP64 reference
    # -s 100 after the cycle counts bench.py ends its timed region on
    # (warm-up + steps: 5 + 20, 5 + 100, 5 + 500, 5 + 1000); the bench checks
    # its energy against these
    (100, 25),
    (100, 105),
    (100, 505),
    (100, 1005),
]


def main():
    runs = {}
    for nx, its in CASES:
        args = ["-s", str(nx), "x", str(its)]
        out = subprocess.run([REF_CUDA, *args], capture_output=True, text=True, check=True,
                             cwd=os.path.join(REPO, "oracle", "_ref")).stdout
        r = parse_report(out)
        r.pop("elapsed", None)
        r.pop("grind", None)
        runs[f"-s {nx} -i {its}"] = dict(nx=nx, its=its, **r)
        print(nx, its, r, flush=True)
    doc = {
        "source": "reference LULESH/cuda/src single-domain build (oracle/Makefile, nvcc "
                  "-O3 -DNDEBUG sm_100a, USE_MPI undefined), run on one B200, 17-digit "
                  "print hook",
        "runs": runs,
    }
    # an optional path argument writes the table elsewhere (to bring it back
    # from the GPU machine); the default is the committed fixture
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "cuda_reference.json")
    with open(out, "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main()
