"""lulesh_volume_force_noalloc: nodal forces for callers that cannot allocate.

Some callers of this library cannot allocate device memory -- a host code
whose own memory manager owns the GPU's whole budget, or a loop that cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree.  The
no-allocation entry point serves them with a fixed scratch array inside the
library.  This test gives it caller-owned device buffers (allocated here by
torch, on the caller's side) and checks its forces against the forces the
regular entry point (lulesh_lagrange_leapfrog with the materialize flag)
computes from the same state, on two calls in a row, so the second call
also shows that the shared scratch array is reused correctly.

Collected last on purpose (file name), so a stopping run has already run
every other test if this one fails.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# The no-allocation kernel evaluates every force expression in the same
# written form, and sums each node's corners in the same order (corner 0..7),
# as the regular force and nodal kernels, so nvcc makes the same multiply-add
# contractions and the forces agree bit for bit; RTOL is the parity tolerance
# of the one-cycle field tests, kept as the bound the bit-for-bit check
# tightens.
RTOL = 1e-12

NODE_IN = ["x", "y", "z", "xd", "yd", "zd"]
ELEM_IN = ["volo", "v", "p", "q", "ss", "elemMass"]


def _call(lib, torch, nx, state, bad_elem=True):
    dev = [torch.from_numpy(state[k]).cuda() for k in NODE_IN + ELEM_IN]
    nn = (nx + 1) ** 3
    out = [torch.empty(nn, dtype=torch.float64, device="cuda") for _ in range(3)]
    bad = torch.full((1,), 12345, dtype=torch.int32, device="cuda")
    ptr = [ctypes.c_void_p(t.data_ptr()) for t in dev]
    st = lib.lulesh_volume_force_noalloc(
        nx, *ptr, 3.0, *[ctypes.c_void_p(t.data_ptr()) for t in out],
        ctypes.c_void_p(bad.data_ptr()) if bad_elem else None,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st, [t.cpu().numpy() for t in out], int(bad.cpu().item())


def _state(s):
    return {k: s.field(k) for k in NODE_IN + ELEM_IN}


@pytest.mark.parametrize("nx", [14, 32])  # 32: the array's full capacity (32,768 elements)
def test_noalloc_forces_match_regular_entry_point(lulesh, nx):
    torch = pytest.importorskip("torch")
    lib = lulesh.load_library()
    with lulesh.LuleshSet(nx=nx, its=-1, flags=lulesh.FLAG_MATERIALIZE, device=0) as s:
        # at cycle 0 pressure and velocity are zero everywhere and so is every
        # force; a few cycles in, the blast gives both calls non-zero forces
        s.step(4)
        for call in range(2):
            state = _state(s)  # state at the start of the next cycle
            s.step(1)          # regular path: forces of that state, kept in fx/fy/fz
            ref = [s.field(f) for f in ("fx", "fy", "fz")]
            st, got, bad = _call(lib, torch, nx, state)
            assert st == lulesh.OK, lib.lulesh_last_error()
            assert bad == -1
            for g, r in zip(got, ref):
                scale = max(float(np.max(np.abs(r))), 1e-300)
                assert np.allclose(g, r, rtol=RTOL, atol=RTOL * scale), f"call {call}"
                assert np.array_equal(g, r), f"call {call}: not bit-identical"
            assert np.any(got[0] != 0.0)


def test_noalloc_rejects_meshes_above_the_fixed_scratch(lulesh):
    lib = lulesh.load_library()
    # rejected on nx before any pointer is looked at or any launch is made
    st = lib.lulesh_volume_force_noalloc(33, *([None] * 12), 3.0, None, None, None, None, None)
    assert st == lulesh.INVALID_ARG
    assert b"32" in lib.lulesh_last_error()


def test_noalloc_reports_volume_error(lulesh):
    torch = pytest.importorskip("torch")
    lib = lulesh.load_library()
    nx = 5
    with lulesh.LuleshSet(nx=nx, its=-1, device=0) as s:
        state = _state(s)
    state["v"][7] = -1.0
    st, _, bad = _call(lib, torch, nx, state)
    assert st == lulesh.OK and bad == 7


_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import lulesh_b200 as L

lib = L.load_library()
rt = ctypes.CDLL("libcudart.so.12")  # the runtime the library already loaded
NODE_IN = ["x", "y", "z", "xd", "yd", "zd"]
ELEM_IN = ["volo", "v", "p", "q", "ss", "elemMass"]
nx = 8
with L.LuleshSet(nx=nx, its=-1, device=0) as s:
    s.step(4)
    state = [s.field(k) for k in NODE_IN + ELEM_IN]

def ck(e, what):
    if e != 0:
        raise SystemExit(f"{what}: cudaError {e}")

def forces():
    ptrs = []
    for a in state:
        p = ctypes.c_void_p()
        ck(rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(a.nbytes)), "cudaMalloc")
        ck(rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes), 1),
           "cudaMemcpy H2D")
        ptrs.append(p)
    nn = (nx + 1) ** 3
    outs = []
    for _ in range(3):
        p = ctypes.c_void_p()
        ck(rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(8 * nn)), "cudaMalloc")
        outs.append(p)
    st = lib.lulesh_volume_force_noalloc(nx, *ptrs, 3.0, *outs, None, None)
    if st != 0:
        raise SystemExit(f"noalloc status {st}: {lib.lulesh_last_error()}")
    ck(rt.cudaDeviceSynchronize(), "cudaDeviceSynchronize")
    res = []
    for p in outs:
        h = np.empty(nn, dtype=np.float64)
        ck(rt.cudaMemcpy(h.ctypes.data_as(ctypes.c_void_p), p, ctypes.c_size_t(8 * nn), 2),
           "cudaMemcpy D2H")
        res.append(h)
    for p in ptrs + outs:
        ck(rt.cudaFree(p), "cudaFree")
    return res

before = forces()
ck(rt.cudaDeviceReset(), "cudaDeviceReset")  # ends this process's own context only
after = forces()
assert all(np.array_equal(a, b) for a, b in zip(before, after)), "forces changed"
assert np.any(before[0] != 0.0)
print("RESET_OK")
"""


def test_noalloc_after_device_reset(lulesh):
    """A device reset reloads the library's module, which may move the
    scratch array; the next call looks its address up again and gives the
    same forces.  Run in a child process so the reset ends only that
    process's own context, not the one the other tests share."""
    import subprocess
    import sys

    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, lulesh.HERE],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "RESET_OK" in r.stdout, r.stdout + r.stderr
