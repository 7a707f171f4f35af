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

RTOL = 1e-12  # the parity tolerance of the one-cycle field tests

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


def test_noalloc_forces_match_regular_entry_point(lulesh):
    torch = pytest.importorskip("torch")
    lib = lulesh.load_library()
    nx = 14
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
