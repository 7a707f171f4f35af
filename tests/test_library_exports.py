"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from conftest import REPO


def _declared():
    names = set()
    inc = os.path.join(REPO, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(inc, fn)) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(lulesh_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(lulesh):
    lib = lulesh.load_library()
    declared = _declared()
    assert len(declared) >= 30
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # the binding's list covers the header
    assert declared <= set(lulesh.EXPORTED), declared - set(lulesh.EXPORTED)


def test_checked_build_exports_the_same_symbols(lulesh):
    """liblulesh_b200_checked.so (-DLULESH_CHECKED=1) is a drop-in for the
    normal library: same symbols, and the bounds status has its name."""
    path = os.path.join(REPO, "cuda-ipc-benchmarks_b200", "liblulesh_b200_checked.so")
    assert os.path.exists(path), "build it with make -C cuda-ipc-benchmarks_b200"
    lib = lulesh.load_library(path)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.lulesh_status_string(lulesh.BOUNDS_ERROR).startswith(b"index out of range")


def test_status_strings_without_device(lulesh):
    lib = lulesh.load_library()
    assert lib.lulesh_status_string(-1) == b"VolumeError"
    assert lib.lulesh_status_string(-2) == b"QStopError"
    assert lib.lulesh_status_string(-3) == b"LFileError"


def test_footprint_model_without_device(lulesh):
    """The admission model is host arithmetic: ~0.6 kB per element."""
    one = lulesh.footprint_bytes([lulesh.JobSpec(100)])
    assert 400 * 10**6 < one < 800 * 10**6
    two = lulesh.footprint_bytes([lulesh.JobSpec(50)], tp=2)
    assert two > one * 0.9  # 8 subdomains of 50^3 plus comm buffers


def test_oversize_job_rejected_before_touching_a_device(lulesh):
    """nx above LULESH_MAX_NX (645) would overflow the 32-bit corner index
    elem + padded_numElem * corner; lulesh_create refuses it up front."""
    lib = lulesh.load_library()
    h = ctypes.c_void_p()
    for nx in (646, 1000):
        job = lulesh.JobSpec(nx).c()
        st = lib.lulesh_create(ctypes.byref(job), 1, 0, -1, ctypes.byref(h))
        assert st == lulesh.INVALID_ARG and not h.value
        assert b"645" in lib.lulesh_last_error()
    assert lulesh.MAX_NX == 645
