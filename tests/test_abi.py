"""CPU checks of the C ABI: the library loads, exports every symbol its header
declares, and reports errors as status codes (no compute call needs a GPU here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, load_pkg

HEADER = os.path.join(ROOT, "include", "ndb_b200.h")


def header_symbols(path=HEADER):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ndb_b200_\w+)\s*\(", text)))


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_header_declares_entry_points():
    syms = header_symbols()
    for s in ("ndb_b200_create", "ndb_b200_run", "ndb_b200_classify", "ndb_b200_assign_labels",
              "ndb_b200_strerror"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    pkg = load_pkg()
    lib = pkg.lib.load()
    for s in header_symbols():
        assert hasattr(lib, s), f"{s} declared in ndb_b200.h but not exported"
    assert set(pkg.lib.EXPORTED) <= set(header_symbols())


def test_every_header_under_include_is_exported():
    pkg = load_pkg()
    lib = pkg.lib.load()
    inc = os.path.join(ROOT, "include")
    for h in os.listdir(inc):
        if h.endswith(".h"):
            for s in header_symbols(os.path.join(inc, h)):
                assert hasattr(lib, s), f"{s} ({h}) not exported"


def test_strerror_and_version():
    lib = load_pkg().lib.load()
    assert lib.ndb_b200_strerror(0) == b"ok"
    assert b"dimensionality" in lib.ndb_b200_strerror(2)
    assert lib.ndb_b200_strerror(12345) == b"unknown status"
    assert lib.ndb_b200_version().count(b".") == 2


def test_status_codes_without_gpu():
    pkg = load_pkg()
    lib = pkg.lib.load()
    h = ctypes.c_void_p()
    assert lib.ndb_b200_create(None, 0) == 1  # null out-pointer
    assert lib.ndb_b200_set_memory_limit(None, 0) == 1
    assert lib.ndb_b200_device_bytes(None, None) == 1
    assert lib.ndb_b200_set_tuning(None, None) == 1
    assert lib.ndb_b200_get_tuning(None, None) == 1
    if cuda_available():
        pytest.skip("a GPU is present; the no-device path is not reachable")
    assert lib.ndb_b200_create(ctypes.byref(h), 0) == 7  # NDB_ERR_NO_DEVICE
    assert lib.ndb_b200_classify(None, None, 0, 2, ctypes.c_float(1.0), 1, 0, None) == 1
    assert lib.ndb_b200_assign_labels(None, None, None) == 1
    assert lib.ndb_b200_destroy(None) == 0


def test_python_mirror_fails_loudly_without_device():
    pkg = load_pkg()
    if cuda_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.lib.NdbError):
        pkg.Context(0)


def test_autotune_candidates():
    at = load_pkg().autotune
    assert at.candidates(3) == []
    c8 = at.candidates(8)
    assert c8[0] == at.EXACT_ONLY and c8[1] == at.GRAM_ONLY and len(c8) == 2 + len(at.ITEM_SIZES)
    assert all(c["tc_min_dim"] == 8 for c in c8[2:])
