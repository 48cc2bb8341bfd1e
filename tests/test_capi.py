"""liberq.so loads and exports every entry point include/*.h declares.

No compute calls: these run without a GPU.
"""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from conftest import PKG, REPO

LIB = os.path.join(PKG, "lib", "liberq.so")


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        names.update(re.findall(r"ERQ_API\s+[\w\s\*]+?\b(erq_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", PKG], check=True)
    return C.CDLL(LIB)


def test_headers_declare_entry_points():
    names = declared_symbols()
    for n in ("erq_index_load", "erq_search", "erq_rotate", "erq_index_free", "erq_search_raw"):
        assert n in names


def test_every_declared_symbol_is_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s+(erq_\w+)", out))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for n in declared_symbols():
        assert hasattr(lib, n)


def test_python_binding_symbol_list_matches_headers():
    import erq_b200

    assert sorted(erq_b200.EXPORTED_SYMBOLS) == declared_symbols()


def test_version_and_status_strings(lib):
    lib.erq_version.restype = C.c_int
    assert lib.erq_version() == 1
    lib.erq_status_string.restype = C.c_char_p
    lib.erq_status_string.argtypes = [C.c_int]
    assert lib.erq_status_string(0) == b"ok"
    assert lib.erq_status_string(4) == b"unsupported"
    lib.erq_last_error.restype = C.c_char_p
    assert isinstance(lib.erq_last_error(), bytes)


def test_null_arguments_are_rejected_without_touching_the_gpu(lib):
    """Argument checks run before any CUDA call."""
    import erq_b200._lib as L

    lib2 = L.load_library()
    out = C.c_void_p()
    assert lib2.erq_index_load(None, 0, C.byref(out)) == 1
    assert b"NULL" in lib2.erq_last_error()
    info = L.IndexInfo()
    assert lib2.erq_index_get_info(None, C.byref(info)) == 1
    assert lib2.erq_search(None, None, 1, 10, 1, None, None, None) == 1
    assert lib2.erq_rotate(None, None, 1, None, None) == 1


def test_no_cpu_fallback_when_library_missing(tmp_path, monkeypatch):
    import erq_b200._lib as L

    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(ImportError, match="no CPU fallback"):
        L.load_library(str(tmp_path / "missing.so"))
