"""The C-ABI library loads and exports every entry point include/nqs.h declares (no GPU needed:
no compute call is made)."""
import os
import re

from nqs import _lib

HDR = os.path.join(os.path.dirname(__file__), os.pardir, "include", "nqs.h")


def declared():
    src = open(HDR).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*|unsigned long long)\s+(nqs_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in declared() if getattr(L, n, None) is None]
    assert not missing, missing
    assert L.nqs_version() >= 1


def test_bindings_cover_header():
    assert set(declared()) <= set(_lib._SIGS)


def test_status_strings_and_bad_args():
    import ctypes
    L = _lib.lib()
    assert L.nqs_status_string(0) == b"ok"
    h = ctypes.c_void_p()
    assert L.nqs_model_create(None, ctypes.byref(h)) != 0
    d = _lib.NqsModelDesc()
    assert L.nqs_model_create(ctypes.byref(d), ctypes.byref(h)) == _lib.NQS_ERR_INVALID_ARG
    assert b"non-positive" in L.nqs_last_error()
