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


def test_model_descriptor_validation_on_host():
    """nqs_model_create validates the descriptor on the host before any device call (status
    codes and messages; reference errors: a ValueError for a bad setup, rashba_reference.py:95-96):
    a valid descriptor passes validation and then needs a device, while sizes beyond the
    compiled limits, heads not dividing the width, a singular cell and out-of-range parameter
    offsets are refused."""
    import ctypes
    import numpy as np
    from helpers import build
    L = _lib.lib()
    g, model = build(N=5, L=7.0, embed=16, heads=4)

    def create(mutate=None):
        desc, keep = model.descriptor()
        if mutate:
            mutate(desc)
        h = ctypes.c_void_p()
        return L.nqs_model_create(ctypes.byref(desc), ctypes.byref(h)), L.nqs_last_error()

    st, msg = create(lambda d: setattr(d, "n_elec", 65))
    assert st == _lib.NQS_ERR_UNSUPPORTED and b"compiled limits" in msg
    st, _ = create(lambda d: setattr(d, "n_heads", 3))
    assert st == _lib.NQS_ERR_UNSUPPORTED
    st, msg = create(lambda d: [d.A.__setitem__(i, v) for i, v in enumerate((1.0, 2.0, 2.0, 4.0))])
    assert st == _lib.NQS_ERR_INVALID_ARG and b"singular" in msg
    st, msg = create(lambda d: setattr(d, "off_embed_kernel", d.n_params))
    assert st == _lib.NQS_ERR_INVALID_ARG and b"offset" in msg
    st, _ = create(lambda d: setattr(d, "n_freq", 0))
    assert st == _lib.NQS_ERR_INVALID_ARG
    if not __import__("torch").cuda.is_available():
        st, _ = create()  # valid: validation passes, the device upload has no device
        assert st == _lib.NQS_ERR_CUDA
