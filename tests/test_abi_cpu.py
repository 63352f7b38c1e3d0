"""CPU-only checks of the C ABI: the library loads and exports every symbol
include/rpb200.h declares; calls that need a device fail loudly (no CPU
fallback)."""
import ctypes as C

import pytest

from reapers_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert sorted(_lib._SIGS) == declared


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    bits = (C.c_uint64 * 1)(1)
    coeff = (C.c_double * 2)(1.0, 0.0)
    rc = lib.rp_ham_create(C.byref(h), 4, 2, 1, bits, coeff)
    assert rc != 0
    assert b"device" in lib.rp_last_error().lower()


def test_device_count_without_device():
    n = C.c_int(-1)
    assert _lib.load().rp_device_count(C.byref(n)) == 0
    assert n.value >= 0
