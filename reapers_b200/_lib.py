"""ctypes binding of librpb200.so (the C ABI declared in include/rpb200.h).

The shared library is built in-tree (reapers_b200/librpb200.so) by
``__graft_entry__.build()`` / ``make -C reapers_b200/csrc``.  There is no
fallback: if the library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librpb200.so")

RP_C64 = 1
RP_C128 = 2

_lib = None


class RPError(RuntimeError):
    """A librpb200 call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"librpb200 error {code}: {msg}")
        self.code = code


class HamInfo(C.Structure):
    _fields_ = [("len", C.c_int), ("dtype", C.c_int), ("nterms", C.c_int),
                ("tile_exp", C.c_int), ("ngroups", C.c_int), ("threads", C.c_int),
                ("stages", C.c_int), ("grid", C.c_int), ("alg_bytes", C.c_double),
                ("kernel", C.c_int), ("window", C.c_int), ("alg_bytes_dram", C.c_double),
                ("smem_bytes", C.c_double), ("nreads", C.c_int), ("diag_terms", C.c_int)]


class EvolveStats(C.Structure):
    _fields_ = [("restarts", C.c_int), ("applies", C.c_int), ("passes", C.c_int),
                ("prods", C.c_int), ("breakdown", C.c_int), ("last_err", C.c_double)]


class IpcHandle(C.Structure):
    _fields_ = [("handle", C.c_ubyte * 64), ("offset", C.c_uint64)]


class ArnoldiInfo(C.Structure):
    _fields_ = [("m_eff", C.c_int), ("breakdown", C.c_int), ("passes", C.c_int),
                ("pad", C.c_int), ("beta", C.c_double),
                ("beta0", C.c_double)]


# name -> (restype, argtypes); every exported symbol of include/rpb200.h
_VP = C.c_void_p
_SIGS = {
    "rp_init": (C.c_int, [C.c_int]),
    "rp_shutdown": (C.c_int, []),
    "rp_last_error": (C.c_char_p, []),
    "rp_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "rp_stream": (_VP, []),
    "rp_synchronize": (C.c_int, []),
    "rp_alloc": (C.c_int, [C.POINTER(_VP), C.c_size_t]),
    "rp_free": (C.c_int, [_VP]),
    "rp_memcpy": (C.c_int, [_VP, _VP, C.c_size_t, C.c_int]),
    "rp_vec_zero": (C.c_int, [C.c_int, C.c_uint64, _VP]),
    "rp_vec_copy": (C.c_int, [C.c_int, _VP, C.c_int, _VP, C.c_uint64]),
    "rp_vec_axpy": (C.c_int, [C.c_int, C.c_uint64, _VP, C.c_double, C.c_double, _VP]),
    "rp_vec_add": (C.c_int, [C.c_int, C.c_uint64, _VP, _VP, _VP]),
    "rp_vec_scale": (C.c_int, [C.c_int, C.c_uint64, _VP, C.c_double, C.c_double]),
    "rp_vec_dot": (C.c_int, [C.c_int, C.c_uint64, _VP, _VP, C.POINTER(C.c_double)]),
    "rp_vec_dot_noalloc": (C.c_int, [C.c_int, C.c_uint64, _VP, _VP, C.POINTER(C.c_double)]),
    "rp_vec_norm": (C.c_int, [C.c_int, C.c_uint64, _VP, C.POINTER(C.c_double)]),
    "rp_vec_random": (C.c_int, [C.c_int, C.c_uint64, _VP, C.c_uint64]),
    "rp_ham_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, C.c_uint64,
                                C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "rp_ham_create_ex": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, C.c_uint64,
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int]),
    "rp_ham_destroy": (C.c_int, [_VP]),
    "rp_ham_info": (C.c_int, [_VP, C.POINTER(HamInfo)]),
    "rp_apply": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "rp_test_withhold_tile": (C.c_int, [C.c_int64, C.c_uint32]),
    "rp_apply_host": (C.c_int, [_VP, C.c_int, C.POINTER(_VP), C.POINTER(_VP)]),
    "rp_apply_shard": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(_VP), _VP, C.c_int]),
    "rp_ipc_export": (C.c_int, [_VP, C.POINTER(IpcHandle)]),
    "rp_ipc_open": (C.c_int, [C.POINTER(IpcHandle), C.POINTER(_VP)]),
    "rp_ipc_close": (C.c_int, [_VP]),
    "rp_evolve": (C.c_int, [_VP, _VP, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                            C.POINTER(EvolveStats)]),
    "rp_workspace_release": (C.c_int, []),
    "rp_arnoldi": (C.c_int, [_VP, _VP, C.c_int, C.POINTER(C.c_double), C.POINTER(ArnoldiInfo)]),
    "rp_arnoldi_combine": (C.c_int, [C.POINTER(C.c_double), _VP]),
    "rp_expm_first_column": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]),
    "rp_dense_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, C.c_uint64,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "rp_dense_eigenvalues": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "rp_dense_eigenvector": (C.c_int, [_VP, C.c_int64, _VP]),
    "rp_dense_eigenvectors": (C.c_int, [_VP, C.POINTER(_VP)]),
    "rp_dense_expm": (C.c_int, [_VP, C.c_double, C.c_double, _VP]),
    "rp_dense_destroy": (C.c_int, [_VP]),
    "rp_mat_vec": (C.c_int, [C.c_int, C.c_uint64, _VP, _VP, _VP]),
    "rp_mlp_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, C.c_uint64]),
    "rp_mlp_num_params": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "rp_mlp_get_params": (C.c_int, [_VP, C.POINTER(C.c_float)]),
    "rp_mlp_set_params": (C.c_int, [_VP, C.POINTER(C.c_float)]),
    "rp_mlp_forward": (C.c_int, [_VP, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float)]),
    "rp_mlp_grad": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                              C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "rp_mlp_train": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int,
                               C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "rp_mlp_destroy": (C.c_int, [_VP]),
    "rp_batch_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_uint64)),
                                  C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_double), C.POINTER(_VP), C.POINTER(C.c_int),
                                  C.c_int, C.c_double, C.c_int]),
    "rp_batch_create_ex": (C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_uint64)),
                                     C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_double), C.POINTER(_VP), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.c_int, C.c_double, C.c_int]),
    "rp_batch_otoc": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.POINTER(C.c_int), C.c_int]),
    "rp_batch_probe": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_double)]),
    "rp_batch_destroy": (C.c_int, [_VP]),
}


def header_symbols():
    """Function names declared in include/rpb200.h (parsed from the header)."""
    import re
    path = os.path.join(os.path.dirname(_HERE), "include", "rpb200.h")
    with open(path) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(rp_[a-z0-9_]+)\s*\(", text)))


def load():
    """Load the library (no GPU needed to load) and declare all signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C reapers_b200/csrc`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc):
    if rc != 0:
        raise RPError(rc, load().rp_last_error().decode())
    return rc


def call(name, *args):
    return check(getattr(load(), name)(*args))
