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


def _header_prototypes():
    """name -> (return type, [parameter declarations]) from include/rpb200.h."""
    import pathlib
    import re
    h = (pathlib.Path(__file__).resolve().parents[1] / "include" / "rpb200.h").read_text()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    h = re.sub(r"//[^\n]*", "", h)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w\s]*?\**)\s*\b(rp_\w+)\s*\(([^;{}()]*)\)\s*;", h):
        ps = [p.strip() for p in m.group(3).split(",") if p.strip() not in ("", "void")]
        out[m.group(2)] = (m.group(1).split("\n")[-1].strip(), ps)
    return out


def _c_class(decl):
    import re
    if "*" in decl or re.search(r"\brp_(ham|dense|mlp|batch)_t\b", decl):
        return "ptr"
    ty = re.sub(r"\s*\b\w+$", "", decl.strip())      # drop the parameter name
    for cls, pat in (("f64", r"\bdouble\b"), ("f32", r"\bfloat\b"),
                     ("i64", r"\b(u?int64_t|size_t)\b"), ("i32", r"\b(int|u?int32_t)\b")):
        if re.search(pat, ty):
            return cls
    return "other:" + decl


def _py_class(a):
    if a in (C.c_void_p, C.c_char_p) or (isinstance(a, type) and issubclass(a, C._Pointer)):
        return "ptr"
    for cls, types in (("f64", (C.c_double,)), ("f32", (C.c_float,)),
                       ("i64", (C.c_uint64, C.c_int64, C.c_size_t, C.c_ssize_t)),
                       ("i32", (C.c_int, C.c_uint32, C.c_int32))):
        if a in types:
            return cls
    return "other:" + repr(a)


def test_binding_signatures_match_the_header():
    """Every prototype's parameters agree in number, order and kind (pointer,
    64-bit integer, 32-bit integer, double, float) with the Python binding,
    and its return type with the binding's restype: a drift between the two
    would pass wrong-width arguments without any error."""
    protos = _header_prototypes()
    assert sorted(protos) == sorted(_lib._SIGS)
    bad = []
    for name, (ret, params) in protos.items():
        res, args = _lib._SIGS[name]
        if [_c_class(p) for p in params] != [_py_class(a) for a in args]:
            bad.append((name, params, args))
        want = {"int": C.c_int, "const char *": C.c_char_p, "void *": C.c_void_p}[
            " ".join(ret.replace("*", " * ").split()).replace(" *", " *")]
        if res is not want:
            bad.append((name, ret, res))
    assert not bad, bad
