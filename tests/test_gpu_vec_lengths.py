"""BLAS-1 entry points (GPUImpl's zero / copy / add / axpy / scale / vec_prod /
vec_norm, inc/gpuimpl.h:853-1002) on ragged lengths: one element, odd
counts (complex64 vectors of odd length leave the 16-byte packet path),
lengths that are no multiple of a block, and an empty vector.

Tolerances: inner products and norms accumulate in FP64 with compensation,
within 1e-12 relative of numpy on the same (upcast) inputs in both
precisions; axpy and scale compute in FP64 and round once, within 1e-6
relative in complex64 and 1e-14 in complex128; add and precision
conversion are exact (bit-identical to numpy's rounding).
"""
import ctypes as C

import numpy as np
import pytest
import torch

import reapers_b200 as rb
from reapers_b200 import _lib

pytestmark = pytest.mark.gpu

LENGTHS = [1, 3, 255, 257, 4097, 100003, (1 << 20) + 1]
TDT = {"c64": torch.complex64, "c128": torch.complex128}
NDT = {"c64": np.complex64, "c128": np.complex128}


def _vec(rng, n, dtype):
    v = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(NDT[dtype])
    return v, torch.from_numpy(v).cuda()


def _host(t):
    rb.synchronize()
    return t.cpu().numpy()


def _rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("n", LENGTHS)
def test_reductions_on_ragged_lengths(cuda, dtype, n):
    rng = np.random.default_rng(n)
    a, ta = _vec(rng, n, dtype)
    b, tb = _vec(rng, n, dtype)
    ref = np.vdot(a.astype(np.complex128), b.astype(np.complex128))
    got = rb.dot(ta, tb)
    assert abs(got - ref) <= 1e-12 * abs(ref) + 1e-300, (n, got, ref)
    nrm = np.linalg.norm(a.astype(np.complex128))
    assert abs(rb.norm(ta) - nrm) <= 1e-12 * nrm


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("n", LENGTHS)
def test_elementwise_on_ragged_lengths(cuda, dtype, n):
    rng = np.random.default_rng(1000 + n)
    a, ta = _vec(rng, n, dtype)
    b, tb = _vec(rng, n, dtype)
    tol = 1e-6 if dtype == "c64" else 1e-14
    c = 0.75 - 0.5j
    rb.axpy(ta, c, tb)
    ref = a.astype(np.complex128) + c * b.astype(np.complex128)
    assert _rel(_host(ta), ref) < tol
    a2 = _host(ta).astype(np.complex128)
    rb.scale(ta, 2.5j)
    assert _rel(_host(ta), 2.5j * a2) < tol
    code = rb.dtype_code(dtype)
    tr = torch.empty_like(ta)
    _lib.call("rp_vec_add", code, n, C.c_void_p(tr.data_ptr()), C.c_void_p(ta.data_ptr()),
              C.c_void_p(tb.data_ptr()))
    assert np.array_equal(_host(tr), _host(ta) + b)
    _lib.call("rp_vec_zero", code, n, C.c_void_p(tr.data_ptr()))
    assert not np.any(_host(tr))


@pytest.mark.parametrize("n", LENGTHS)
def test_precision_conversion_on_ragged_lengths(cuda, n):
    rng = np.random.default_rng(2000 + n)
    d, td = _vec(rng, n, "c128")
    f = torch.empty(n, dtype=torch.complex64, device="cuda")
    rb.copy(f, td)
    assert np.array_equal(_host(f), d.astype(np.complex64))     # round to nearest
    back = torch.empty(n, dtype=torch.complex128, device="cuda")
    rb.copy(back, f)
    assert np.array_equal(_host(back), d.astype(np.complex64).astype(np.complex128))


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_empty_vectors(cuda, dtype):
    """n = 0 with valid pointers: the inner product and norm are zero and
    the element-wise calls touch nothing."""
    code = rb.dtype_code(dtype)
    t = torch.ones(4, dtype=TDT[dtype], device="cuda")
    p = C.c_void_p(t.data_ptr())
    out = (C.c_double * 2)(7.0, 7.0)
    _lib.call("rp_vec_dot", code, 0, p, p, out)
    assert (out[0], out[1]) == (0.0, 0.0)
    nrm = C.c_double(7.0)
    _lib.call("rp_vec_norm", code, 0, p, C.byref(nrm))
    assert nrm.value == 0.0
    _lib.call("rp_vec_axpy", code, 0, p, 1.0, 0.0, p)
    _lib.call("rp_vec_scale", code, 0, p, 0.0, 0.0)
    _lib.call("rp_vec_zero", code, 0, p)
    assert np.array_equal(_host(t), np.ones(4))


def test_misaligned_vectors_are_refused(cuda):
    """A vector starting off a 16-byte boundary is refused on the host, before
    any launch (the kernels read 16-byte packets)."""
    t = torch.zeros(64, dtype=torch.complex64, device="cuda")
    out = (C.c_double * 2)()
    with pytest.raises(rb.RPError, match="16-byte aligned"):
        _lib.call("rp_vec_dot", 1, 8, C.c_void_p(t.data_ptr() + 8), C.c_void_p(t.data_ptr()), out)
