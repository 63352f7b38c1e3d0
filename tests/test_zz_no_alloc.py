"""rp_vec_dot_noalloc: the inner product for callers that cannot let the
library allocate device memory (it keeps its scratch in a fixed device array).

Checked through the C ABI against rp_vec_dot, the allocating entry point, on
two calls in a row -- the second shorter than the first, so partial sums left
in the shared scratch array by the first call must not leak into the second.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # relative; both entry points accumulate in FP64 with compensation


def _dot(lib, name, dtype, n, a, b):
    out = (C.c_double * 2)()
    rc = getattr(lib, name)(dtype, n, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), out)
    assert rc == 0, lib.rp_last_error().decode()
    return complex(out[0], out[1])


@pytest.mark.parametrize("dtype_name", ["c128", "c64"])
def test_noalloc_dot_matches_allocating_dot_twice(dtype_name):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import reapers_b200 as rb
    from reapers_b200 import _lib
    rb.init(0)
    lib = _lib.load()
    code = rb.dtype_code(dtype_name)
    tdt = torch.complex128 if dtype_name == "c128" else torch.complex64
    rng = np.random.default_rng(17)
    for n in ((3 << 18) + 5, 1000):   # several scratch blocks, then one
        a = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to(tdt).cuda()
        b = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).to(tdt).cuda()
        ref = _dot(lib, "rp_vec_dot", code, n, a, b)
        got = _dot(lib, "rp_vec_dot_noalloc", code, n, a, b)
        assert abs(got - ref) <= TOL * abs(ref), (n, got, ref)
        direct = np.vdot(a.cpu().numpy().astype(np.complex128), b.cpu().numpy().astype(np.complex128))
        assert abs(got - direct) <= 1e-9 * abs(direct)


def test_noalloc_dot_rejects_too_long_vectors():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import reapers_b200 as rb
    from reapers_b200 import _lib
    rb.init(0)
    lib = _lib.load()
    a = torch.zeros(16, dtype=torch.complex128, device="cuda")
    out = (C.c_double * 2)()
    # the length check comes before any launch, so no memory is touched
    rc = lib.rp_vec_dot_noalloc(2, (1 << 28) + 1, C.c_void_p(a.data_ptr()),
                                C.c_void_p(a.data_ptr()), out)
    assert rc == -2
    assert b"exceeds the fixed scratch limit" in lib.rp_last_error()


def test_noalloc_dot_rejects_misaligned_vectors():
    """A vector that starts off a 16-byte boundary is refused before any
    launch, as by every other vector entry point."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import reapers_b200 as rb
    from reapers_b200 import _lib
    rb.init(0)
    lib = _lib.load()
    a = torch.zeros(64, dtype=torch.complex64, device="cuda")
    out = (C.c_double * 2)()
    rc = lib.rp_vec_dot_noalloc(1, 8, C.c_void_p(a.data_ptr() + 8), C.c_void_p(a.data_ptr()), out)
    assert rc == -2
    assert b"16-byte aligned" in lib.rp_last_error()
