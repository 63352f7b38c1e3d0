"""The fused diagonal of the row kernel, restated on the CPU.

For real Z strings (X mask 0) the kernel replaces sum_t c_t
(-1)^popc(z_t & i) at element i = (hi << logC) | e by bucket sums over the
strings' in-row Z bits b = z_t & (C - 1), a_b = sum c_t (-1)^popc(zhi_t & hi),
followed by a Walsh-Hadamard transform over the in-row bits,
d(e) = sum_b a_b (-1)^popc(b & e).  This checks that identity for both row
widths (16 complex64 or 8 complex128 elements per 128-byte row) against the
direct sum, on every element of a small state, with the same in-place
butterfly order as the kernel.
"""
import numpy as np
import pytest


def _direct(z, c, n):
    i = np.arange(n, dtype=np.uint64)
    par = np.bitwise_count(i[:, None] & z[None, :].astype(np.uint64)) & 1
    return (np.where(par.astype(bool), -c[None, :], c[None, :])).sum(axis=1)


def _fused(z, c, n, logC):
    C = 1 << logC
    zhi = z >> logC
    out = np.zeros(n)
    for hi in range(n >> logC):
        a = np.zeros(C)
        for b in range(C):
            sel = (z & (C - 1)) == b
            s = (np.bitwise_count(zhi[sel].astype(np.uint64) & np.uint64(hi)) & 1).astype(bool)
            a[b] = np.where(s, -c[sel], c[sel]).sum()
        h = 1
        while h < C:                       # the kernel's in-place butterflies
            for e in range(C):
                if not e & h:
                    u, v = a[e], a[e | h]
                    a[e], a[e | h] = u + v, u - v
            h <<= 1
        out[hi * C:(hi + 1) * C] = a
    return out


@pytest.mark.parametrize("logC", [4, 3])
def test_bucket_sums_and_walsh_hadamard_give_the_diagonal(logC):
    rng = np.random.default_rng(logC)
    L = 10
    n = 1 << L
    # fields, couplings, and random Z strings over in-row and high bits
    z = [1 << i for i in range(L)] + [(1 << i) | (1 << (i + 1)) for i in range(L - 1)]
    z += list(rng.integers(1, n, 20))
    z = np.array(z, dtype=np.int64)
    c = rng.uniform(-1, 1, len(z))
    np.testing.assert_allclose(_fused(z, c, n, logC), _direct(z, c, n), rtol=0, atol=1e-12)
