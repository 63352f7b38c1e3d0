"""Edges of the restarted Krylov evolve (Krylov<Impl>::evolve,
inc/algo.h:267-365) against the oracle, FP64: the smallest and largest basis
sizes, a start vector that is an eigenvector (breakdown on the first basis
vector), an empty Hamiltonian, and pure imaginary time.  FP64: the final
state within 1e-12 relative; restart, H.psi, pass and inner-product counts
and the breakdown flag identical.  Mixed path (complex64 vectors, FP64
Krylov internals): within 1e-5 relative of the FP64 oracle."""
import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L = 10
KEYS = ("restarts", "applies", "passes", "prods", "breakdown")


def _start():
    rng = np.random.default_rng(11)
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    return v / np.linalg.norm(v)


def _run(bits, coeff, v, t, beta, m):
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    st = rb.evolve(ham, x, t, beta, m, 1e-12)
    got = x.cpu().numpy()
    ham.close()
    ref, st2 = O.evolve(L, bits, coeff, v, t, beta, m, 1e-12)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err
    for k in KEYS:
        assert st[k] == st2[k], (k, st, st2)
    return got, st


@pytest.mark.parametrize("m", [2, 64])
def test_smallest_and_largest_basis(cuda, m):
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=10)
    _run(bits, coeff, _start(), 1.0, 0.0, m)


def test_eigenvector_start_breaks_down_at_once(cuda):
    """Z fields only and a basis state: H psi is parallel to psi, the basis
    stops at one vector and the result is the phase exp(-i t E)."""
    h = np.linspace(-1.0, 1.0, L)
    bits = np.array([1 << (2 * i + 1) for i in range(L)], dtype=np.uint64)
    e = np.zeros(1 << L, dtype=np.complex128)
    e[5] = 1.0
    got, st = _run(bits, h.astype(np.complex128), e, 0.9, 0.0, 6)
    assert st["breakdown"] == 1 and st["applies"] == 1
    E = sum(h[i] * (-1.0 if (5 >> i) & 1 else 1.0) for i in range(L))
    assert abs(got[5] - np.exp(-0.9j * E)) < 1e-14
    assert np.count_nonzero(got) == 1


def test_empty_hamiltonian_leaves_the_state(cuda):
    v = _start()
    got, st = _run(np.zeros(0, np.uint64), np.zeros(0, np.complex128), v, 0.9, 0.0, 6)
    assert st["breakdown"] == 1
    assert np.array_equal(got, v)


def test_pure_imaginary_time(cuda):
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=10)
    got, _ = _run(bits, coeff, _start(), 0.0, 0.7, 8)
    assert np.linalg.norm(got) > 1.0      # exp(-beta H) is not unitary


def _run_mixed(bits, coeff, v, t, beta, m):
    """The mixed path (complex64 vectors, FP64 Krylov internals) against the
    FP64 oracle, to the path's FP32 tolerance."""
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    x = torch.from_numpy(np.ascontiguousarray(v)).to(torch.complex64).cuda()
    st = rb.evolve(ham, x, t, beta, m, float(np.finfo(np.float32).eps))
    got = x.cpu().numpy().astype(np.complex128)
    ham.close()
    ref, _ = O.evolve(L, bits, coeff, v.astype(np.complex64).astype(np.complex128), t, beta, m,
                      1e-12)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
    return got, st


@pytest.mark.parametrize("m", [2, 64])
def test_mixed_smallest_and_largest_basis(cuda, m):
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=10)
    _run_mixed(bits, coeff, _start(), 1.0, 0.0, m)


def test_mixed_empty_hamiltonian_and_imaginary_time(cuda):
    v = _start()
    got, st = _run_mixed(np.zeros(0, np.uint64), np.zeros(0, np.complex128), v, 0.9, 0.0, 6)
    assert st["breakdown"] == 1
    assert np.array_equal(got, v.astype(np.complex64).astype(np.complex128))
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=10)
    _run_mixed(bits, coeff, v, 0.0, 0.7, 8)
