"""Parity at the full sizes, where the CPU oracle cannot apply the whole
operator, through properties that do not depend on the size:

* sampled output rows (4096 random indices plus the first and last) against
  the oracle's index-sampled apply (oracle.apply_at, the same sum as the C
  restatement, pinned against it in tests/test_oracle_cpu.py);
* Hermiticity of the SYK Hamiltonian: <a|H b> = conj(<b|H a>);
* linearity: H(a + s b) = H a + s H b;
* the restarted Krylov evolve: unitarity and time reversal.

Sizes: the N = 56 sparse SYK of the headline (28 qubits, 448 terms, the
bench's seeded terms) in FP32 and FP64, and the longest chains the library
accepts, 31 and 32 qubits (16 and 32 GB complex64 states).
"""
import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def _spot_relerr(bits, coeff, x, y, L, rng, n=4096):
    """||y - H x|| / ||H x|| over sampled rows, H x from the oracle."""
    idx = np.unique(np.concatenate([[0, (1 << L) - 1], rng.integers(0, 1 << L, n)]))

    def fetch(j):
        return x[torch.from_numpy(j).to(x.device)].cpu().numpy().astype(np.complex128)

    ref = O.apply_at(bits, coeff, idx, fetch)
    got = y[torch.from_numpy(idx.astype(np.int64)).to(y.device)].cpu().numpy().astype(np.complex128)
    return np.linalg.norm(got - ref) / np.linalg.norm(ref)


def _release(*objs):
    for o in objs:
        if hasattr(o, "close"):
            o.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dtype", ["c64", "c128"])
def test_syk_n56_rows_hermiticity_linearity(cuda, dtype):
    L, N = 28, 56
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=1000)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    assert ham.info()["kernel"] == 2
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    rng = np.random.default_rng(56)
    a = rb.random_state(L, dtype, seed=1)
    b = rb.random_state(L, dtype, seed=2)
    ha, hb = torch.empty_like(a), torch.empty_like(b)
    ham.apply(ha, a)
    ham.apply(hb, b)
    assert _spot_relerr(bits, coeff, a, ha, L, rng) < tol
    assert _spot_relerr(bits, coeff, b, hb, L, rng) < tol
    x = rb.dot(a, hb)
    y = rb.dot(b, ha)
    scale = rb.norm(ha) * rb.norm(b)
    assert abs(x - y.conjugate()) <= tol * scale, (x, y)
    s = 0.75 - 1.25j
    c = a.clone()
    rb.axpy(c, s, b)
    hc = torch.empty_like(c)
    ham.apply(hc, c)
    rb.axpy(ha, s, hb)          # ha <- H a + s H b
    rb.axpy(hc, -1.0, ha)
    assert rb.norm(hc) <= tol * rb.norm(ha) * 4
    del a, b, c, ha, hb, hc
    _release(ham)


def test_syk_n56_mixed_evolve_unitarity_and_time_reversal(cuda):
    L, N = 28, 56
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=1000)
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    eps = float(np.finfo(np.float32).eps)
    psi0 = rb.random_state(L, "c64", seed=5)
    psi = psi0.clone()
    st = rb.evolve(ham, psi, 0.25, 0.0, 16, eps)
    assert st["applies"] >= 16
    assert abs(rb.norm(psi) - 1.0) <= 1e-5
    # exp(-iHt) moved the state: it is not the identity on it
    moved = psi.clone()
    rb.axpy(moved, -1.0, psi0)
    assert rb.norm(moved) > 1e-3
    rb.evolve(ham, psi, -0.25, 0.0, 16, eps)
    rb.axpy(psi, -1.0, psi0)
    assert rb.norm(psi) <= 1e-4
    del psi0, psi, moved
    _release(ham)


@pytest.mark.parametrize("L", [31, 32])
def test_longest_chains(cuda, L):
    """The largest states the library accepts: sampled rows against the
    oracle and, at 31 qubits, Hermiticity."""
    N = 2 * L
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=L)
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    assert ham.info()["kernel"] == 2
    rng = np.random.default_rng(L)
    a = rb.random_state(L, "c64", seed=11)
    ha = torch.empty_like(a)
    ham.apply(ha, a)
    assert _spot_relerr(bits, coeff, a, ha, L, rng, n=2048) < FP32_TOL
    if L == 31:
        b = rb.random_state(L, "c64", seed=12)
        hb = torch.empty_like(b)
        ham.apply(hb, b)
        x = rb.dot(a, hb)
        y = rb.dot(b, ha)
        assert abs(x - y.conjugate()) <= FP32_TOL * rb.norm(ha) * rb.norm(b)
        del b, hb
    del a, ha
    _release(ham)
