"""Term lists that repeat a Pauli string (the same X and Z masks with
different coefficients, in any order), given straight to Hamiltonian: the
reference's SumOps merges such terms on construction, a caller of the C ABI
need not.  Every kernel (direct, bulk-copy tiled, TMA row kernel with and
without the fused diagonal) must apply the sum, as the oracle does in list
order.  Tolerances: 1e-12 relative in FP64, 1e-5 in FP32."""
import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-12, "c64": 1e-5}


def _with_repeats(rng, bits, coeff, frac=0.4):
    k = max(1, int(frac * len(bits)))
    pick = rng.choice(len(bits), size=k, replace=False)
    extra_c = rng.standard_normal(k) * np.abs(coeff[pick]).max()
    # real Z strings keep real coefficients so the fused diagonal still sees them
    extra_c = np.where(coeff[pick].imag == 0, extra_c, extra_c * 1j)
    b = np.concatenate([bits, bits[pick]])
    c = np.concatenate([coeff, extra_c.astype(np.complex128)])
    order = rng.permutation(len(b))
    return b[order], c[order]


def _check(L, bits, coeff, dtype, rng, kernel=None):
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    if kernel is not None:
        assert ham.info()["kernel"] == kernel, ham.info()
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    x = torch.from_numpy(v).to(torch.complex64 if dtype == "c64" else torch.complex128).cuda()
    out = torch.empty_like(x)
    ham.apply(out, x)
    vin = x.cpu().numpy().astype(np.complex128)
    ref = O.apply(L, bits, coeff, vin)
    got = out.cpu().numpy().astype(np.complex128)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    ham.close()
    return err


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("L", [8, 14, 20])
def test_repeated_syk_terms(cuda, dtype, L):
    rng = np.random.default_rng(300 + L)
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=L)
    bits, coeff = _with_repeats(rng, bits, coeff)
    assert len(np.unique(bits)) < len(bits)
    assert _check(L, bits, coeff, dtype, rng) < TOL[dtype]


@pytest.mark.parametrize("dtype,L", [("c64", 19), ("c128", 18)])
def test_repeated_diagonal_terms_on_the_fused_path(cuda, dtype, L):
    """Repeated real Z strings are summed into the per-row diagonal factor."""
    rng = np.random.default_rng(L)
    bits, coeff = rb.syk.xxz_chain(L, 0.8, rng.uniform(-1, 1, L), periodic=True)
    bits, coeff = _with_repeats(rng, bits, coeff, frac=0.6)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    assert ham.info()["diag_terms"] >= 4
    ham.close()
    assert _check(L, bits, coeff, dtype, rng, kernel=2) < TOL[dtype]


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_cancelling_terms(cuda, dtype):
    """A string added with c and with -c contributes nothing."""
    L = 19
    rng = np.random.default_rng(5)
    bits, coeff = rb.syk.sparse_syk(2 * L, k=4, seed=7)
    b2 = np.concatenate([bits, bits[:5]])
    c2 = np.concatenate([coeff, -coeff[:5]])
    ham = rb.Hamiltonian(L, b2, c2, dtype)
    kept = rb.Hamiltonian(L, bits[5:], coeff[5:], dtype)
    x = rb.random_state(L, dtype, seed=3)
    out, ref = torch.empty_like(x), torch.empty_like(x)
    ham.apply(out, x)
    kept.apply(ref, x)
    rb.synchronize()
    a, b = out.cpu().numpy().astype(np.complex128), ref.cpu().numpy().astype(np.complex128)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < TOL[dtype]
    ham.close()
    kept.close()
