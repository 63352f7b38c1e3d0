"""GPU results against golden fixtures made by the reference library itself
(tests/golden/make_golden.py): FP64 within 1e-12 relative, operation counts
exact."""
import os

import numpy as np
import pytest
import torch

import reapers_b200 as rb

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


def dev(v):
    return torch.from_numpy(np.ascontiguousarray(v)).cuda()


def test_apply_reference_fixture(cuda):
    g = gold("apply_L10.npz")
    L = int(g["len"])
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    out = torch.empty(1 << L, dtype=torch.complex128, device=cuda)
    ham.apply(out, dev(g["vec"]))
    o = out.cpu().numpy()
    assert np.linalg.norm(o - g["out"]) / np.linalg.norm(g["out"]) < 1e-13


def test_dense_syk_n24_evolve_reference_fixture(cuda):
    """Dense SYK N = 24 (12 qubits, all 10626 quartets from the
    reference's SYK::gen_ham), m = 20, tol 1e-12, t = 0.5, 2.5, 5.0."""
    g = gold("dense_syk_N24.npz")
    L = int(g["len"])
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    for k, t in enumerate(g["times"]):
        x = dev(g["psi0"])
        st = rb.evolve(ham, x, float(t), 0.0, int(g["krydim"]), float(g["tol"]))
        o = x.cpu().numpy()
        assert np.linalg.norm(o - g["out"][k]) / np.linalg.norm(g["out"][k]) < 1e-12
        assert st["applies"] == g["applies"][k]
        assert st["prods"] == g["prods"][k]


def test_imaginary_time_evolve_reference_fixture(cuda):
    g = gold("evolve_sparse_N20.npz")
    L = int(g["len"])
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    x = dev(g["psi0"])
    st = rb.evolve(ham, x, float(g["t"]), float(g["beta"]), int(g["krydim"]), float(g["tol"]))
    o = x.cpu().numpy()
    assert np.linalg.norm(o - g["out"]) / np.linalg.norm(g["out"]) < 1e-12
    assert st["applies"] == int(g["applies"]) and st["prods"] == int(g["prods"])


def test_otoc_reference_fixture(cuda):
    g = gold("otoc_N16.npz")
    L = int(g["len"])
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    w = rb.Hamiltonian(L, g["w_bits"], g["w_coeff"], "c128")
    v = rb.Hamiltonian(L, g["v_bits"], g["v_coeff"], "c128")
    vals, applies = rb.otoc(ham, w, v, dev(g["psi0"]), g["times"], int(g["krydim"]),
                            float(g["tol"]))
    assert np.abs(vals - g["F"]).max() < 1e-12
    # the reference counts the four single-string products per point too
    # (State::operator*= goes through Impl::apply_ops)
    assert applies + 4 * len(g["times"]) == int(g["applies"])


def test_parity_block_otoc_reference_fixture(cuda):
    """The parity-block OTOC of examples/syk.cc (one block of N/2 - 1 = 5
    qubits, dense SYK N = 12 from the reference's generator, op = LR block of
    b_{N-2}) against the reference's own values (FP64, <= 1e-12)."""
    import reapers_b200 as rb
    g = np.load(os.path.join(GOLD, "syk_block_N12.npz"))
    L = int(g["len"])
    ll = rb.Hamiltonian(L, g["ll_bits"], g["ll_coeff"], "c128")
    rr = rb.Hamiltonian(L, g["rr_bits"], g["rr_coeff"], "c128")
    op = rb.Hamiltonian(L, g["op_bits"], g["op_coeff"], "c128")
    psi0 = torch.from_numpy(g["psi0"]).cuda()
    F, applies = rb.otoc_block(ll, rr, op, psi0, g["times"], int(g["krydim"]), float(g["tol"]))
    assert np.abs(F - g["F"]).max() <= 1e-12 * abs(g["F"][0]), (F, g["F"])
    assert applies > 0
