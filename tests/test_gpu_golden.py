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


def test_dense_syk_n24_evolve_all_ten_points(cuda):
    """The dense SYK N = 24 workload at all ten time points t = 0.5 .. 5.0
    (m = 20, tol 1e-12) against the reference's own FP64 State::evolve:
    final states within 1e-12, H.psi and inner-product counts identical."""
    g = gold("dense_syk_N24_t10.npz")
    L = int(g["len"])
    assert len(g["times"]) == 10
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    for k, t in enumerate(g["times"]):
        x = dev(g["psi0"])
        st = rb.evolve(ham, x, float(t), 0.0, int(g["krydim"]), float(g["tol"]))
        o = x.cpu().numpy()
        assert np.linalg.norm(o - g["out"][k]) / np.linalg.norm(g["out"][k]) < 1e-12, t
        assert st["applies"] == g["applies"][k], t
        assert st["prods"] == g["prods"][k], t


def _n40_problem():
    """Regenerates the evolve_sparse_N40 problem from its seeds (the same code
    as tests/golden/make_golden.py:n40_problem, restated here so that the
    GPU tests need no fixture script)."""
    g = gold("evolve_sparse_N40.npz")
    L = int(g["len"])
    s_ham, s_psi, s_probe = (int(v) for v in g["seeds"])
    bits, coeff = rb.syk.sparse_syk(40, k=8, seed=s_ham)
    assert np.array_equal(bits, g["bits"]) and np.array_equal(coeff, g["coeff"])
    rng = np.random.default_rng(s_psi)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    prng = np.random.default_rng(s_probe)
    probes = prng.standard_normal((8, 1 << L)) + 1j * prng.standard_normal((8, 1 << L))
    return g, L, psi, probes


def test_sparse_syk_n40_evolve_t10_reference_fixture(cuda):
    """Evolve parity at size: 20 qubits (sparse SYK N = 40, k = 8, 320 terms),
    t = 10, m = 30, tol = FP64 epsilon, the reference's own FP64
    State::evolve as the oracle.  The FP64 GPU evolve matches it within 1e-12
    on 4096 sampled entries and on 8 projections of the whole state (a
    checksum), with identical H.psi and inner-product counts; the mixed path
    (FP32 vectors and H.psi, FP64 Krylov internals, tol = FP32 epsilon) is
    within 1e-5 of it (its error is printed)."""
    g, L, psi, probes = _n40_problem()
    ham = rb.Hamiltonian(L, g["bits"], g["coeff"], "c128")
    x = dev(psi)
    st = rb.evolve(ham, x, float(g["t"]), 0.0, int(g["krydim"]), float(g["tol"]))
    o = x.cpu().numpy()
    idx = g["idx"]
    assert np.linalg.norm(o[idx] - g["vals"]) / np.linalg.norm(g["vals"]) < 1e-12
    assert abs(np.linalg.norm(o) - float(g["norm"])) < 1e-12
    proj = probes.conj() @ o
    assert np.abs(proj - g["proj"]).max() < 1e-12 * np.abs(g["proj"]).max() * 10
    assert st["applies"] == int(g["applies"]) and st["prods"] == int(g["prods"])
    ham.close()
    # the mixed path on the same problem, against the reference's FP64 result
    hm = rb.Hamiltonian(L, g["bits"], g["coeff"], "c64")
    xm = torch.empty(1 << L, dtype=torch.complex64, device=cuda)
    rb.copy(xm, dev(psi))
    rb.evolve(hm, xm, float(g["t"]), 0.0, int(g["krydim"]), float(np.finfo(np.float32).eps))
    om = xm.cpu().numpy().astype(np.complex128)
    err_rows = np.linalg.norm(om[idx] - g["vals"]) / np.linalg.norm(g["vals"])
    err_proj = np.abs(probes.conj() @ om - g["proj"]).max() / np.abs(g["proj"]).max()
    print(f"mixed vs reference FP64 at 20 qubits, t = 10: rows {err_rows:.2e}, "
          f"projections {err_proj:.2e}")
    assert err_rows < 1e-5 and err_proj < 1e-5
    hm.close()


def test_sparse_syk_n48_evolve_t10_reference_fixture(cuda):
    """Evolve parity on the sparse SYK N = 48 evolve workload itself (24
    qubits, k = 8, 384 terms, t = 10, m = 30, tol = FP64 epsilon) against the
    reference's own FP64 State::evolve: within 1e-12 on 4096 sampled entries
    and on 4 projections of the whole state onto seeded random vectors,
    identical H.psi and inner-product counts; the mixed path's error against
    it is printed and bounded by 1e-5."""
    path = os.path.join(GOLD, "evolve_sparse_N48.npz")
    if not os.path.exists(path):
        pytest.skip("evolve_sparse_N48.npz not generated")
    g = np.load(path)
    L = int(g["len"])
    s_ham, s_psi, s_probe = (int(v) for v in g["seeds"])
    bits, coeff = rb.syk.sparse_syk(48, k=8, seed=s_ham)
    assert np.array_equal(bits, g["bits"]) and np.array_equal(coeff, g["coeff"])
    rng = np.random.default_rng(s_psi)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)

    def projections(x):
        prng = np.random.default_rng(s_probe)
        prng.integers(0, 1 << L, size=4096)     # the sampled indices come first
        out = []
        for _ in range(len(g["proj"])):
            r = prng.standard_normal(1 << L) + 1j * prng.standard_normal(1 << L)
            out.append(np.vdot(r, x))
        return np.array(out)

    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = dev(psi)
    st = rb.evolve(ham, x, float(g["t"]), 0.0, int(g["krydim"]), float(g["tol"]))
    o = x.cpu().numpy()
    idx = g["idx"]
    assert np.linalg.norm(o[idx] - g["vals"]) / np.linalg.norm(g["vals"]) < 1e-12
    assert abs(np.linalg.norm(o) - float(g["norm"])) < 1e-12
    assert np.abs(projections(o) - g["proj"]).max() < 1e-11 * np.abs(g["proj"]).max()
    assert st["applies"] == int(g["applies"]) and st["prods"] == int(g["prods"])
    ham.close()
    hm = rb.Hamiltonian(L, bits, coeff, "c64")
    xm = torch.empty(1 << L, dtype=torch.complex64, device=cuda)
    rb.copy(xm, dev(psi))
    rb.evolve(hm, xm, float(g["t"]), 0.0, int(g["krydim"]), float(np.finfo(np.float32).eps))
    om = xm.cpu().numpy().astype(np.complex128)
    err_rows = np.linalg.norm(om[idx] - g["vals"]) / np.linalg.norm(g["vals"])
    err_proj = np.abs(projections(om) - g["proj"]).max() / np.abs(g["proj"]).max()
    print(f"mixed vs reference FP64 at 24 qubits, t = 10: rows {err_rows:.2e}, "
          f"projections {err_proj:.2e}")
    assert err_rows < 1e-5 and err_proj < 1e-5
    hm.close()
