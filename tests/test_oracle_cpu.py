"""CPU checks: the oracle (oracle/rp_oracle.c) against the reference's own
unit-test known answers (tests/ops.cc of the reference) and against golden
fixtures made by running the reference library itself
(tests/golden/make_golden.py); the product's host-side term generator
(reapers_b200/syk.py) against both."""
import math
import os

import numpy as np
import pytest

import reapers_b200.syk as S
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = np.finfo(float).eps * 1e2   # the reference's unit-test tolerance (tests/ops.cc:23)

I2 = np.eye(2)
SX = np.array([[0, 1], [1, 0]], complex)
SY = np.array([[0, -1j], [1j, 0]], complex)
SZ = np.array([[1, 0], [0, -1]], complex)


def gold(name):
    return np.load(os.path.join(GOLD, name))


def op(kind, site):
    b, c = S.sigma(kind, site)
    return int(b), complex(c)


# --- reference known answers (tests/ops.cc) ---------------------------------

def test_single_site_products():
    """tests/ops.cc:26-44: sx*sy = i sz, sz*sx = i sy, ... through the
    oracle's product rule (bits and the carry-over sign)."""
    i = 1j
    table = {("x", "y"): ("z", i), ("x", "z"): ("y", -i), ("y", "x"): ("z", -i),
             ("y", "z"): ("x", i), ("z", "x"): ("y", i), ("z", "y"): ("x", -i)}
    for (a, b), (r, f) in table.items():
        ba, ca = op(a, 0)
        bb, cb = op(b, 0)
        bo, co = O.spin_mul(ba, ca, bb, cb)
        br, cr = op(r, 0)
        assert bo == br and abs(co - f * cr) < TOL
    for a in "xyz":
        ba, ca = op(a, 0)
        bo, co = O.spin_mul(ba, ca, ba, ca)
        assert bo == 0 and abs(co - 1) < TOL


def test_matrix_representation():
    """tests/ops.cc:46-161: dense matrices of 1- and 2-site strings pin the
    bit encoding and the index order (site 1 is the high bit)."""
    mats = {"x": SX, "y": SY, "z": SZ}
    for k, m in mats.items():
        b, c = op(k, 0)
        M = O.dense_matrix(1, np.array([b], np.uint64), np.array([c]))
        assert np.abs(M - m).max() < TOL
    for k1, m1 in list(mats.items()) + [("i", I2)]:
        for k0, m0 in list(mats.items()) + [("i", I2)]:
            b, c = 0, 1 + 0j
            if k1 != "i":
                b, c = O.spin_mul(b, c, *op(k1, 1))
            if k0 != "i":
                b, c = O.spin_mul(b, c, *op(k0, 0))
            M = O.dense_matrix(2, np.array([b], np.uint64), np.array([c]))
            assert np.abs(M - np.kron(m1, m0)).max() < TOL, (k1, k0)


def test_matrix_exponential_known_answers():
    """tests/ops.cc:198-229 (e, cosh 1, sinh 1, cos 1, sin 1) through the
    oracle's Pade-13 expm."""
    e, ch, sh, co, si = 2.71828182845905, 1.54308063481524, 1.17520119364380, \
        0.540302305868140, 0.841470984807897
    cases = [(I2, 1, [[e, 0], [0, e]]), (SX, 1, [[ch, sh], [sh, ch]]),
             (SY, 1, [[ch, -sh * 1j], [sh * 1j, ch]]), (SZ, 1, [[e, 0], [0, 0.367879441171442]]),
             (SX, 1j, [[co, si * 1j], [si * 1j, co]]), (SY, 1j, [[co, si], [-si, co]]),
             (SZ, 1j, [[co + si * 1j, 0], [0, co - si * 1j]])]
    for m, f, want in cases:
        assert np.abs(O.expm(f * m) - np.array(want)).max() < 1e-13


def test_expm_against_scipy():
    import scipy.linalg as sl
    rng = np.random.default_rng(0)
    for s in [1e-3, 0.1, 0.8, 2.0, 5.0, 40.0]:
        A = (rng.standard_normal((24, 24)) + 1j * rng.standard_normal((24, 24))) * s / 24
        E, E2 = O.expm(A), sl.expm(A)
        assert np.abs(E - E2).max() <= 1e-13 * np.abs(E2).max()


@pytest.mark.parametrize("N", range(4, 22, 2))
def test_majorana_anticommutators(N):
    """tests/ops.cc:299-346: {g_i, g_j} = delta_ij for the non-block form."""
    mb, mc = S.majoranas(N)
    for i in range(N):
        for j in range(N):
            b1, c1 = O.spin_mul(int(mb[i]), mc[i], int(mb[j]), mc[j])
            b2, c2 = O.spin_mul(int(mb[j]), mc[j], int(mb[i]), mc[i])
            assert b1 == b2
            s = c1 + c2
            if i == j:
                assert b1 == 0 and abs(s - 1) < TOL
            else:
                assert abs(s) < TOL


# --- golden fixtures made by the reference ----------------------------------

@pytest.mark.parametrize("N", range(4, 22, 2))
def test_majoranas_match_reference(N):
    g = gold(f"majorana_N{N}.npz")
    for n in range(N):
        bo, co = O.majorana(N, n)
        bp, cp = S.majorana(N, n)
        assert bo == int(g["bits"][n]) == int(bp)
        assert co == g["coeff"][n] == cp


def test_syk_terms_match_reference_generator():
    g = gold("syk_dense_N8_seed5.npz")
    q = S.all_quartets(8)
    ob, oc = O.syk_terms(8, q, np.ones(len(q)))
    assert np.array_equal(ob, g["bits"])
    J = (g["coeff"] / oc).real
    pb, pc = S.quartic_terms(8, q, J)
    assert np.array_equal(pb, g["bits"])
    assert np.abs(pc - g["coeff"]).max() < 1e-16
    assert abs(np.std(J / S.syk_scale(8)) - 1) < 0.3


def test_apply_matches_reference():
    g = gold("apply_L10.npz")
    out = O.apply(int(g["len"]), g["bits"], g["coeff"], g["vec"])
    assert np.linalg.norm(out - g["out"]) / np.linalg.norm(g["out"]) < 1e-14
    # the reference's HostSumOps round trip keeps the (unique) terms and order
    assert np.array_equal(g["rt_bits"], g["bits"])
    assert np.abs(g["rt_coeff"] - g["coeff"]).max() == 0


def test_dense_syk_n24_evolve_matches_reference():
    g = gold("dense_syk_N24.npz")
    L = int(g["len"])
    for k, t in enumerate(g["times"]):
        o, st = O.evolve(L, g["bits"], g["coeff"], g["psi0"], t, 0.0, int(g["krydim"]),
                         float(g["tol"]))
        assert np.linalg.norm(o - g["out"][k]) / np.linalg.norm(g["out"][k]) < 1e-12
        assert st["applies"] == g["applies"][k]
        assert st["prods"] == g["prods"][k]


def test_ten_point_fixture_agrees_with_the_oracle_pinned_one():
    """dense_syk_N24_t10.npz (all ten points of the dense SYK N = 24 workload)
    and dense_syk_N24.npz, whose points the oracle reproduces above, come from
    two builds of the reference driver: the same quartets and start state,
    couplings equal to 1e-12 relative (the two builds round the coupling
    scale's arithmetic differently), and at the shared times t = 0.5, 2.5,
    5.0 the same counts and states within 1e-13."""
    a, b = gold("dense_syk_N24.npz"), gold("dense_syk_N24_t10.npz")
    assert np.array_equal(a["bits"], b["bits"])
    assert np.all(np.abs(a["coeff"] - b["coeff"]) <= 1e-12 * np.abs(a["coeff"]))
    assert np.array_equal(a["psi0"], b["psi0"])
    assert np.allclose(b["times"], 0.5 * np.arange(1, 11))
    for k, t in enumerate(a["times"]):
        j = int(np.argmin(np.abs(b["times"] - t)))
        assert np.linalg.norm(a["out"][k] - b["out"][j]) < 1e-13
        assert a["applies"][k] == b["applies"][j] and a["prods"][k] == b["prods"][j]


def test_imaginary_time_evolve_matches_reference():
    g = gold("evolve_sparse_N20.npz")
    o, st = O.evolve(int(g["len"]), g["bits"], g["coeff"], g["psi0"], float(g["t"]),
                     float(g["beta"]), int(g["krydim"]), float(g["tol"]))
    assert np.linalg.norm(o - g["out"]) / np.linalg.norm(g["out"]) < 1e-12
    assert st["applies"] == int(g["applies"]) and st["prods"] == int(g["prods"])


def test_otoc_matches_reference():
    g = gold("otoc_N16.npz")
    vals = O.otoc(int(g["len"]), g["bits"], g["coeff"], (g["w_bits"], g["w_coeff"]),
                  (g["v_bits"], g["v_coeff"]), g["psi0"], g["times"], int(g["krydim"]),
                  float(g["tol"]))
    assert np.abs(vals - g["F"]).max() < 1e-12


def test_sparse_generator_draws_k_n_distinct_quartets():
    for N, k in [(20, 4), (32, 8), (48, 8)]:
        b, c = S.sparse_syk(N, k=k, seed=1)
        assert len(b) == k * N and len(np.unique(b)) == k * N
        # the reference's sparse normalisation: var = 6 J^2 / (N^3 p)
        assert math.isclose(S.syk_scale(N, k), O.syk_scale(N, k, 1.0), rel_tol=1e-15)


def test_xxz_chain_terms():
    b, c = S.xxz_chain(4, Jz=1.0, fields=[0.1, -0.2, 0.3, 0.0])
    assert len(b) == 3 * 3 + 4
    M = O.dense_matrix(4, b, c)
    assert np.abs(M - M.conj().T).max() < TOL   # Hermitian


# --- parity-block form (FermionOpBlockForm, inc/fermions.h:308-366) ---------
@pytest.mark.parametrize("N", [6, 8, 10, 12])
def test_block_majoranas_match_reference(N):
    import reapers_b200.syk as S
    g = gold(f"majorana_block_N{N}.npz")
    for n in range(N):
        (lb, lc), (rb_, rc) = S.majorana_block(N, n)
        assert int(g["bits"][2 * n]) == int(lb) and int(g["bits"][2 * n + 1]) == int(rb_)
        assert abs(g["coeff"][2 * n] - lc) < 1e-15 and abs(g["coeff"][2 * n + 1] - rc) < 1e-15


def test_block_hamiltonian_matches_reference_and_spectrum():
    """The block form built from the reference's couplings (recovered from its
    full-form terms) equals the reference's block gen_ham, and H_LL + H_RR
    has the spectrum of the full Hamiltonian."""
    import reapers_b200.syk as S
    g = gold("syk_block_N12.npz")
    N = 12
    q = S.all_quartets(N)
    ub, uc = S.quartic_terms(N, q, np.ones(len(q)))
    assert np.array_equal(ub, g["full_bits"])
    J = (g["full_coeff"] / uc).real
    (llb, llc), (rrb, rrc) = S.quartic_terms_block(N, q, J)
    assert np.array_equal(llb, g["ll_bits"]) and np.array_equal(rrb, g["rr_bits"])
    assert np.abs(llc - g["ll_coeff"]).max() < 1e-15 and np.abs(rrc - g["rr_coeff"]).max() < 1e-15
    Lb = int(g["len"])
    ev_full = np.linalg.eigvalsh(O.dense_matrix(N // 2, g["full_bits"], g["full_coeff"]))
    ev_blk = np.sort(np.concatenate([np.linalg.eigvalsh(O.dense_matrix(Lb, llb, llc)),
                                     np.linalg.eigvalsh(O.dense_matrix(Lb, rrb, rrc))]))
    np.testing.assert_allclose(ev_blk, ev_full, atol=1e-12)


def test_apply_at_matches_the_full_apply():
    """The index-sampled apply used for full-size spot checks equals the C
    restatement's full apply on the sampled rows, bit for bit in the sum
    order."""
    L = 11
    rng = np.random.default_rng(4)
    bits = rng.integers(0, 1 << (2 * L), 57, dtype=np.uint64)
    coeff = rng.standard_normal(57) + 1j * rng.standard_normal(57)
    vec = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    full = O.apply(L, bits, coeff, vec)
    idx = np.concatenate([[0, (1 << L) - 1], rng.integers(0, 1 << L, 300)])
    got = O.apply_at(bits, coeff, idx, lambda j: vec[j])
    np.testing.assert_allclose(got, full[idx], rtol=1e-14, atol=1e-14)
