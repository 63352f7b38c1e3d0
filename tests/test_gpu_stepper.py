"""GPU parity of the time-stepped Krylov primitives and of the step-controller MLP.

* rp_expm_first_column against scipy's expm; rp_arnoldi against a dense
  Lanczos with full reorthogonalisation on the oracle's dense matrix;
* the stepped evolve (plain controller) against exp(-iHT) of the oracle's
  dense matrix, both precisions;
* the MLP's CUDA forward, backward and Adam kernels against the numpy
  restatement in oracle/mlp_oracle.py (backprop and central differences);
* the learned controller, trained here on traces of the plain method, against
  the plain controller on held-out problems: lower modelled cost (H.psi and
  orthogonalisation passes) at equal tolerance.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import mlp_oracle as MO
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    import reapers_b200 as R
    R.init(0)
    return R


@pytest.fixture(scope="module")
def SP(R):
    from reapers_b200 import stepper
    return stepper


def _xxz(L, W, seed):
    from reapers_b200 import syk
    rng = np.random.default_rng(seed)
    return syk.xxz_chain(L, 1.0, rng.uniform(-W, W, L))


def test_expm_first_column_matches_scipy(SP):
    rng = np.random.default_rng(0)
    for n in (1, 7, 33, 49):
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        f = np.array([0.05j, -0.7j, 0.3 + 0.2j, -2.5j])
        got = SP.expm_first_columns(A, f)
        ref = np.stack([sla.expm(x * A)[:, 0] for x in f])
        assert np.max(np.abs(got - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("model", ["xxz", "syk"])
def test_arnoldi_matches_dense_lanczos(R, SP, model):
    from reapers_b200 import syk
    L = 8
    bits, coeff = _xxz(L, 1.0, 1) if model == "xxz" else syk.sparse_syk(16, 8, seed=2)
    ham = R.Hamiltonian(L, bits, coeff, "c128")
    Hd = O.dense_matrix(L, bits, coeff)
    psi = R.random_state(L, "c128", seed=3)
    p0 = psi.cpu().numpy()
    m = 12
    b = SP.arnoldi(ham, psi, m)
    V = [p0 / np.linalg.norm(p0)]
    Hl = np.zeros((m + 1, m), complex)
    for j in range(m):
        w = Hd @ V[j]
        for _ in range(2):
            for i in range(j + 1):
                h = np.vdot(V[i], w)
                Hl[i, j] += h
                w = w - h * V[i]
        Hl[j + 1, j] = np.linalg.norm(w)
        V.append(w / Hl[j + 1, j])
    scale = np.max(np.abs(Hl))
    assert b.m_eff == m and not b.breakdown
    assert np.max(np.abs(b.H - Hl[:m, :m])) <= 1e-12 * scale
    assert abs(b.beta - Hl[m, m - 1]) <= 1e-12 * scale
    assert abs(b.beta0 - np.linalg.norm(p0)) <= 1e-13
    ham.close()


@pytest.mark.parametrize("model,dtype,tol,bound", [
    ("xxz", "c128", 1e-10, 1e-9), ("syk", "c128", 1e-10, 1e-9),
    ("xxz", "c64", 1e-6, 2e-5), ("syk", "c64", 1e-6, 2e-5)])
def test_stepped_evolve_matches_dense_expm(R, SP, model, dtype, tol, bound):
    import torch
    from reapers_b200 import syk
    L, T = 10, 2.0
    bits, coeff = _xxz(L, 2.0, 4) if model == "xxz" else syk.sparse_syk(20, 8, seed=5)
    ham = R.Hamiltonian(L, bits, coeff, dtype)
    psi = R.random_state(L, dtype, seed=7)
    p0 = psi.cpu().numpy().astype(np.complex128)
    exact = sla.expm(-1j * T * O.dense_matrix(L, bits, coeff)) @ p0
    for m in (30, 12):
        ps = psi.clone()
        st = SP.step_evolve(ham, ps, T, tol, SP.PlainController(m))
        got = ps.cpu().numpy().astype(np.complex128)
        err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
        assert err <= bound, (m, err, st)
        assert st["err_sum"] <= tol * (1 + 1e-9)
        assert st["applies"] <= m * st["steps"]
    ham.close()
    torch.cuda.synchronize()


def test_mlp_forward_and_gradient_match_oracle(SP):
    rng = np.random.default_rng(11)
    net = SP.Mlp(SP.N_IN, SP.N_OUT, seed=5)
    p = net.get_params()
    assert p.size == MO.num_params(SP.N_IN, SP.N_OUT)
    X = rng.standard_normal((700, SP.N_IN)).astype(np.float32)
    Y = rng.standard_normal((700, SP.N_OUT)).astype(np.float32)
    p64, X64, Y64 = p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64)
    np.testing.assert_allclose(net.forward(X), MO.forward(p64, X64, SP.N_IN, SP.N_OUT),
                               rtol=1e-5, atol=1e-5)
    loss, g = net.grad(X, Y)
    L0, g0 = MO.grad(p64, X64, Y64, SP.N_IN, SP.N_OUT)
    assert abs(loss - L0) <= 1e-5 * L0
    assert np.max(np.abs(g - g0)) <= 1e-5 * np.max(np.abs(g0))
    # and against central differences of the loss (float64 oracle)
    idx = rng.choice(p.size, 40, replace=False)
    fd = MO.finite_diff(p64, X64[:64], Y64[:64], SP.N_IN, SP.N_OUT, idx)
    _, g64 = net.grad(X[:64], Y[:64])
    np.testing.assert_allclose(g64[idx], fd, rtol=2e-3, atol=2e-6)
    net.close()


def test_mlp_adam_step_matches_oracle(SP):
    rng = np.random.default_rng(12)
    net = SP.Mlp(SP.N_IN, SP.N_OUT, seed=6)
    p = net.get_params().astype(np.float64)
    X = rng.standard_normal((200, SP.N_IN)).astype(np.float32)
    Y = rng.standard_normal((200, SP.N_OUT)).astype(np.float32)
    _, g = MO.grad(p, X.astype(np.float64), Y.astype(np.float64), SP.N_IN, SP.N_OUT)
    z = np.zeros_like(p)
    p1, m1, v1 = MO.adam_step(p, g, z, z, 1, lr=1e-3)
    p2, _, _ = MO.adam_step(p1, MO.grad(p1, X.astype(np.float64), Y.astype(np.float64),
                                        SP.N_IN, SP.N_OUT)[1], m1, v1, 2, lr=1e-3)
    net.train(X, Y, epochs=2, batch=200, lr=1e-3)   # two full-batch Adam steps
    got = net.get_params()
    # components whose gradient is at rounding level may step either way
    sig = np.abs(g) > 1e-4 * np.max(np.abs(g))
    np.testing.assert_allclose(got[sig], p2[sig], rtol=1e-5, atol=2e-6)
    net.close()


def test_mlp_training_fits_a_smooth_map(SP):
    rng = np.random.default_rng(13)
    X = rng.uniform(-1, 1, (4000, SP.N_IN)).astype(np.float32)
    Y = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], np.tanh(X[:, 3] - X[:, 4])], 1)
    Y = Y.astype(np.float32)
    net = SP.Mlp(SP.N_IN, SP.N_OUT, seed=7)
    l0, _ = net.grad(X, Y)
    l1 = net.train(X, Y, epochs=40, batch=128, lr=3e-3)
    l2, _ = net.grad(X, Y)
    assert l2 < 0.05 * l0 and l1 < 0.1 * l0
    net.close()


def test_learned_controller_beats_plain(R, SP):
    """Train on plain-method traces of small random problems, then compare on
    problems the network has not seen, at equal tolerance."""
    import torch
    from reapers_b200 import syk
    runs = []
    for p in SP.training_problems(40, seed=21):
        runs.extend(SP.generate_traces([p]))
        p["ham"].close()
    X, Y = SP.make_dataset(runs)
    assert len(X) > 500
    model, loss = SP.train(X, Y, epochs=40)
    assert loss < 0.2
    tol, T = 1e-8, 10.0
    # the controller minimises the modelled cost per unit time (H.psi and
    # orthogonalisation passes over the state), so that is what it must lower
    tot = {"plain": 0.0, "plain+stretch": 0.0, "learned": 0.0}
    for L, (bits, coeff) in [(14, _xxz(14, 0.5, 901)), (14, _xxz(14, 3.0, 902)),
                             (14, syk.sparse_syk(28, 8, seed=903))]:
        ham = R.Hamiltonian(L, bits, coeff, "c128")
        psi = R.random_state(L, "c128", seed=904)
        out = {}
        for ctl in (SP.PlainController(30), SP.PlainController(30, stretch=True),
                    SP.LearnedController(model)):
            ps = psi.clone()
            st = SP.step_evolve(ham, ps, T, tol, ctl)
            assert st["err_sum"] <= tol
            tot[ctl.name] += st["cost"]
            out[ctl.name] = ps
        assert torch.linalg.vector_norm(out["plain"] - out["learned"]).item() <= 4 * tol
        ham.close()
    model.close()
    assert tot["learned"] < 0.97 * tot["plain"], tot
