"""CPU checks of the learned step controller's host logic and of the MLP oracle.

No GPU: the oracle's backprop is pinned against finite differences, and the
label computation (largest admissible step per basis size) against the
exponential of the augmented Hessenberg matrix that the GPU error estimate
uses.
"""
import math

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import mlp_oracle as MO
from reapers_b200 import stepper as SP


def test_oracle_backprop_matches_finite_differences():
    rng = np.random.default_rng(3)
    n_in, n_out, n = SP.N_IN, SP.N_OUT, 9
    p = rng.standard_normal(MO.num_params(n_in, n_out)) * 0.3
    X = rng.standard_normal((n, n_in))
    Y = rng.standard_normal((n, n_out))
    L, g = MO.grad(p, X, Y, n_in, n_out)
    assert abs(L - MO.loss(p, X, Y, n_in, n_out)) < 1e-12
    idx = rng.choice(p.size, 60, replace=False)
    fd = MO.finite_diff(p, X, Y, n_in, n_out, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_oracle_adam_first_step_is_signed_lr():
    g = np.array([0.5, -2.0, 1e-3])
    p, m, v = MO.adam_step(np.zeros(3), g, np.zeros(3), np.zeros(3), 1, lr=0.1)
    np.testing.assert_allclose(p, -0.1 * np.sign(g), rtol=1e-4)


def _tridiag(k, rng, scale=1.0):
    a = rng.standard_normal(k) * scale
    b = np.abs(rng.standard_normal(k)) * scale + 0.3 * scale
    H = np.diag(a).astype(np.complex128)
    H += np.diag(b[:k - 1], -1) + np.diag(b[:k - 1], 1)
    return H, b[k - 1]


def _estimate(H, beta, dt):
    k = H.shape[0]
    A = np.zeros((k + 1, k + 1), np.complex128)
    A[:k, :k] = H
    A[k, k - 1] = beta
    return abs(sla.expm(-1j * dt * A)[k, 0])


@pytest.mark.parametrize("k", [6, 12, 20])
def test_admissible_dt_sits_on_the_error_boundary(k):
    rng = np.random.default_rng(k)
    Hs, betas = [], []
    for _ in range(5):
        H, b = _tridiag(k, rng)
        Hs.append(H)
        betas.append(b)
    tol_u = 1e-8
    dt = SP.admissible_dt(np.stack(Hs), np.array(betas), tol_u, np.full(5, 1e-4),
                          np.full(5, 1e3))
    for H, b, d in zip(Hs, betas, dt):
        # error estimate per unit step equals the tolerance at dt* ...
        np.testing.assert_allclose(_estimate(H, b, d) / d, tol_u, rtol=1e-5)
        # ... and is below it just under dt*
        assert _estimate(H, b, 0.99 * d) / (0.99 * d) < tol_u


def test_labels_pick_the_cheapest_basis_per_unit_time():
    rng = np.random.default_rng(1)
    steps = []
    for _ in range(4):
        H, b = _tridiag(48, rng)
        steps.append({"H": H, "beta": b, "passes": 60})
    for A in (5.0, 400.0):
        kstar, dtstar, table = SP.label_steps(steps, 1e-8, A)
        for i in range(len(steps)):
            rho = 60 / 48
            per = [SP.step_cost(k, A, rho) / table[i, j] for j, k in enumerate(SP.K_SET)]
            assert kstar[i] == SP.K_SET[int(np.argmin(per))]
            assert dtstar[i] == table[i, int(np.argmin(per))]
    # an expensive H.psi favours larger bases
    k_cheap, _, _ = SP.label_steps(steps, 1e-8, 5.0)
    k_dear, _, _ = SP.label_steps(steps, 1e-8, 400.0)
    assert np.all(k_dear >= k_cheap)


class _FakeBasis:
    def __init__(self, H, beta, passes):
        self.H, self.beta, self.passes, self.m_eff = H, beta, passes, H.shape[0]

    lanczos = SP.Basis.lanczos


def test_features_are_scale_free():
    rng = np.random.default_rng(2)
    H, b = _tridiag(16, rng)
    x1, s1 = SP.features(_FakeBasis(H, b, 20), 16, 1e-9, 30.0)
    x2, s2 = SP.features(_FakeBasis(7.5 * H, 7.5 * b, 20), 16, 7.5e-9, 30.0)
    assert x1.shape == (SP.N_IN,)
    np.testing.assert_allclose(x1, x2, rtol=1e-5, atol=1e-6)
    assert math.isclose(s2 / s1, 7.5, rel_tol=1e-12)


def test_dataset_pairs_previous_features_with_next_labels():
    rng = np.random.default_rng(4)
    steps = []
    for _ in range(3):
        H, b = _tridiag(48, rng)
        steps.append({"H": H, "beta": b, "passes": 50})
    runs = [{"steps": steps, "tol_u": 1e-8, "A": 20.0, "len": 12}]
    X, Y = SP.make_dataset(runs)
    assert X.shape == (2 * len(SP.K_SET), SP.N_IN) and Y.shape == (len(X), SP.N_OUT)
    kstar, dtstar, _ = SP.label_steps(steps[1:], 1e-8, 20.0)
    # every k_prev variant of step 0 carries step 1's label
    np.testing.assert_allclose(Y[:len(SP.K_SET), 1], kstar[0] / 32.0)
    assert np.all(np.isfinite(X))
