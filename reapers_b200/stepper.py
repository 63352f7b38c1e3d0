"""Time-stepped Krylov evolution psi <- exp(-iHT) psi with two step controllers.

The reference evolves over the whole interval with its restarted Krylov
method (Krylov::evolve, inc/algo.h:267-365) and has no sub-stepping.  This
module adds the sub-stepped form that a step controller needs; each sub-step
is built from the same pieces on the GPU:

* ``rp_arnoldi`` -- one Arnoldi cycle of m vectors from the current state
  with the reference's orthogonalisation (inc/algo.h:77-173); the basis
  stays on the device, H_m and h_{m+1,m} come back;
* ``rp_expm_first_column`` -- exp(tau Hbar) e_1 for one or more step sizes,
  FP64 Pade-13 on the GPU, where Hbar is the (m+1) x (m+1) matrix
  [[H_m, 0], [h_{m+1,m} e_m^T, 0]].  Its first m entries are the step's
  Krylov coefficients; its last entry, tau h_{m+1,m} e_m^T phi_1(tau H_m) e_1,
  is the step's error estimate.  It is the reference's convergence measure
  (the norm of the newest block of column 0 of exp(f Hfull), inc/algo.h:350)
  for a following cycle of one vector whose own Hessenberg block is zero,
  and Saad's (1992) a-posteriori estimate;
* ``rp_arnoldi_combine`` -- psi <- beta_0 sum_i c_i v_i.

A sub-step of size dt is accepted when its relative error estimate is at
most tol * dt / T, so the estimates of all steps add up to at most tol.

``PlainController`` is Expokit's step control (Sidje, ACM TOMS 24 (1998),
routine expv): fixed basis size m (30 by default, Expokit's), first step
from a norm bound, next step gamma dt (tol dt / err)^(1/m) with gamma = 0.9
rounded to two significant digits, and the same formula to shrink a rejected
step (a rejection only recomputes the small exponential; no H.psi).

``LearnedController`` asks a small MLP (``StepModel``; forward, backward and
Adam are the CUDA kernels of rp_mlp.cu) for each step's (dt, m) from the
previous step's Lanczos coefficients alpha_1..8, beta_1..8, its residual norm
h_{m+1,m} and the problem's cost figures.  The plain error estimate accepts
or rejects the proposal; a rejected proposal falls back to the plain
shrink rule on the same basis.  The network is trained on traces of the
plain method (``generate_traces`` / ``make_dataset`` / ``train``), with
labels computed from each traced step's Hessenberg matrix: for every basis
size k the largest admissible step dt*(k), and the k that minimises the
modelled cost per unit time.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import _lib

__all__ = ["Basis", "arnoldi", "combine", "expm_first_columns", "step_errors",
           "PlainController", "LearnedController", "StepModel", "step_evolve",
           "generate_traces", "make_dataset", "train", "DEFAULT_MODEL"]

M_MIN, M_MAX = 10, 48          # basis sizes the learned controller may pick
K_SET = (10, 14, 18, 24, 30, 36, 42, 48)   # basis sizes labels are computed for
NFEAT = 8                      # Lanczos coefficients fed to the network
N_IN, N_OUT = 2 * NFEAT + 5, 2
STEP_OVERHEAD = 3.0            # fixed cost of a step in vector passes (norm, combine)
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                             "step_controller.npz")


# ---------------------------------------------------------------------------
# GPU primitives
# ---------------------------------------------------------------------------
class Basis:
    """One Arnoldi cycle: H (m_eff x m_eff), beta = h_{m+1,m}, beta0 = ||psi||."""

    def __init__(self, m, H, info):
        self.m = m
        self.m_eff = info.m_eff
        self.breakdown = bool(info.breakdown)
        self.passes = info.passes
        self.beta = 0.0 if info.breakdown else info.beta
        self.beta0 = info.beta0
        self.H = H[:self.m_eff, :self.m_eff].copy()

    def lanczos(self, k=NFEAT):
        """alpha_1..k (real diagonal) and beta_1..k (subdiagonal; beyond the
        basis, the residual norm, then zeros)."""
        d = self.H.diagonal().real
        sub = np.abs(np.diagonal(self.H, -1))
        a = np.zeros(k)
        b = np.zeros(k)
        a[:min(k, len(d))] = d[:k]
        sb = np.concatenate([sub, [self.beta]])
        b[:min(k, len(sb))] = sb[:k]
        return a, b


def arnoldi(ham, psi, m):
    """Arnoldi cycle of m vectors from psi (a CUDA tensor of ham's precision)."""
    from . import _ptr, _tcode
    if _tcode(psi) != ham.dtype:
        raise ValueError("state precision does not match the Hamiltonian's")
    m = int(m)
    Hbuf = np.zeros(2 * m * m)
    info = _lib.ArnoldiInfo()
    _lib.call("rp_arnoldi", ham.handle, _ptr(psi), m,
              Hbuf.ctypes.data_as(C.POINTER(C.c_double)), C.byref(info))
    H = Hbuf.view(np.complex128).reshape(m, m).T   # column-major -> [i, j]
    return Basis(m, H, info)


def combine(coef, out):
    """out = sum_i coef_i v_i over the last Arnoldi basis."""
    from . import _ptr
    c = np.ascontiguousarray(coef, dtype=np.complex128)
    _lib.call("rp_arnoldi_combine", c.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
              _ptr(out))
    return out


def expm_first_columns(A, factors):
    """Rows c: first column of exp(factors[c] * A), on the GPU (FP64)."""
    A = np.asarray(A, dtype=np.complex128)
    n = A.shape[0]
    f = np.atleast_1d(np.asarray(factors, dtype=np.complex128))
    if len(f) > 64:
        return np.concatenate([expm_first_columns(A, f[i:i + 64])
                               for i in range(0, len(f), 64)])
    Ac = np.ascontiguousarray(A.T)                  # [j, i] = column-major A
    fr = np.ascontiguousarray(f.real)
    fi = np.ascontiguousarray(f.imag)
    out = np.zeros((len(f), n), dtype=np.complex128)
    dp = C.POINTER(C.c_double)
    _lib.call("rp_expm_first_column", n, Ac.view(np.float64).ctypes.data_as(dp), len(f),
              fr.ctypes.data_as(dp), fi.ctypes.data_as(dp), out.view(np.float64).ctypes.data_as(dp))
    return out


def augmented(basis):
    """Hbar = [[H_m, 0], [h_{m+1,m} e_m^T, 0]]."""
    m = basis.m_eff
    A = np.zeros((m + 1, m + 1), dtype=np.complex128)
    A[:m, :m] = basis.H
    A[m, m - 1] = basis.beta
    return A


def step_errors(basis, dts):
    """(coefficients, relative error estimates) of steps exp(-i dt H) for each dt."""
    dts = np.atleast_1d(np.asarray(dts, dtype=np.float64))
    cols = expm_first_columns(augmented(basis), -1j * dts)
    return cols[:, :basis.m_eff], np.abs(cols[:, basis.m_eff])


def _round2(x):
    """Round up to two significant digits (Expokit's step rounding)."""
    if not np.isfinite(x) or x <= 0:
        return x
    s = 10.0 ** (math.floor(math.log10(x)) - 1)
    return math.ceil(x / s) * s


# ---------------------------------------------------------------------------
# Controllers
# ---------------------------------------------------------------------------
STRETCH = (1.25, 1.5, 2.0, 3.0, 4.0, 6.0, 8.0)   # step extensions tried on one basis


class PlainController:
    """Expokit's step-size control with a fixed basis size.  With
    stretch=True every accepted step is also tried at the multiples STRETCH of
    its size on the same basis (one small-matrix launch, no H.psi) and the
    largest admissible one is taken."""

    name = "plain"
    gamma = 0.9

    def __init__(self, m=30, stretch=False):
        self.m = int(m)
        self.stretch = bool(stretch)
        if self.stretch:
            self.name = "plain+stretch"

    def start(self, ham, T, tol):
        self.T, self.tol = float(T), float(tol)
        anorm = float(np.sum(np.abs(ham.coeff))) or 1.0   # bound on ||H||_2
        m = self.m
        fact = ((m + 1) / math.e) ** (m + 1) * math.sqrt(2 * math.pi * (m + 1))
        tol_u = self.tol / self.T
        self.dt_next = _round2((1.0 / anorm) * (fact * tol_u / (4.0 * anorm)) ** (1.0 / m))

    def propose(self, prev, t_left):
        return self.dt_next, self.m, False

    def shrink(self, dt, err, m):
        tol_u = self.tol / self.T
        return _round2(self.gamma * dt * (dt * tol_u / max(err, 1e-300)) ** (1.0 / m))

    def accepted(self, basis, dt, err, t_left):
        tol_u = self.tol / self.T
        if basis.breakdown or err <= 0:
            self.dt_next = t_left
        else:
            grow = self.gamma * dt * (dt * tol_u / err) ** (1.0 / basis.m_eff)
            self.dt_next = _round2(min(grow, 1e3 * dt))


class StepModel:
    """Trained MLP and its input/output standardisation, on the GPU."""

    def __init__(self, params, x_mean, x_std, y_mean, y_std, meta=None):
        self.params = np.asarray(params, dtype=np.float32)
        self.x_mean = np.asarray(x_mean, dtype=np.float32)
        self.x_std = np.asarray(x_std, dtype=np.float32)
        self.y_mean = np.asarray(y_mean, dtype=np.float32)
        self.y_std = np.asarray(y_std, dtype=np.float32)
        self.meta = dict(meta or {})
        self.net = Mlp(N_IN, N_OUT)
        self.net.set_params(self.params)

    def predict(self, X):
        Z = (np.asarray(X, np.float32) - self.x_mean) / self.x_std
        return self.net.forward(Z) * self.y_std + self.y_mean

    def save(self, path):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params, x_mean=self.x_mean, x_std=self.x_std,
                 y_mean=self.y_mean, y_std=self.y_std, meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path=DEFAULT_MODEL):
        d = np.load(path)
        return cls(d["params"], d["x_mean"], d["x_std"], d["y_mean"], d["y_std"],
                   json.loads(str(d["meta"])))

    def close(self):
        self.net.close()


class Mlp:
    """in -> 64 -> 64 -> out tanh network on the GPU (rp_mlp_* of the C ABI)."""

    def __init__(self, n_in, n_out, seed=0):
        self.n_in, self.n_out = int(n_in), int(n_out)
        h = C.c_void_p()
        _lib.call("rp_mlp_create", C.byref(h), self.n_in, self.n_out, int(seed))
        self._h = h
        n = C.c_int()
        _lib.call("rp_mlp_num_params", h, C.byref(n))
        self.num_params = n.value

    def get_params(self):
        p = np.zeros(self.num_params, np.float32)
        _lib.call("rp_mlp_get_params", self._h, p.ctypes.data_as(C.POINTER(C.c_float)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError("wrong number of parameters")
        _lib.call("rp_mlp_set_params", self._h, p.ctypes.data_as(C.POINTER(C.c_float)))

    def forward(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.n_in)
        Y = np.zeros((X.shape[0], self.n_out), np.float32)
        fp = C.POINTER(C.c_float)
        _lib.call("rp_mlp_forward", self._h, X.ctypes.data_as(fp), X.shape[0], Y.ctypes.data_as(fp))
        return Y

    def grad(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.n_in)
        Y = np.ascontiguousarray(Y, dtype=np.float32).reshape(-1, self.n_out)
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float()
        fp = C.POINTER(C.c_float)
        _lib.call("rp_mlp_grad", self._h, X.ctypes.data_as(fp), Y.ctypes.data_as(fp), X.shape[0],
                  g.ctypes.data_as(fp), C.byref(loss))
        return loss.value, g

    def train(self, X, Y, epochs=50, batch=256, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, self.n_in)
        Y = np.ascontiguousarray(Y, dtype=np.float32).reshape(-1, self.n_out)
        loss = C.c_float()
        fp = C.POINTER(C.c_float)
        _lib.call("rp_mlp_train", self._h, X.ctypes.data_as(fp), Y.ctypes.data_as(fp), X.shape[0],
                  int(epochs), int(batch), float(lr), int(seed), C.byref(loss))
        return loss.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().rp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SMEM_OVER_HBM = 5.7   # B200: shared-memory bandwidth (128 B/clk/SM) over HBM bandwidth


def problem_figures(ham):
    """A, the cost of one H.psi in units of one streaming pass over a vector:
    the larger of its compulsory DRAM bytes and its shared-memory gather
    bytes scaled by the shared-memory / HBM bandwidth ratio, over the bytes
    of one vector."""
    info = ham.info()
    vec = float(1 << ham.len) * (8 if ham.dtype == 1 else 16)
    return max(1.0, info["alg_bytes_dram"] / vec, info["smem_bytes"] / SMEM_OVER_HBM / vec)


def features(basis, m_prev, tol_u, A):
    """Network input from the previous step's Arnoldi data.  All quantities
    are made dimensionless with s, the RMS of the first Lanczos coefficients
    (tol_u = tol / T is an inverse time)."""
    a, b = basis.lanczos(NFEAT)
    s = math.sqrt(float(np.mean(a * a + b * b))) or 1.0
    rho = basis.passes / max(1, basis.m_eff)
    x = np.concatenate([a / s, b / s,
                        [basis.beta / s, m_prev / 32.0, math.log10(max(tol_u / s, 1e-300)) / 10.0,
                         math.log10(A) / 2.0, rho - 1.0]])
    return x.astype(np.float32), s


def step_cost(k, A, rho):
    """Modelled cost of one step with k basis vectors, in vector passes:
    k H.psi products; per basis vector j and orthogonalisation pass (rho per
    vector) a projection pass over the j + 1 vectors so far (w re-read once
    per group of 8) and an update pass over them (w read and written); the
    final combination of k vectors and the fixed overhead."""
    ortho = 1.125 * k * (k + 1) / 2.0 + k * (k + 5) / 2.0   # sum over j < k
    return k * A + rho * ortho + k + 1 + STEP_OVERHEAD


class LearnedController(PlainController):
    """MLP-proposed (dt, m), checked by the plain error estimate.

    When the proposed step reaches the end of the interval, the basis is cut
    to the smallest size whose admissible step -- estimated from the previous
    restart's Hessenberg matrix exactly as the training labels are -- still
    covers the remaining time."""

    name = "learned"

    def __init__(self, model, m_first=30, safety=0.95, stretch=True):
        super().__init__(m_first, stretch)
        self.name = "learned"
        self.model = model
        self.safety = float(safety)

    def start(self, ham, T, tol):
        super().start(ham, T, tol)
        self.A = problem_figures(ham)

    def propose(self, prev, t_left):
        if prev is None or prev.m_eff < NFEAT + 1:
            return self.dt_next, self.m, False
        tol_u = self.tol / self.T
        x, s = features(prev, prev.m_eff, tol_u, self.A)
        y = self.model.predict(x[None, :])[0]
        m = int(np.clip(round(float(y[1]) * 32.0), M_MIN, M_MAX))
        dt = self.safety * math.exp(float(np.clip(y[0], -12.0, 12.0))) / s
        # growth limit: at most 4x the last accepted step
        dt = min(dt, 4.0 * self.dt_last)
        if dt >= t_left:
            m = self._last_step_basis(prev, t_left, m, tol_u)
        self.m = m
        return dt, m, True

    @staticmethod
    def _last_step_basis(prev, t_left, m, tol_u):
        for k in range(M_MIN, min(m - 1, prev.m_eff) + 1, 2):
            beta = abs(prev.H[k, k - 1]) if k < prev.m_eff else prev.beta
            d = admissible_dt(prev.H[None, :k, :k], np.array([beta]), tol_u,
                              np.array([t_left * 1e-3]), np.array([t_left]))
            if d[0] >= t_left:
                return k
        return m

    def accepted(self, basis, dt, err, t_left):
        super().accepted(basis, dt, err, t_left)
        self.dt_last = dt


# ---------------------------------------------------------------------------
# The stepped evolve
# ---------------------------------------------------------------------------
def step_evolve(ham, psi, T, tol=1e-8, controller=None, record=False, max_steps=100000,
                max_reject=30):
    """psi <- exp(-i T H) psi in place by accepted sub-steps; returns statistics.

    The sum of the accepted steps' relative error estimates is at most tol."""
    import torch
    ctl = controller or PlainController()
    ctl.start(ham, T, tol)
    tol_u = float(tol) / float(T)
    t = 0.0
    prev = None
    st = {"controller": ctl.name, "steps": 0, "applies": 0, "proposals": 0,
          "proposals_accepted": 0, "rejections": 0, "stretched": 0, "err_sum": 0.0, "cost": 0.0,
          "ms_mlp": 0.0, "trace": [] if record else None}
    A = problem_figures(ham)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while T - t > 1e-12 * T:
        if st["steps"] >= max_steps:
            raise RuntimeError("step_evolve: too many steps")
        t_left = T - t
        tm = time.perf_counter()
        dt, m, learned = ctl.propose(prev, t_left)
        st["ms_mlp"] += (time.perf_counter() - tm) * 1e3 if learned else 0.0
        basis = arnoldi(ham, psi, m)
        st["applies"] += basis.m_eff
        st["cost"] += step_cost(basis.m_eff, A, basis.passes / max(1, basis.m_eff))
        dt = t_left if basis.breakdown else min(dt, t_left)
        coef, err = step_errors(basis, [dt])
        err = float(err[0])
        ok = err <= tol_u * dt
        if learned:
            st["proposals"] += 1
            st["proposals_accepted"] += int(ok)
        nrej = 0
        while not ok:
            st["rejections"] += 1
            nrej += 1
            if nrej > max_reject:
                raise RuntimeError("step_evolve: step size could not be controlled")
            dt = min(ctl.shrink(dt, err, basis.m_eff), t_left)
            coef, err = step_errors(basis, [dt])
            err = float(err[0])
            ok = err <= tol_u * dt
        if ctl.stretch and dt < t_left:
            cands = sorted({min(dt * f, t_left) for f in STRETCH} - {dt})
            c2, e2 = step_errors(basis, cands)
            good = [i for i in range(len(cands)) if e2[i] <= tol_u * cands[i]]
            if good:
                i = good[-1]
                dt, err = cands[i], float(e2[i])
                coef = c2[i:i + 1]
                st["stretched"] += 1
        combine(basis.beta0 * coef[0], psi)
        if record:
            st["trace"].append({"t": t, "dt": dt, "m": basis.m_eff, "err": err,
                                "H": basis.H.copy(), "beta": basis.beta,
                                "passes": basis.passes, "beta0": basis.beta0})
        t += dt
        st["steps"] += 1
        st["err_sum"] += err
        ctl.accepted(basis, dt, err, T - t)
        prev = basis
    torch.cuda.synchronize()
    st["seconds"] = time.perf_counter() - t0
    return st


# ---------------------------------------------------------------------------
# Traces, labels, training
# ---------------------------------------------------------------------------
def _phi1(z):
    out = np.ones_like(z)
    big = np.abs(z) > 1e-6
    out[big] = np.expm1(z[big]) / z[big]
    small = ~big
    out[small] = 1 + z[small] / 2 + z[small] ** 2 / 6
    return out


def admissible_dt(Hs, betas, tol_u, lo, hi, iters=48):
    """Largest dt in [lo, hi] (per row) with dt beta |e_k^T phi_1(-i dt T_k) e_1|
    <= tol_u dt, T_k the Hermitian part of each leading k x k block.

    Hs: (n, k, k) complex; betas: (n,) the coupling h_{k+1,k}; lo, hi: (n,)."""
    Tk = 0.5 * (Hs + np.conj(np.swapaxes(Hs, 1, 2)))
    lam, Q = np.linalg.eigh(Tk)
    w = Q[:, -1, :] * np.conj(Q[:, 0, :])            # (n, k)
    lo = np.log(lo)
    hi = np.log(hi)

    def ok(logdt):
        dt = np.exp(logdt)[:, None]
        g = betas * np.abs(np.sum(w * _phi1(-1j * dt * lam), axis=1))
        return g <= tol_u

    good_hi = ok(hi)
    a, b = lo.copy(), hi.copy()
    for _ in range(iters):
        mid = 0.5 * (a + b)
        o = ok(mid)
        a = np.where(o, mid, a)
        b = np.where(o, b, mid)
    return np.where(good_hi, np.exp(hi), np.exp(a))


def label_steps(steps, tol_u, A, ksizes=K_SET):
    """Per traced step: dt*(k) for k in ksizes and the cost-optimal (k*, dt*).

    steps: list of dicts with 'H' (m x m), 'beta', 'passes'.  Returns
    (kstar, dtstar, table) with table (n, len(ksizes)) of dt*(k)."""
    n = len(steps)
    table = np.full((n, len(ksizes)), np.nan)
    rho = np.array([s["passes"] / max(1, s["H"].shape[0]) for s in steps])
    for ci, k in enumerate(ksizes):
        idx = [i for i, s in enumerate(steps) if s["H"].shape[0] >= k]
        if not idx:
            continue
        Hs = np.stack([steps[i]["H"][:k, :k] for i in idx])
        betas = np.array([abs(steps[i]["H"][k, k - 1]) if steps[i]["H"].shape[0] > k
                          else steps[i]["beta"] for i in idx])
        s = np.array([max(1e-300, float(np.sqrt(np.mean(np.abs(steps[i]["H"][:NFEAT + 1,
                                                                              :NFEAT + 1]) ** 2))))
                      for i in idx])
        lo = 1e-4 / s
        hi = 1e3 / s
        table[idx, ci] = admissible_dt(Hs, betas, tol_u, lo, hi)
    cost = np.array([[step_cost(k, A, rho[i]) for k in ksizes] for i in range(n)])
    per_time = cost / table
    per_time[~np.isfinite(per_time)] = np.inf
    best = np.argmin(per_time, axis=1)
    kstar = np.array(ksizes)[best]
    dtstar = table[np.arange(n), best]
    return kstar, dtstar, table


def generate_traces(problems, m=M_MAX, log=None):
    """Run the plain method (basis size m) on each problem and record its steps.

    problems: iterable of dicts {'ham': Hamiltonian, 'psi': CUDA tensor,
    'T': float, 'tol': float}.  Returns a list of runs
    {'steps': [...], 'tol_u', 'A', 'len'}."""
    runs = []
    for i, p in enumerate(problems):
        st = step_evolve(p["ham"], p["psi"], p["T"], p["tol"], PlainController(m), record=True)
        runs.append({"steps": st["trace"], "tol_u": p["tol"] / p["T"],
                     "A": problem_figures(p["ham"]), "len": p["ham"].len})
        if log:
            log(f"trace {i}: L={p['ham'].len} steps={st['steps']} applies={st['applies']}")
    return runs


class _Prev:
    """The parts of a Basis that features() reads, cut to k vectors."""

    def __init__(self, H, beta, passes, k):
        self.H = H[:k, :k]
        self.m_eff = k
        self.beta = abs(H[k, k - 1]) if H.shape[0] > k else beta
        self.passes = passes * k / H.shape[0]

    lanczos = Basis.lanczos


def make_dataset(runs, prev_sizes=K_SET):
    """(X, Y) pairs: features of step i (as if it had used k_prev vectors, for
    each k_prev in prev_sizes) -> the optimal (log(dt* s), k*/32) of step i+1."""
    X, Y = [], []
    for run in runs:
        steps = run["steps"]
        if len(steps) < 2:
            continue
        kstar, dtstar, _ = label_steps(steps[1:], run["tol_u"], run["A"])
        for i in range(len(steps) - 1):
            if not np.isfinite(dtstar[i]):
                continue
            S = steps[i]
            for kp in prev_sizes:
                if S["H"].shape[0] < kp:
                    continue
                prev = _Prev(S["H"], S["beta"], S["passes"], kp)
                x, s = features(prev, kp, run["tol_u"], run["A"])
                X.append(x)
                Y.append([math.log(dtstar[i] * s), kstar[i] / 32.0])
    return np.array(X, np.float32), np.array(Y, np.float32)


def train(X, Y, epochs=60, batch=512, lr=2e-3, seed=0, meta=None):
    """Standardise (X, Y), train the MLP on the GPU; returns (StepModel, loss)."""
    xm, xs = X.mean(0), X.std(0) + 1e-6
    ym, ys = Y.mean(0), Y.std(0) + 1e-6
    net = Mlp(N_IN, N_OUT, seed=seed)
    loss = net.train((X - xm) / xs, (Y - ym) / ys, epochs=epochs, batch=batch, lr=lr, seed=seed)
    params = net.get_params()
    net.close()
    model = StepModel(params, xm, xs, ym, ys, dict(meta or {}, samples=int(len(X)),
                                                   epochs=epochs, batch=batch, lr=lr,
                                                   loss=float(loss)))
    return model, loss


def training_problems(count, seed=0, dtype="c128"):
    """Yield small problems for the traces, ordered by qubit count: XXZ chains
    (L = 12..20, J = Jz = 1 in Pauli units, fields U[-W, W] with W in
    [0.3, 4]) and sparse SYK (N = 24..32 Majoranas, k = 8), tolerances
    1e-10..1e-6 and times 1..10, each with a random normalised state."""
    from . import Hamiltonian, random_state, syk
    rng = np.random.default_rng(seed)
    kinds = []
    for i in range(count):
        if rng.random() < 0.6:
            L = int(rng.choice([12, 14, 16, 18, 20]))
            kinds.append(("xxz", L, float(rng.uniform(0.3, 4.0)), int(rng.integers(1 << 30))))
        else:
            N = int(rng.choice([24, 28, 32]))
            kinds.append(("syk", N // 2, N, int(rng.integers(1 << 30))))
    kinds.sort(key=lambda k: k[1])
    for kind in kinds:
        r = np.random.default_rng(kind[3])
        if kind[0] == "xxz":
            L, W = kind[1], kind[2]
            bits, coeff = syk.xxz_chain(L, 1.0, r.uniform(-W, W, L))
        else:
            L, N = kind[1], kind[2]
            bits, coeff = syk.sparse_syk(N, 8, seed=kind[3])
        ham = Hamiltonian(L, bits, coeff, dtype)
        psi = random_state(L, dtype, seed=kind[3])
        yield {"ham": ham, "psi": psi, "T": float(r.choice([1.0, 2.0, 5.0, 10.0])),
               "tol": float(10.0 ** r.uniform(-10, -6)), "kind": kind[0]}


def _main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="train the learned Krylov step controller")
    ap.add_argument("--problems", type=int, default=400)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    args = ap.parse_args(argv)
    t0 = time.perf_counter()
    runs = []
    for p in training_problems(args.problems, args.seed):
        runs.extend(generate_traces([p]))
        p["ham"].close()
    t1 = time.perf_counter()
    X, Y = make_dataset(runs)
    t2 = time.perf_counter()
    nsteps = sum(len(r["steps"]) for r in runs)
    model, loss = train(X, Y, epochs=args.epochs, seed=args.seed,
                        meta={"problems": args.problems, "trace_steps": nsteps})
    t3 = time.perf_counter()
    model.meta.update(trace_seconds=t1 - t0, label_seconds=t2 - t1, train_seconds=t3 - t2)
    model.save(args.out)
    print(json.dumps(model.meta))


if __name__ == "__main__":
    _main()
