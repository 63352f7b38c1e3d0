"""REAPERS hot path on B200: Pauli-sum H.psi and restarted Krylov exp(-iHt)psi.

Python host layer over the C ABI of ``librpb200.so`` (include/rpb200.h).
State vectors are CUDA tensors (complex64 / complex128, contiguous); the
library reads and writes them in place through their device pointers.  The
operations mirror the reference's backend concept (inc/gpuimpl.h:853-1047)
and ``State::evolve`` (inc/state.h:415-424).  There is no CPU fallback: every
call goes to the CUDA kernels and raises if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import RP_C64, RP_C128, RPError
from . import syk  # noqa: F401  (term generators)

__all__ = ["Hamiltonian", "evolve", "ground_state", "ipc_export", "ipc_open", "ipc_close", "dot", "norm", "axpy", "scale", "random_state",
           "stream", "synchronize", "RPError", "RP_C64", "RP_C128", "dtype_code", "syk",
           "otoc", "otoc_block"]


def dtype_code(dtype):
    """'c64'/'c128'/torch dtype/numpy dtype -> RP_C64 / RP_C128."""
    s = str(dtype)
    if s in ("c64", "complex64", "torch.complex64", "1"):
        return RP_C64
    if s in ("c128", "complex128", "torch.complex128", "2"):
        return RP_C128
    raise ValueError(f"unsupported dtype {dtype!r}")


def _ptr(t):
    """Device pointer of a contiguous CUDA tensor (or a raw integer pointer)."""
    if isinstance(t, int):
        return C.c_void_p(t)
    if not t.is_cuda:
        raise ValueError("vector must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("vector must be contiguous")
    return C.c_void_p(t.data_ptr())


def _tcode(t):
    import torch
    if t.dtype == torch.complex64:
        return RP_C64
    if t.dtype == torch.complex128:
        return RP_C128
    raise ValueError(f"vector dtype {t.dtype} is not complex64/complex128")


def init(device=0):
    _lib.call("rp_init", int(device))


def stream():
    """The library's CUDA stream as a torch.cuda.ExternalStream."""
    import torch
    return torch.cuda.ExternalStream(_lib.load().rp_stream())


def synchronize():
    _lib.call("rp_synchronize")


class Hamiltonian:
    """A sum of Pauli strings uploaded and grouped for the H.psi kernel.

    bits: uint64 SpinOp bit strings (bit 2i = X on site i, bit 2i+1 = Z);
    coeff: the stored complex coefficients (sigma_y carries its i here, as in
    inc/ops.h:285-288).  Mirrors DevSumOps::upload (inc/gpuimpl.h:1065-1085).
    """

    def __init__(self, length, bits, coeff, dtype="c128", tile_exp=None):
        self.len = int(length)
        self.dtype = dtype_code(dtype)
        b = np.ascontiguousarray(bits, dtype=np.uint64)
        c = np.ascontiguousarray(coeff, dtype=np.complex128)
        if b.shape != c.shape:
            raise ValueError("bits and coeff must have the same length")
        self.nterms = len(b)
        cd = c.view(np.float64)
        h = C.c_void_p()
        _lib.call("rp_ham_create_ex", C.byref(h), self.len, self.dtype, self.nterms,
                  b.ctypes.data_as(C.POINTER(C.c_uint64)),
                  cd.ctypes.data_as(C.POINTER(C.c_double)), int(tile_exp or 0))
        self._h = h
        self.bits, self.coeff = b.copy(), c.copy()

    @property
    def handle(self):
        return self._h

    def info(self):
        i = _lib.HamInfo()
        _lib.call("rp_ham_info", self._h, C.byref(i))
        return {k: getattr(i, k) for k, _ in _lib.HamInfo._fields_}

    def apply(self, out, inp, accumulate=False):
        """out = H inp (out += H inp with accumulate)."""
        if _tcode(out) != self.dtype or _tcode(inp) != self.dtype:
            raise ValueError("vector precision does not match the Hamiltonian's")
        _lib.call("rp_apply", self._h, _ptr(out), _ptr(inp), 1 if accumulate else 0)
        return out

    def apply_host(self, outs, ins):
        """outs[i] = H ins[i] for CPU tensors (pinned for overlap): one call,
        the host<->device copies pipelined with the products (rp_apply_host)."""
        n = len(ins)
        if len(outs) != n:
            raise ValueError("outs and ins differ in length")
        want = 1 << self.len
        for t in list(ins) + list(outs):
            if t.is_cuda or not t.is_contiguous() or t.numel() != want or _tcode(t) != self.dtype:
                raise ValueError("host vectors must be contiguous CPU tensors of the "
                                 "Hamiltonian's size and precision")
        ip = (C.c_void_p * n)(*[t.data_ptr() for t in ins])
        op = (C.c_void_p * n)(*[t.data_ptr() for t in outs])
        _lib.call("rp_apply_host", self._h, n, ip, op)
        return outs

    def apply_shard(self, out, shards, rank, accumulate=False):
        """out = output shard `rank` of H applied to the state whose 2^k
        shards (top k qubits, k = log2 len(shards)) are the device tensors or
        raw device pointers `shards`; a shard may be a peer's memory (see
        ``ipc_export`` / ``ipc_open``).  One row-kernel launch reading every
        source tile from the shard that holds it (rp_apply_shard)."""
        n = len(shards)
        k = n.bit_length() - 1
        if n < 2 or 1 << k != n:
            raise ValueError("the number of shards must be a power of two, at least 2")
        if not 0 <= rank < n:
            raise ValueError("rank must name one of the shards")
        want = 1 << (self.len - k)
        if _tcode(out) != self.dtype or out.numel() != want:
            raise ValueError("the output shard must have 2^(len - k) elements of the "
                             "Hamiltonian's precision")
        ptrs = []
        for t in shards:
            if isinstance(t, int):
                ptrs.append(t)
            else:
                if _tcode(t) != self.dtype or t.numel() != want or not t.is_contiguous():
                    raise ValueError("every shard must be a contiguous 2^(len - k) vector of "
                                     "the Hamiltonian's precision")
                ptrs.append(_ptr(t).value)
        arr = (C.c_void_p * n)(*ptrs)
        _lib.call("rp_apply_shard", self._h, k, rank, arr, _ptr(out), 1 if accumulate else 0)
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().rp_ham_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def evolve(ham, psi, t, beta=0.0, krydim=5, tol=None, max_iters=0):
    """psi <- exp(-(beta + i t) H) psi in place (State::evolve, inc/state.h:415-424).

    tol defaults to the machine epsilon of the state's precision, as
    Krylov::evolve's default (inc/algo.h:267-269)."""
    if _tcode(psi) != ham.dtype:
        raise ValueError("state precision does not match the Hamiltonian's")
    if tol is None:
        tol = float(np.finfo(np.float32 if ham.dtype == RP_C64 else np.float64).eps)
    st = _lib.EvolveStats()
    _lib.call("rp_evolve", ham.handle, _ptr(psi), float(t), float(beta), int(krydim),
              float(tol), int(max_iters), C.byref(st))
    return {k: getattr(st, k) for k, _ in _lib.EvolveStats._fields_}


def ground_state(ham, krydim=5, eps=None, maxiter=0, seed=0):
    """(energy, state) of the lowest eigenvalue of a Hermitian H by the
    reference's restarted Lanczos (Krylov::ground_state, inc/algo.h:180-257):
    from a random state, krydim Lanczos steps without reorthogonalisation,
    the tridiagonal eigenproblem on the host, restart from the Ritz vector
    until beta_0 <= eps (default 10 machine epsilons) or maxiter iterations
    (0 = no limit).  Vectors and H.psi on the GPU."""
    import torch
    from scipy.linalg import eigh_tridiagonal
    m = int(krydim)
    if m < 2:
        raise ValueError("krydim must be at least 2")
    prec = np.float32 if ham.dtype == RP_C64 else np.float64
    if eps is None:
        eps = 10 * float(np.finfo(prec).eps)
    v0 = random_state(ham.len, "c64" if ham.dtype == RP_C64 else "c128", seed=seed)
    numiter = 0
    while True:
        V = [v0]
        alpha, beta = [], []
        for i in range(m):
            w = torch.empty_like(v0)
            ham.apply(w, V[i])
            alpha.append(dot(V[i], w).real)
            if i == m - 1:
                break
            axpy(w, -alpha[i], V[i])
            if i:
                axpy(w, -beta[i - 1], V[i - 1])
            b = norm(w)
            if b == 0.0:          # invariant subspace: the Ritz values are exact
                break
            beta.append(b)
            scale(w, 1.0 / b)
            V.append(w)
        k = len(alpha)
        evals, evecs = eigh_tridiagonal(np.array(alpha), np.array(beta[:k - 1]))
        idx = int(np.argmin(evals))
        g = torch.zeros_like(v0)
        for i in range(k):
            axpy(g, float(evecs[i, idx]), V[i])
        scale(g, 1.0 / norm(g))
        numiter += 1
        v0 = g
        if not (beta and beta[0] > eps and (not maxiter or numiter < maxiter)):
            return float(evals[idx]), g


def ipc_export(t):
    """A device tensor (or raw device pointer) as (64-byte CUDA IPC handle of
    its allocation, offset) for another process on this node."""
    h = _lib.IpcHandle()
    _lib.call("rp_ipc_export", t if isinstance(t, int) else _ptr(t), C.byref(h))
    return bytes(h.handle), int(h.offset)


def ipc_open(handle):
    """The device pointer of another process's exported tensor (an
    ``ipc_export`` result), peer access enabled; release with ``ipc_close``."""
    data, offset = handle
    h = _lib.IpcHandle()
    C.memmove(h.handle, data, 64)
    h.offset = offset
    p = C.c_void_p()
    _lib.call("rp_ipc_open", C.byref(h), C.byref(p))
    return p.value


def ipc_close(ptr):
    _lib.call("rp_ipc_close", ptr)


def dot(a, b):
    """<a|b> (GPUImpl::vec_prod), FP64 compensated."""
    out = (C.c_double * 2)()
    _lib.call("rp_vec_dot", _tcode(a), a.numel(), _ptr(a), _ptr(b), out)
    return complex(out[0], out[1])


def norm(v):
    out = C.c_double()
    _lib.call("rp_vec_norm", _tcode(v), v.numel(), _ptr(v), C.byref(out))
    return out.value


def axpy(y, a, x):
    """y += a x."""
    a = complex(a)
    _lib.call("rp_vec_axpy", _tcode(y), y.numel(), _ptr(y), a.real, a.imag, _ptr(x))
    return y


def scale(v, a):
    a = complex(a)
    _lib.call("rp_vec_scale", _tcode(v), v.numel(), _ptr(v), a.real, a.imag)
    return v


def copy(dst, src):
    _lib.call("rp_vec_copy", _tcode(dst), _ptr(dst), _tcode(src), _ptr(src), dst.numel())
    return dst


def random_state(length, dtype="c128", seed=0, normalize=True, device="cuda"):
    """Complex Gaussian vector of 2^length entries made on the GPU (counter-based,
    deterministic per seed), optionally normalised (GPUImpl::init_random)."""
    import torch
    code = dtype_code(dtype)
    t = torch.empty(1 << length, dtype=torch.complex64 if code == RP_C64 else torch.complex128,
                    device=device)
    _lib.call("rp_vec_random", code, t.numel(), _ptr(t), int(seed))
    if normalize:
        scale(t, 1.0 / norm(t))
    return t


class BatchOTOC:
    """Many independent OTOC problems (disorder realisations x states, uneven
    qubit counts) run by one persistent launch per time step (rp_batch_*).

    problems: list of dicts with keys len, bits, coeff, w (bits, coeff),
    v (bits, coeff), psi0 (complex64 CUDA tensor) and optionally tile (8..12),
    team (CTAs per problem: 1, 2, 4, 8 or 16) and path ('batched', the
    default, or 'single': the autotuner found the single-problem path faster
    for this shape, so the problem runs alone on the whole GPU through
    ``otoc`` after the batched launches).  FP32 vectors, FP64 Krylov
    internals (the mixed-precision form)."""

    def __init__(self, problems, krydim=16, tol=1.2e-7, max_restarts=16):
        self.n = len(problems)
        self.krydim, self.tol = int(krydim), float(tol)
        self._single = [i for i, p in enumerate(problems) if p.get("path") == "single"]
        self._batched = [i for i, p in enumerate(problems) if p.get("path") != "single"]
        self._singles = []
        for i in self._single:
            p = problems[i]
            if _tcode(p["psi0"]) != RP_C64:
                raise ValueError("batched states are complex64")
            self._singles.append((Hamiltonian(p["len"], p["bits"], p["coeff"], "c64"),
                                  Hamiltonian(p["len"], *p["w"], "c64"),
                                  Hamiltonian(p["len"], *p["v"], "c64"), p["psi0"]))
        self._h = None
        if self._batched:
            self._create([problems[i] for i in self._batched], krydim, tol, max_restarts)

    def _create(self, problems, krydim, tol, max_restarts):
        n = len(problems)
        self._keep = problems
        lens = (C.c_int * n)(*[int(p["len"]) for p in problems])
        self._bits = [np.ascontiguousarray(p["bits"], dtype=np.uint64) for p in problems]
        self._coeff = [np.ascontiguousarray(p["coeff"], dtype=np.complex128).view(np.float64)
                       for p in problems]
        nterms = (C.c_int64 * n)(*[len(b) for b in self._bits])
        bitp = (C.POINTER(C.c_uint64) * n)(*[b.ctypes.data_as(C.POINTER(C.c_uint64))
                                             for b in self._bits])
        coefp = (C.POINTER(C.c_double) * n)(*[c.ctypes.data_as(C.POINTER(C.c_double))
                                              for c in self._coeff])
        wb = (C.c_uint64 * n)(*[int(np.asarray(p["w"][0]).ravel()[0]) for p in problems])
        vb = (C.c_uint64 * n)(*[int(np.asarray(p["v"][0]).ravel()[0]) for p in problems])
        wc = (C.c_double * (2 * n))()
        vc = (C.c_double * (2 * n))()
        for i, p in enumerate(problems):
            a = complex(np.asarray(p["w"][1]).ravel()[0])
            b = complex(np.asarray(p["v"][1]).ravel()[0])
            wc[2 * i], wc[2 * i + 1] = a.real, a.imag
            vc[2 * i], vc[2 * i + 1] = b.real, b.imag
        for p in problems:
            if _tcode(p["psi0"]) != RP_C64:
                raise ValueError("batched states are complex64")
        psis = (C.c_void_p * n)(*[p["psi0"].data_ptr() for p in problems])
        tiles = (C.c_int * n)(*[int(p.get("tile", 0)) for p in problems])
        teams = (C.c_int * n)(*[int(p.get("team", 0)) for p in problems])
        h = C.c_void_p()
        _lib.call("rp_batch_create_ex", C.byref(h), n, lens, nterms, bitp, coefp, wb, wc, vb, vc,
                  psis, tiles, teams, int(krydim), float(tol), int(max_restarts))
        self._h = h
        self._nb = n

    def run(self, times, use_graph=True):
        """Returns (F[n, ntimes] complex, applies[n, ntimes]): the batched
        problems by one persistent launch per time step (and team size),
        captured in a CUDA graph when use_graph, then the single-path ones."""
        times = np.ascontiguousarray(times, dtype=np.float64)
        k = len(times)
        Fall = np.zeros((self.n, k), dtype=np.complex128)
        apall = np.zeros((self.n, k), np.int32)
        if self._h is not None:
            F = np.zeros(2 * self._nb * k)
            ap = np.zeros(self._nb * k, np.int32)
            _lib.call("rp_batch_otoc", self._h, k, times.ctypes.data_as(C.POINTER(C.c_double)),
                      F.ctypes.data_as(C.POINTER(C.c_double)),
                      ap.ctypes.data_as(C.POINTER(C.c_int)), 1 if use_graph else 0)
            Fall[self._batched] = F.view(np.complex128).reshape(self._nb, k)
            apall[self._batched] = ap.reshape(self._nb, k)
        for i, (ham, w, v, psi0) in zip(self._single, self._singles):
            for j, t in enumerate(times):
                val, a = otoc(ham, w, v, psi0, [t], self.krydim, self.tol)
                Fall[i, j] = val[0]
                apall[i, j] = a
        return Fall, apall

    def probe(self, napplies=2):
        """Device ms of one launch doing napplies H.psi products per batched
        problem."""
        if self._h is None:
            raise ValueError("no problem of this batch runs on the batched path")
        ms = C.c_double()
        _lib.call("rp_batch_probe", self._h, int(napplies), C.byref(ms))
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().rp_batch_destroy(self._h)
            self._h = None
        for trio in getattr(self, "_singles", []):
            for h in trio[:3]:
                h.close()
        self._singles = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def otoc_block(ham_ll, ham_rr, op, psi0, times, krydim=5, tol=None):
    """The parity-block OTOC of examples/syk.cc (OTOC::evolve, lines 270-283)
    at beta = 0 on one block of N/2 - 1 qubits: s = op psi0; e^{-iH_RR t};
    e^{+iH_LL t}; op; e^{-iH_RR t}; e^{+iH_LL t}; F(t) = <psi0|s>, with op a
    Hamiltonian holding the LR block of the perturbing Majorana (b_{N-2} in
    the example).  Returns (F values, H.psi count of the evolves)."""
    import torch
    vals, applies = [], 0
    a = torch.empty_like(psi0)
    b = torch.empty_like(psi0)
    for t in times:
        op.apply(a, psi0)
        applies += evolve(ham_rr, a, t, 0.0, krydim, tol)["applies"]
        applies += evolve(ham_ll, a, -t, 0.0, krydim, tol)["applies"]
        op.apply(b, a)
        applies += evolve(ham_rr, b, t, 0.0, krydim, tol)["applies"]
        applies += evolve(ham_ll, b, -t, 0.0, krydim, tol)["applies"]
        vals.append(dot(psi0, b))
    return np.array(vals), applies


def otoc(ham, w, v, psi0, times, krydim=5, tol=None):
    """F(t) = <psi0| W(t) V W(t) V |psi0> at beta = 0, in the operation order of
    examples/simple-syk-krylov.cc:42-57 (psi = V psi0; e^{-iHt}; W; e^{iHt};
    V; e^{-iHt}; W; e^{iHt}; <psi0|psi>).  w and v are Hamiltonian objects of
    single Majorana strings.  Returns (values, total H.psi count)."""
    import torch
    vals = []
    applies = 0
    psi = torch.empty_like(psi0)
    tmp = torch.empty_like(psi0)
    for t in times:
        v.apply(psi, psi0)
        for op, tt in ((w, t), (v, -t), (w, t), (None, -t)):
            applies += evolve(ham, psi, tt, 0.0, krydim, tol)["applies"]
            if op is not None:
                op.apply(tmp, psi)
                psi, tmp = tmp, psi
        vals.append(dot(psi0, psi))
    return np.array(vals), applies
