"""CPU oracle for the REAPERS hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker: only tests/, ``__graft_entry__.smoke()`` and the
cpu_baseline leg of ``bench.py`` import it.  The product (``reapers_b200``)
never calls it and has no CPU fallback.

Two layers:

* ``librporacle.so`` -- the C restatement in ``rp_oracle.c`` (Pauli apply,
  the reference's MGS restarted Krylov, Higham's Pade-13 expm, Jordan-Wigner
  Majoranas), wrapped with ctypes below.  Each C function cites the reference
  file:line it follows.
* ``_ref/ref_driver`` -- the reference library itself compiled from its own
  headers against ``eigen_shim`` (built only where the reference checkout is
  present; the built binary is kept out of version control and travels with
  the working tree).  ``RefDriver``
  runs it through files.

Parity of the restatement is pinned against the reference driver and against
the reference's own unit-test known answers (tests/ops.cc) in
tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "librporacle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", _HERE, "librporacle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(path)
        u64p = C.POINTER(C.c_uint64)
        dp = C.POINTER(C.c_double)
        L.or_spin_mul.argtypes = [C.c_uint64, dp, C.c_uint64, dp, u64p, dp]
        L.or_majorana.argtypes = [C.c_int, C.c_int, C.c_int, u64p, dp]
        L.or_syk_scale.argtypes = [C.c_int, C.c_double, C.c_double]
        L.or_syk_scale.restype = C.c_double
        L.or_syk_terms.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), dp, u64p, dp]
        L.or_apply.argtypes = [C.c_int, C.c_int64, u64p, dp, dp, dp, C.c_int]
        L.or_expm.argtypes = [C.c_int, dp, dp]
        L.or_expm.restype = C.c_int
        L.or_krylov_evolve.argtypes = [C.c_int, C.c_int64, u64p, dp, dp, C.c_double,
                                       C.c_double, C.c_int, C.c_double, C.c_int,
                                       C.POINTER(EvolveStats)]
        L.or_krylov_evolve.restype = C.c_int
        L.or_dense_matrix.argtypes = [C.c_int, C.c_int64, u64p, dp, dp]
        _LIB = L
    return _LIB


class EvolveStats(C.Structure):
    _fields_ = [("restarts", C.c_int), ("applies", C.c_int), ("passes", C.c_int),
                ("prods", C.c_int), ("breakdown", C.c_int), ("last_err", C.c_double)]


def _u64(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def split_bits(bits):
    """Interleaved SpinOp bits -> (xmask, zmask) arrays (bit 2i = X_i, 2i+1 = Z_i)."""
    bits = np.asarray(bits, dtype=np.uint64)
    x = np.zeros(bits.shape, np.uint64)
    z = np.zeros(bits.shape, np.uint64)
    for i in range(32):
        x |= ((bits >> np.uint64(2 * i)) & np.uint64(1)) << np.uint64(i)
        z |= ((bits >> np.uint64(2 * i + 1)) & np.uint64(1)) << np.uint64(i)
    return x, z


def majorana(N, n, standard_gamma=True):
    b = C.c_uint64()
    c = np.zeros(2)
    lib().or_majorana(N, n, 1 if standard_gamma else 0, C.byref(b), _dp(c))
    return int(b.value), complex(c[0], c[1])


def spin_mul(a_bits, a, b_bits, b):
    ca = np.array([a.real, a.imag])
    cb = np.array([b.real, b.imag])
    ob = C.c_uint64()
    oc = np.zeros(2)
    lib().or_spin_mul(a_bits, _dp(ca), b_bits, _dp(cb), C.byref(ob), _dp(oc))
    return int(ob.value), complex(oc[0], oc[1])


def syk_scale(N, sp=0.0, J=1.0):
    return lib().or_syk_scale(N, sp, J)


def syk_terms(N, quartets, couplings):
    """Quartic SYK terms J_q b_i b_j b_k b_l (non-block JW form)."""
    q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
    J = np.ascontiguousarray(couplings, dtype=np.float64)
    T = q.shape[0]
    bits = np.zeros(T, np.uint64)
    coeff = np.zeros(2 * T)
    lib().or_syk_terms(N, T, q.ctypes.data_as(C.POINTER(C.c_int)), _dp(J), _u64(bits),
                       _dp(coeff))
    return bits, coeff.view(np.complex128)


def apply_at(bits, coeff, idx, fetch):
    """(H vec)[i] for the output indices idx only: the sum of or_apply
    (inc/cpuimpl.h:747-753 with SpinOp::apply, inc/ops.h:421-440),
    out[i] = sum_k c_k (-1)^popc(z_k & (i ^ x_k)) vec[i ^ x_k] in list order,
    with fetch(j) returning vec at the int64 index array j as complex128 --
    spot checks of states too large for the CPU apply."""
    x, z = split_bits(bits)
    idx = np.asarray(idx, dtype=np.uint64)
    c = np.asarray(coeff, dtype=np.complex128)
    src = idx[:, None] ^ x[None, :]
    minus = (np.bitwise_count(z[None, :] & src) & np.uint8(1)).astype(bool)
    vals = np.asarray(fetch(src.reshape(-1).astype(np.int64)), dtype=np.complex128).reshape(src.shape)
    out = np.zeros(idx.shape[0], dtype=np.complex128)
    for k in range(c.shape[0]):
        out += np.where(minus[:, k], -c[k], c[k]) * vals[:, k]
    return out


def apply(length, bits, coeff, vec, out=None):
    """H.vec, complex128 in and out."""
    bits = np.ascontiguousarray(bits, dtype=np.uint64)
    c = np.ascontiguousarray(coeff, dtype=np.complex128).view(np.float64)
    v = np.ascontiguousarray(vec, dtype=np.complex128)
    acc = 1 if out is not None else 0
    if out is None:
        out = np.zeros(1 << length, np.complex128)
    lib().or_apply(length, len(bits), _u64(bits), _dp(c), _dp(v.view(np.float64)),
                   _dp(out.view(np.float64)), acc)
    return out


def expm(A):
    A = np.asfortranarray(A, dtype=np.complex128)
    n = A.shape[0]
    E = np.zeros((n, n), np.complex128, order="F")
    rc = lib().or_expm(n, _dp(A.reshape(-1, order="F").view(np.float64)),
                       _dp(E.reshape(-1, order="F").view(np.float64)))
    if rc:
        raise RuntimeError("or_expm failed")
    return E


def evolve(length, bits, coeff, psi, t, beta=0.0, krydim=5, tol=np.finfo(float).eps,
           max_iters=0):
    """exp(-(beta + i t) H) psi by the reference's restarted Krylov (algo.h:267-365).

    Returns (result, stats dict)."""
    bits = np.ascontiguousarray(bits, dtype=np.uint64)
    c = np.ascontiguousarray(coeff, dtype=np.complex128).view(np.float64)
    out = np.array(psi, dtype=np.complex128, copy=True)
    st = EvolveStats()
    rc = lib().or_krylov_evolve(length, len(bits), _u64(bits), _dp(c),
                                _dp(out.view(np.float64)), float(t), float(beta),
                                int(krydim), float(tol), int(max_iters), C.byref(st))
    if rc:
        raise RuntimeError("or_krylov_evolve failed")
    return out, {"restarts": st.restarts, "applies": st.applies, "passes": st.passes,
                 "prods": st.prods, "breakdown": st.breakdown, "last_err": st.last_err}


def dense_matrix(length, bits, coeff):
    D = 1 << length
    bits = np.ascontiguousarray(bits, dtype=np.uint64)
    c = np.ascontiguousarray(coeff, dtype=np.complex128).view(np.float64)
    M = np.zeros(D * D, np.complex128)
    lib().or_dense_matrix(length, len(bits), _u64(bits), _dp(c), _dp(M.view(np.float64)))
    return M.reshape(D, D, order="F")


def otoc(length, bits, coeff, w, v, psi0, times, krydim=5, tol=np.finfo(float).eps):
    """F(t) = <psi0| W(t) V W(t) V |psi0> in the order of
    examples/simple-syk-krylov.cc:42-57 at beta = 0.  w and v are (bits, coeff)."""
    out = []
    for t in times:
        psi = apply(length, v[0], v[1], psi0)
        psi, _ = evolve(length, bits, coeff, psi, t, 0.0, krydim, tol)
        psi = apply(length, w[0], w[1], psi)
        psi, _ = evolve(length, bits, coeff, psi, -t, 0.0, krydim, tol)
        psi = apply(length, v[0], v[1], psi)
        psi, _ = evolve(length, bits, coeff, psi, t, 0.0, krydim, tol)
        psi = apply(length, w[0], w[1], psi)
        psi, _ = evolve(length, bits, coeff, psi, -t, 0.0, krydim, tol)
        out.append(np.vdot(psi0, psi))
    return np.array(out)


# ---------------------------------------------------------------------------
# The reference itself (prebuilt oracle/_ref/ref_driver)
# ---------------------------------------------------------------------------
REF_DRIVER = os.path.join(_HERE, "_ref", "ref_driver")
# the same driver for x86-64-v4 (AVX-512) hosts: the timed CPU baseline there
REF_DRIVER_V4 = os.path.join(_HERE, "_ref", "ref_driver_v4")
_V4_FLAGS = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def ref_available():
    return os.path.exists(REF_DRIVER)


def host_is_v4():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split(":", 1)[1].split())
                    return all(x in fl for x in _V4_FLAGS)
    except OSError:
        pass
    return False


def bench_driver():
    """The reference driver built for this host's ISA level (x86-64-v4 where
    the CPU has AVX-512, else the portable x86-64-v3 build) and its name."""
    if host_is_v4() and os.path.exists(REF_DRIVER_V4):
        return REF_DRIVER_V4, "x86-64-v4"
    return REF_DRIVER, "x86-64-v3"


def write_terms(path, length, bits, coeff):
    bits = np.asarray(bits, dtype=np.uint64)
    coeff = np.asarray(coeff, dtype=np.complex128)
    rec = np.zeros(len(bits), dtype=[("bits", "<u8"), ("re", "<f8"), ("im", "<f8")])
    rec["bits"] = bits
    rec["re"] = coeff.real
    rec["im"] = coeff.imag
    with open(path, "wb") as f:
        f.write(np.int64(len(bits)).tobytes())
        f.write(np.int32(length).tobytes())
        f.write(rec.tobytes())


def read_terms(path):
    with open(path, "rb") as f:
        T = int(np.frombuffer(f.read(8), np.int64)[0])
        length = int(np.frombuffer(f.read(4), np.int32)[0])
        rec = np.frombuffer(f.read(24 * T),
                            dtype=[("bits", "<u8"), ("re", "<f8"), ("im", "<f8")])
    return length, rec["bits"].copy(), rec["re"] + 1j * rec["im"]


def write_vec(path, v):
    v = np.ascontiguousarray(v, dtype=np.complex128)
    with open(path, "wb") as f:
        f.write(np.int64(len(v)).tobytes())
        f.write(v.tobytes())


def read_vec(path):
    with open(path, "rb") as f:
        D = int(np.frombuffer(f.read(8), np.int64)[0])
        return np.frombuffer(f.read(16 * D), np.complex128).copy()


class RefDriver:
    """Runs the reference library (compiled CPU build) through files."""

    def __init__(self, threads=None):
        if not ref_available():
            raise FileNotFoundError(REF_DRIVER)
        self.env = dict(os.environ)
        if threads:
            self.env["OMP_NUM_THREADS"] = str(threads)
        self.tmp = tempfile.mkdtemp(prefix="rpref_")

    def _run(self, *args):
        r = subprocess.run([REF_DRIVER, *map(str, args)], check=True, env=self.env,
                           capture_output=True, text=True)
        return r.stdout

    def syk(self, N, sp, J, seed):
        p = os.path.join(self.tmp, "syk.terms")
        self._run("syk", N, sp, J, seed, p)
        return read_terms(p)

    def majorana(self, N):
        p = os.path.join(self.tmp, "maj.terms")
        self._run("majorana", N, p)
        return read_terms(p)

    def majorana_block(self, N):
        """Parity-block Majoranas: (len, bits, coeff) with records LR_0, RL_0, LR_1, ..."""
        p = os.path.join(self.tmp, "majb.terms")
        self._run("majorana_block", N, p)
        return read_terms(p)

    def syk_block(self, N, sp, J, seed):
        """SYK::gen_ham(mt19937(seed)) in parity-block form: (LL terms, RR terms)."""
        a, b = os.path.join(self.tmp, "ll.terms"), os.path.join(self.tmp, "rr.terms")
        self._run("syk_block", N, sp, J, seed, a, b)
        return read_terms(a), read_terms(b)

    def otoc_block(self, length, LL, RR, op, psi0, times, krydim, tol):
        """examples/syk.cc's OTOC::evolve sequence at beta = 0 on one parity block."""
        fl, fr, fo = (os.path.join(self.tmp, n) for n in ("ob_ll", "ob_rr", "ob_op"))
        fv, fout = os.path.join(self.tmp, "ob_v"), os.path.join(self.tmp, "ob_out")
        write_terms(fl, length, *LL)
        write_terms(fr, length, *RR)
        write_terms(fo, length, *op)
        write_vec(fv, psi0)
        self._run("otoc_block", fl, fr, fo, fv, fout, krydim, tol, *times)
        with open(fout, "rb") as f:
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            v = np.frombuffer(f.read(16 * n), np.float64)
        return v[0::2] + 1j * v[1::2]

    def roundtrip(self, length, bits, coeff):
        p, q = os.path.join(self.tmp, "rt.in"), os.path.join(self.tmp, "rt.out")
        write_terms(p, length, bits, coeff)
        self._run("roundtrip", p, q)
        return read_terms(q)

    def apply(self, length, bits, coeff, vec):
        p, i, o = (os.path.join(self.tmp, n) for n in ("a.terms", "a.in", "a.out"))
        write_terms(p, length, bits, coeff)
        write_vec(i, vec)
        self._run("apply", p, i, o)
        return read_vec(o)

    def evolve(self, length, bits, coeff, psi, t, beta=0.0, krydim=5,
               tol=np.finfo(float).eps, max_iters=0):
        p, i, o = (os.path.join(self.tmp, n) for n in ("e.terms", "e.in", "e.out"))
        write_terms(p, length, bits, coeff)
        write_vec(i, psi)
        out = self._run("evolve", p, i, o, repr(float(t)), repr(float(beta)), krydim,
                        repr(float(tol)), max_iters)
        return read_vec(o), json.loads(out)

    def otoc(self, length, bits, coeff, w, v, psi0, times, krydim=5,
             tol=np.finfo(float).eps):
        p, pw, pv, i, o = (os.path.join(self.tmp, n)
                           for n in ("o.terms", "o.w", "o.v", "o.in", "o.out"))
        write_terms(p, length, bits, coeff)
        write_terms(pw, length, *w)
        write_terms(pv, length, *v)
        write_vec(i, psi0)
        out = self._run("otoc", p, pw, pv, i, o, krydim, repr(float(tol)),
                        *[repr(float(t)) for t in times])
        with open(o, "rb") as f:
            n = int(np.frombuffer(f.read(8), np.int64)[0])
            vals = np.frombuffer(f.read(16 * n), np.complex128).copy()
        return vals, json.loads(out)

    def bench_apply(self, length, bits, coeff, reps):
        p = os.path.join(self.tmp, "b.terms")
        write_terms(p, length, bits, coeff)
        return json.loads(self._run("bench_apply", p, reps))
