"""Pauli-string algebra and model Hamiltonians (host side, numpy).

Encoding as SpinOp (inc/ops.h:117-165): bit 2i = X on site i, bit 2i+1 = Z;
sigma_y is the real product sx.sz with the factor i kept in the coefficient.
The product of two strings a.b has bits a ^ b and the carry-over sign of
the four products sz.sx, sz.sy, sy.sx, sy.sy (inc/ops.h:151-161), which is
(-1)^popcount(Z(a) & X(b)).

Majoranas follow the non-block Jordan-Wigner form of FermionOpNonBlockForm
(inc/fermions.h:276-296); SYK couplings use the scale of SYK's constructor
(inc/syk.h:104-119) and quartets i > j > k > l in gen_ham's loop order
(inc/syk.h:244-257).
"""
from __future__ import annotations

import functools
import math

import numpy as np

_X = np.uint64(0x5555555555555555)
_Z = np.uint64(0xAAAAAAAAAAAAAAAA)


def xmask(bits):
    """X mask of interleaved bits (compress even bits)."""
    b = np.asarray(bits, dtype=np.uint64)
    out = np.zeros_like(b)
    for i in range(32):
        out |= ((b >> np.uint64(2 * i)) & np.uint64(1)) << np.uint64(i)
    return out


def zmask(bits):
    b = np.asarray(bits, dtype=np.uint64)
    out = np.zeros_like(b)
    for i in range(32):
        out |= ((b >> np.uint64(2 * i + 1)) & np.uint64(1)) << np.uint64(i)
    return out


def _parity64(v):
    v = np.asarray(v, dtype=np.uint64).copy()
    for s in (32, 16, 8, 4, 2, 1):
        v ^= v >> np.uint64(s)
    return (v & np.uint64(1)).astype(np.int64)


def mul(a_bits, a_coeff, b_bits, b_coeff):
    """Product of Pauli strings (vectorised): (bits, coeff) of a.b."""
    a_bits = np.asarray(a_bits, dtype=np.uint64)
    b_bits = np.asarray(b_bits, dtype=np.uint64)
    # Z part of a (odd bits, shifted onto even positions) against X part of b
    za = (a_bits & _Z) >> np.uint64(1)
    xb = b_bits & _X
    sign = 1.0 - 2.0 * _parity64(za & xb)
    return a_bits ^ b_bits, sign * np.asarray(a_coeff) * np.asarray(b_coeff)


def sigma(kind, site):
    """Single-site sigma_x / sigma_y / sigma_z as (bits, coeff)."""
    code = {"x": 1, "z": 2, "y": 3}[kind]
    return np.uint64(code) << np.uint64(2 * site), (1j if kind == "y" else 1.0 + 0j)


def majorana(N, n, standard_gamma=True):
    """b_n = {sy or sz}((n-1)/2) . prod_{(n+1)/2 <= i < N/2} sx(i), / sqrt 2."""
    b, c = np.uint64(0), 1.0 + 0j
    for i in range((n + 1) // 2, N // 2):
        b, c = mul(b, c, *sigma("x", i))
    if n != 0:
        b, c = mul(b, c, *sigma("y" if n & 1 else "z", (n - 1) // 2))
    if standard_gamma:
        c = c * (1.0 / math.sqrt(2.0))
    return np.uint64(b), complex(c)


def majoranas(N, standard_gamma=True):
    out = [majorana(N, n, standard_gamma) for n in range(N)]
    return np.array([o[0] for o in out], np.uint64), np.array([o[1] for o in out])


def syk_scale(N, k=0.0, J=1.0):
    """sqrt(6/N^3) J, divided by sqrt(p), p = 24 k / ((N-1)(N-2)(N-3)), if sparse."""
    s = math.sqrt(6.0 / (N * N * N)) * J
    if k != 0.0:
        p = k * 24 / ((N - 1) * (N - 2) * (N - 3))
        s /= math.sqrt(p)
    return s


def quartic_terms(N, quartets, couplings):
    """Terms J_q b_i b_j b_k b_l (products left to right), as (bits, coeff)."""
    q = np.asarray(quartets, dtype=np.int64).reshape(-1, 4)
    mb, mc = majoranas(N)
    bits = np.zeros(len(q), np.uint64)
    coeff = np.asarray(couplings, dtype=np.float64).astype(np.complex128)
    for f in range(4):
        bits, coeff = mul(bits, coeff, mb[q[:, f]], mc[q[:, f]])
    return bits, coeff


@functools.lru_cache(maxsize=8)
def _all_quartets(N):
    out = [(i, j, k, l) for i in range(N) for j in range(i) for k in range(j) for l in range(k)]
    a = np.array(out, dtype=np.int64).reshape(-1, 4)
    a.setflags(write=False)
    return a


def all_quartets(N):
    """Quartets i > j > k > l in gen_ham's loop order (i outermost)."""
    return _all_quartets(N)


def _unrank_quartets(N, ranks):
    """Map ranks in [0, C(N,4)) to quartets in gen_ham's loop order."""
    q = all_quartets(N) if N <= 64 else None
    return q[np.asarray(ranks)]


def dense_syk(N, seed=0, J=1.0):
    """Dense SYK: all C(N,4) quartets, couplings N(0,1) * sqrt(6/N^3) J."""
    rng = np.random.default_rng(seed)
    q = all_quartets(N)
    Jq = rng.standard_normal(len(q)) * syk_scale(N, 0.0, J)
    return quartic_terms(N, q, Jq)


def sparse_syk_couplings(N, k=8, seed=0, J=1.0):
    """(quartets, couplings) of the sparse SYK model below."""
    rng = np.random.default_rng(seed)
    total = math.comb(N, 4)
    T = int(round(k * N))
    ranks = np.sort(rng.choice(total, size=T, replace=False))
    q = _unrank_quartets(N, ranks)
    Jq = rng.standard_normal(T) * syk_scale(N, k, J)
    return q, Jq


def sparse_syk(N, k=8, seed=0, J=1.0):
    """Sparse SYK with exactly k*N quartets drawn uniformly without replacement,
    kept in gen_ham's loop order, couplings N(0,1) * scale of SYK(N, k, J)."""
    return quartic_terms(N, *sparse_syk_couplings(N, k, seed, J))


def sparse_syk_block(N, k=8, seed=0, J=1.0):
    """The same model (same quartets and couplings) in parity-block form:
    ((H_LL bits, coeff), (H_RR bits, coeff)) on N/2 - 1 qubits."""
    return quartic_terms_block(N, *sparse_syk_couplings(N, k, seed, J))


def majorana_block(N, n, standard_gamma=True):
    """The n-th Majorana in parity-block form, b_n = [[0, LR], [RL, 0]] on
    N/2 - 1 qubits (FermionOpBlockForm, inc/fermions.h:308-366): for
    n <= N - 2, LR = RL = the n-th non-block Majorana of N - 2 fermions without
    the 1/sqrt 2 (n = N - 2 gives sz(N/2 - 2)); for n = N - 1, LR = -i I and
    RL = i I.  Returns ((LR bits, coeff), (RL bits, coeff)), / sqrt 2 when
    standard_gamma."""
    if N < 4 or N & 1 or not 0 <= n < N:
        raise ValueError("need an even N >= 4 and 0 <= n < N")
    if n == N - 1:
        lr, rl = (np.uint64(0), -1j), (np.uint64(0), 1j)
    else:
        b, c = majorana(N - 2, n, standard_gamma=False)
        lr = rl = (b, c)
    f = 1.0 / math.sqrt(2.0) if standard_gamma else 1.0
    return (np.uint64(lr[0]), complex(lr[1]) * f), (np.uint64(rl[0]), complex(rl[1]) * f)


def _merge(bits, coeff):
    """Sum the coefficients of equal strings, in order of first occurrence
    (HostSumOps::operator+=, inc/cpuimpl.h:233-253)."""
    order, acc = [], {}
    for b, c in zip(np.asarray(bits, dtype=np.uint64).tolist(), np.asarray(coeff).tolist()):
        if b in acc:
            acc[b] += c
        else:
            acc[b] = c
            order.append(b)
    return np.array(order, np.uint64), np.array([acc[b] for b in order], np.complex128)


def quartic_terms_block(N, quartets, couplings):
    """Parity blocks of H = sum_q J_q b_i b_j b_k b_l (products left to right):
    H_LL = sum J_q LR_i RL_j LR_k RL_l and H_RR = sum J_q RL_i LR_j RL_k LR_l,
    each as (bits, coeff) on N/2 - 1 qubits with equal strings merged."""
    q = np.asarray(quartets, dtype=np.int64).reshape(-1, 4)
    blocks = [majorana_block(N, n) for n in range(N)]
    lr_b = np.array([blocks[n][0][0] for n in range(N)], np.uint64)
    lr_c = np.array([blocks[n][0][1] for n in range(N)])
    rl_b = np.array([blocks[n][1][0] for n in range(N)], np.uint64)
    rl_c = np.array([blocks[n][1][1] for n in range(N)])
    J = np.asarray(couplings, dtype=np.float64).astype(np.complex128)
    out = []
    for first, second in (((lr_b, lr_c), (rl_b, rl_c)), ((rl_b, rl_c), (lr_b, lr_c))):
        bits = np.zeros(len(q), np.uint64)
        coeff = J.copy()
        for f in range(4):
            src = first if f % 2 == 0 else second
            bits, coeff = mul(bits, coeff, src[0][q[:, f]], src[1][q[:, f]])
        out.append(_merge(bits, coeff))
    return out[0], out[1]


def xxz_chain(L, Jz=1.0, fields=None, J=1.0, periodic=False):
    """XXZ chain sum_i J (sx sx + sy sy) + Jz sz sz + h_i sz_i, open by default."""
    bits, coeff = [], []
    bonds = [(i, i + 1) for i in range(L - 1)] + ([(L - 1, 0)] if periodic and L > 2 else [])
    for a, b in bonds:
        for kind, c in (("x", J), ("y", J), ("z", Jz)):
            b1, c1 = mul(*sigma(kind, a), *sigma(kind, b))
            bits.append(int(b1))
            coeff.append(complex(c1) * c)
    if fields is not None:
        for i, h in enumerate(fields):
            b1, c1 = sigma("z", i)
            bits.append(int(b1))
            coeff.append(complex(c1) * h)
    return np.array(bits, np.uint64), np.array(coeff, np.complex128)
