#!/usr/bin/env python3
"""Generate the golden fixtures in this directory by running the reference
library itself (oracle/_ref/ref_driver: the REAPERS headers compiled as a CPU
program).  Run in a checkout where the reference is present:

    make -C oracle && python tests/golden/make_golden.py

Fixtures (numpy .npz):
  majorana_N{N}.npz        reference Majorana strings b_0..b_{N-1}, N = 4..20
  syk_dense_N8_seed5.npz   SYK::gen_ham(std::mt19937(5)) term list, N = 8
  dense_syk_N24.npz     dense SYK N = 24 (12 qubits, 10626 terms) from
                           SYK::gen_ham(std::mt19937(1)), psi0, and
                           State::evolve results at t = 0.5, 2.5, 5.0 (m = 20,
                           tol = 1e-12) with the reference's call counts
  apply_L10.npz            random terms, vector and State operator* output
  evolve_sparse_N20.npz    sparse SYK N = 20 (seeded project generator),
                           evolve at (t, beta) = (1.5, 0.25), m = 8
  otoc_N16.npz             dense SYK N = 16 from gen_ham(mt19937(3)),
                           F(t) at t = 0, 0.5, 1, 2 in the order of
                           examples/simple-syk-krylov.cc (m = 10, tol 1e-12)
  majorana_block_N{N}.npz  parity-block Majoranas (LR, RL records), N = 6..12
  syk_block_N12.npz        dense SYK N = 12 from gen_ham(mt19937(3)) in both
                           forms (full terms; H_LL, H_RR), and the parity-block
                           OTOC of examples/syk.cc at t = 0, 0.4, 1.1 with
                           op = LR of b_{N-2} (m = 10, tol 1e-12)
  dense_syk_N24_t10.npz    the dense SYK N = 24 evolve at all ten points
                           t = 0.5, 1.0, ..., 5.0 (m = 20, tol = 1e-12)
  evolve_sparse_N40.npz    sparse SYK N = 40 (20 qubits, k = 8, 320 terms,
                           seeded project generator), FP64 State::evolve to
                           t = 10 with m = 30 at the reference's default tol
                           (FP64 epsilon): its call counts, the final state at
                           4096 sampled indices plus the first and last, its
                           norm, and its projections onto 8 seeded random
                           vectors (a checksum of the whole state)
  evolve_sparse_N48.npz    the same for the sparse SYK N = 48 evolve workload
                           (24 qubits, k = 8, 384 terms, t = 10, m = 30, FP64),
                           with 4 projections (an hour of the reference's CPU
                           evolve on 8 threads)

Usage: make_golden.py [name ...] regenerates only the named fixtures (file
stems, e.g. dense_syk_N24_t10); without names, all of them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
import reapers_b200.syk as S  # noqa: E402


N40_SEED, N40_PSI_SEED, N40_PROBE_SEED = 4040, 4041, 4042
N48_SEED, N48_PSI_SEED, N48_PROBE_SEED = 4848, 4849, 4850


def n40_problem():
    """The 20-qubit evolve problem of evolve_sparse_N40.npz: Hamiltonian,
    start state and the probe vectors (all regenerated from seeds)."""
    L = 20
    bits, coeff = S.sparse_syk(40, k=8, seed=N40_SEED)
    rng = np.random.default_rng(N40_PSI_SEED)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    prng = np.random.default_rng(N40_PROBE_SEED)
    probes = prng.standard_normal((8, 1 << L)) + 1j * prng.standard_normal((8, 1 << L))
    idx = np.unique(np.concatenate([[0, (1 << L) - 1],
                                    prng.integers(0, 1 << L, size=4096)])).astype(np.int64)
    return L, bits, coeff, psi, probes, idx


def n48_problem():
    """The 24-qubit evolve problem of evolve_sparse_N48.npz (the sparse SYK
    N = 48 evolve workload: k = 8, 384 terms, m = 30, t = 10)."""
    L = 24
    bits, coeff = S.sparse_syk(48, k=8, seed=N48_SEED)
    rng = np.random.default_rng(N48_PSI_SEED)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    prng = np.random.default_rng(N48_PROBE_SEED)
    idx = np.unique(np.concatenate([[0, (1 << L) - 1],
                                    prng.integers(0, 1 << L, size=4096)])).astype(np.int64)
    return L, bits, coeff, psi, prng, idx


def probe_projections(prng, x, count=4):
    """<r_c|x> for `count` seeded complex Gaussian vectors r_c, drawn one at
    a time (a 24-qubit probe set would not fit in memory at once)."""
    out = []
    for _ in range(count):
        r = prng.standard_normal(len(x)) + 1j * prng.standard_normal(len(x))
        out.append(np.vdot(r, x))
    return np.array(out)


def make_sparse_n48(R):
    L, bits, coeff, psi, prng, idx = n48_problem()
    tol = float(np.finfo(np.float64).eps)
    o, st = R.evolve(L, bits, coeff, psi, 10.0, 0.0, 30, tol)
    np.savez_compressed(os.path.join(HERE, "evolve_sparse_N48.npz"), bits=bits, coeff=coeff,
                        len=L, t=10.0, beta=0.0, krydim=30, tol=tol, idx=idx, vals=o[idx],
                        norm=np.linalg.norm(o), proj=probe_projections(prng, o),
                        applies=st["applies"], prods=st["prods"], ref_seconds=st["seconds"],
                        seeds=np.array([N48_SEED, N48_PSI_SEED, N48_PROBE_SEED]))


def make_dense_t10(R):
    L, b, c = R.syk(24, 0.0, 1.0, 1)
    rng = np.random.default_rng(2024)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    times = [0.5 * k for k in range(1, 11)]
    outs, applies, prods = [], [], []
    for t in times:
        o, st = R.evolve(L, b, c, psi, t, 0.0, 20, 1e-12)
        outs.append(o)
        applies.append(st["applies"])
        prods.append(st["prods"])
    np.savez_compressed(os.path.join(HERE, "dense_syk_N24_t10.npz"), bits=b, coeff=c, len=L,
                        psi0=psi, times=np.array(times), out=np.array(outs),
                        applies=np.array(applies), prods=np.array(prods), krydim=20, tol=1e-12)


def make_sparse_n40(R):
    L, bits, coeff, psi, probes, idx = n40_problem()
    tol = float(np.finfo(np.float64).eps)
    o, st = R.evolve(L, bits, coeff, psi, 10.0, 0.0, 30, tol)
    np.savez_compressed(os.path.join(HERE, "evolve_sparse_N40.npz"), bits=bits, coeff=coeff,
                        len=L, t=10.0, beta=0.0, krydim=30, tol=tol, idx=idx, vals=o[idx],
                        norm=np.linalg.norm(o), proj=probes.conj() @ o,
                        applies=st["applies"], prods=st["prods"], ref_seconds=st["seconds"],
                        seeds=np.array([N40_SEED, N40_PSI_SEED, N40_PROBE_SEED]))


def main():
    R = O.RefDriver(threads=os.cpu_count())
    only = set(sys.argv[1:])
    if only:
        if "dense_syk_N24_t10" in only:
            make_dense_t10(R)
        if "evolve_sparse_N40" in only:
            make_sparse_n40(R)
        if "evolve_sparse_N48" in only:
            make_sparse_n48(R)
        return
    for N in range(4, 22, 2):
        L, b, c = R.majorana(N)
        np.savez_compressed(os.path.join(HERE, f"majorana_N{N}.npz"), bits=b, coeff=c)
    L, b, c = R.syk(8, 0.0, 1.0, 5)
    np.savez_compressed(os.path.join(HERE, "syk_dense_N8_seed5.npz"), bits=b, coeff=c, len=L)

    # dense SYK N = 24, reference generator
    L, b, c = R.syk(24, 0.0, 1.0, 1)
    rng = np.random.default_rng(2024)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    times = [0.5, 2.5, 5.0]
    outs, applies, prods = [], [], []
    for t in times:
        o, st = R.evolve(L, b, c, psi, t, 0.0, 20, 1e-12)
        outs.append(o)
        applies.append(st["applies"])
        prods.append(st["prods"])
    np.savez_compressed(os.path.join(HERE, "dense_syk_N24.npz"), bits=b, coeff=c, len=L,
                        psi0=psi, times=np.array(times), out=np.array(outs),
                        applies=np.array(applies), prods=np.array(prods), krydim=20, tol=1e-12)

    # apply: random terms with every coefficient kind
    rng = np.random.default_rng(7)
    L = 10
    bits = np.unique(rng.integers(0, 1 << (2 * L), size=60, dtype=np.uint64))
    coeff = rng.standard_normal(len(bits)) + 1j * rng.standard_normal(len(bits))
    coeff[::3] = coeff[::3].real
    coeff[1::3] = 1j * coeff[1::3].imag
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    rt_len, rt_bits, rt_coeff = R.roundtrip(L, bits, coeff)
    out = R.apply(L, bits, coeff, v)
    np.savez_compressed(os.path.join(HERE, "apply_L10.npz"), bits=bits, coeff=coeff, len=L,
                        vec=v, out=out, rt_bits=rt_bits, rt_coeff=rt_coeff)

    # evolve with imaginary time as well (sparse SYK from the project generator)
    L = 10
    bits, coeff = S.sparse_syk(20, k=4, seed=33)
    rng = np.random.default_rng(8)
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    v /= np.linalg.norm(v)
    o, st = R.evolve(L, bits, coeff, v, 1.5, 0.25, 8, 1e-12)
    np.savez_compressed(os.path.join(HERE, "evolve_sparse_N20.npz"), bits=bits, coeff=coeff,
                        len=L, psi0=v, t=1.5, beta=0.25, krydim=8, tol=1e-12, out=o,
                        applies=st["applies"], prods=st["prods"])

    # OTOC: the example's operator order, W = b_{N-1}, V = b_{N-2}
    N = 16
    L, b, c = R.syk(N, 0.0, 1.0, 3)
    _, mb, mc = R.majorana(N)
    w = (mb[N - 1:N], mc[N - 1:N])
    vv = (mb[N - 2:N - 1], mc[N - 2:N - 1])
    rng = np.random.default_rng(9)
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi /= np.linalg.norm(psi)
    times = [0.0, 0.5, 1.0, 2.0]
    vals, st = R.otoc(L, b, c, w, vv, psi, times, 10, 1e-12)
    np.savez_compressed(os.path.join(HERE, "otoc_N16.npz"), bits=b, coeff=c, len=L,
                        w_bits=w[0], w_coeff=w[1], v_bits=vv[0], v_coeff=vv[1], psi0=psi,
                        times=np.array(times), F=vals, krydim=10, tol=1e-12,
                        applies=st["applies"])
    # parity-block form: Majorana blocks, block Hamiltonians and the block OTOC
    for N in (6, 8, 10, 12):
        L, b, c = R.majorana_block(N)
        np.savez_compressed(os.path.join(HERE, f"majorana_block_N{N}.npz"), bits=b, coeff=c,
                            len=L)
    N = 12
    Lf, bf, cf = R.syk(N, 0.0, 1.0, 3)
    (Lb, llb, llc), (_, rrb, rrc) = R.syk_block(N, 0.0, 1.0, 3)
    rng = np.random.default_rng(12)
    psi = rng.standard_normal(1 << Lb) + 1j * rng.standard_normal(1 << Lb)
    psi /= np.linalg.norm(psi)
    (ob, oc), _ = S.majorana_block(N, N - 2)
    times = [0.0, 0.4, 1.1]
    F = R.otoc_block(Lb, (llb, llc), (rrb, rrc), (np.array([ob]), np.array([oc])), psi, times,
                     10, 1e-12)
    np.savez_compressed(os.path.join(HERE, "syk_block_N12.npz"), full_bits=bf, full_coeff=cf,
                        ll_bits=llb, ll_coeff=llc, rr_bits=rrb, rr_coeff=rrc, len=Lb, psi0=psi,
                        times=np.array(times), F=F, op_bits=np.array([ob]),
                        op_coeff=np.array([oc]), krydim=10, tol=1e-12)
    make_dense_t10(R)
    make_sparse_n40(R)
    make_sparse_n48(R)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
