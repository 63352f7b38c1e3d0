"""GPU parity of the CUDA hot path against the CPU oracle (oracle/rp_oracle.c).

Tolerances: FP64 (RP_C128) results within 1e-12 relative of the oracle --
the bar the plain path is held to; integer work (indices, signs, operation
counts) exact; FP32 (RP_C64) H.psi within 1e-5 relative.
"""
import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rand_terms(rng, L, T, kinds="mixed"):
    bits = np.unique(rng.integers(0, 1 << (2 * L), size=T, dtype=np.uint64))
    rng.shuffle(bits)
    n = len(bits)
    if kinds == "real":
        coeff = rng.standard_normal(n) + 0j
    elif kinds == "imag":
        coeff = 1j * rng.standard_normal(n)
    else:
        coeff = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        coeff[::3] = coeff[::3].real
        coeff[1::3] = 1j * coeff[1::3].imag
    return bits, coeff


def rand_vec(rng, L):
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    return v / np.linalg.norm(v)


def to_dev(v, dtype):
    t = torch.from_numpy(np.ascontiguousarray(v))
    if dtype == "c64":
        t = t.to(torch.complex64)
    return t.cuda()


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("L", [1, 2, 3, 4, 5, 6, 8, 10, 12, 14])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_apply_random_terms(cuda, L, dtype):
    rng = np.random.default_rng(100 + L)
    bits, coeff = rand_terms(rng, L, 3 * L + 7)
    v = rand_vec(rng, L)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    out = torch.empty(1 << L, dtype=torch.complex128 if dtype == "c128" else torch.complex64,
                      device=cuda)
    ham.apply(out, to_dev(v, dtype))
    ref = O.apply(L, bits, coeff, v)
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    assert relerr(out.cpu().numpy().astype(np.complex128), ref) < tol


@pytest.mark.parametrize("tile", [5, 6, 7, 8, 9, 10, 11, 12])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_apply_every_tile_exponent(cuda, tile, dtype):
    L = 13
    rng = np.random.default_rng(tile)
    bits, coeff = rand_terms(rng, L, 60)
    v = rand_vec(rng, L)
    ham = rb.Hamiltonian(L, bits, coeff, dtype, tile_exp=tile)
    assert ham.info()["tile_exp"] == tile
    x = to_dev(v, dtype)
    out = torch.empty_like(x)
    ham.apply(out, x)
    ref = O.apply(L, bits, coeff, v)
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    assert relerr(out.cpu().numpy().astype(np.complex128), ref) < tol
    # accumulate: out += H x
    ham.apply(out, x, accumulate=True)
    assert relerr(out.cpu().numpy().astype(np.complex128), 2 * ref) < tol


def test_apply_sparse_syk_and_identity(cuda):
    N, L = 32, 16
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=11)
    # add an identity term and a pure-Z term (diagonal, group xh = 0)
    bits = np.concatenate([bits, np.array([0, 2 << 8], np.uint64)])
    coeff = np.concatenate([coeff, np.array([0.3, -0.7j])])
    rng = np.random.default_rng(5)
    v = rand_vec(rng, L)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    out = torch.empty(1 << L, dtype=torch.complex128, device=cuda)
    ham.apply(out, to_dev(v, "c128"))
    assert relerr(out.cpu().numpy(), O.apply(L, bits, coeff, v)) < FP64_TOL


def test_apply_empty_hamiltonian(cuda):
    ham = rb.Hamiltonian(8, np.zeros(0, np.uint64), np.zeros(0, np.complex128), "c128")
    x = to_dev(rand_vec(np.random.default_rng(0), 8), "c128")
    out = torch.ones_like(x)
    ham.apply(out, x)
    assert torch.count_nonzero(out).item() == 0


def test_apply_rejects_bad_arguments(cuda):
    with pytest.raises(rb.RPError):
        rb.Hamiltonian(4, np.array([1 << 10], np.uint64), np.array([1.0 + 0j]), "c128")
    ham = rb.Hamiltonian(6, np.array([1], np.uint64), np.array([1.0 + 0j]), "c128")
    x = torch.zeros(64, dtype=torch.complex128, device=cuda)
    with pytest.raises(rb.RPError):
        ham.apply(x, x)


@pytest.mark.parametrize("L,N,k,t,beta,m", [
    (8, 16, 0, 0.7, 0.0, 6), (10, 20, 4, 2.0, 0.0, 10), (10, 20, 4, -1.5, 0.3, 8),
    (12, 24, 8, 5.0, 0.0, 20), (6, 12, 0, 3.0, 0.5, 5)])
def test_evolve_fp64_matches_oracle(cuda, L, N, k, t, beta, m):
    bits, coeff = rb.syk.sparse_syk(N, k=k, seed=L) if k else rb.syk.dense_syk(N, seed=L)
    v = rand_vec(np.random.default_rng(L), L)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = to_dev(v, "c128")
    st = rb.evolve(ham, x, t, beta, m, 1e-12)
    ref, st2 = O.evolve(L, bits, coeff, v, t, beta, m, 1e-12)
    assert relerr(x.cpu().numpy(), ref) < FP64_TOL
    for key in ("restarts", "applies", "passes", "prods", "breakdown"):
        assert st[key] == st2[key], (key, st, st2)


def test_evolve_fp32_mixed_precision(cuda):
    L, N = 12, 24
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=2)
    v = rand_vec(np.random.default_rng(9), L)
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    x = to_dev(v, "c64")
    rb.evolve(ham, x, 3.0, 0.0, 16, 1e-7)
    ref, _ = O.evolve(L, bits, coeff, v, 3.0, 0.0, 16, 1e-12)
    assert relerr(x.cpu().numpy().astype(np.complex128), ref) < 2e-5


def test_evolve_breakdown_on_invariant_subspace(cuda):
    # diagonal H on a basis state: H v = E v, breakdown at the first step
    L = 6
    bits = np.array([2 << 0, 2 << 2], np.uint64)   # sz(0) + sz(1)
    coeff = np.array([0.4, -1.1 + 0j])
    v = np.zeros(1 << L, np.complex128)
    v[5] = 1.0
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = to_dev(v, "c128")
    st = rb.evolve(ham, x, 1.3, 0.0, 5, 1e-12)
    ref, st2 = O.evolve(L, bits, coeff, v, 1.3, 0.0, 5, 1e-12)
    assert st["breakdown"] == st2["breakdown"] == 1
    assert relerr(x.cpu().numpy(), ref) < FP64_TOL


def test_evolve_zero_time_is_identity(cuda):
    L = 8
    bits, coeff = rb.syk.dense_syk(16, seed=1)
    v = rand_vec(np.random.default_rng(1), L)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = to_dev(v, "c128")
    st = rb.evolve(ham, x, 0.0, 0.0, 5)
    assert st["applies"] == 0
    assert np.array_equal(x.cpu().numpy(), v)


def test_vector_ops(cuda):
    rng = np.random.default_rng(4)
    a, b = rand_vec(rng, 14), rand_vec(rng, 14)
    ta, tb = to_dev(a, "c128"), to_dev(b, "c128")
    assert abs(rb.dot(ta, tb) - np.vdot(a, b)) < 1e-14
    assert abs(rb.norm(ta) - np.linalg.norm(a)) < 1e-14
    rb.axpy(ta, 0.5 - 0.25j, tb)
    assert relerr(ta.cpu().numpy(), a + (0.5 - 0.25j) * b) < 1e-15
    rb.scale(tb, 2j)
    assert relerr(tb.cpu().numpy(), 2j * b) < 1e-15
    f = torch.empty(1 << 14, dtype=torch.complex64, device=cuda)
    rb.copy(f, tb)
    assert relerr(f.cpu().numpy().astype(np.complex128), 2j * b) < 1e-7
    r = rb.random_state(12, "c128", seed=5)
    assert abs(rb.norm(r) - 1.0) < 1e-14
    r2 = rb.random_state(12, "c128", seed=5)
    assert torch.equal(r, r2)


@pytest.mark.parametrize("L,dtype", [(18, "c128"), (19, "c64"), (20, "c128"), (20, "c64")])
def test_apply_row_kernel(cuda, L, dtype):
    """The TMA row-layout kernel (default for >= 18/19 qubits), including
    complex coefficients (split into a real and an imaginary term) and a
    fused projection through the Krylov path."""
    N = 2 * L
    bits, coeff = rb.syk.sparse_syk(N, k=4, seed=L)
    rng = np.random.default_rng(L)
    # a few general terms with complex coefficients and low X/Z bits
    extra = rng.integers(0, 1 << (2 * L), size=12, dtype=np.uint64)
    bits = np.concatenate([bits, extra])
    coeff = np.concatenate([coeff, 0.01 * (rng.standard_normal(12) + 1j * rng.standard_normal(12))])
    bits, idx = np.unique(bits, return_index=True)
    coeff = coeff[idx]
    v = rand_vec(rng, L)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    assert ham.info()["kernel"] == 2
    x = to_dev(v, dtype)
    out = torch.empty_like(x)
    ham.apply(out, x)
    ref = O.apply(L, bits, coeff, v)
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    assert relerr(out.cpu().numpy().astype(np.complex128), ref) < tol
    ham.apply(out, x, accumulate=True)
    assert relerr(out.cpu().numpy().astype(np.complex128), 2 * ref) < tol


def test_evolve_row_kernel_fp64(cuda):
    L, N = 18, 36
    bits, coeff = rb.syk.sparse_syk(N, k=8, seed=4)
    v = rand_vec(np.random.default_rng(2), L)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    assert ham.info()["kernel"] == 2
    x = to_dev(v, "c128")
    st = rb.evolve(ham, x, 0.8, 0.0, 6, 1e-10)
    ref, st2 = O.evolve(L, bits, coeff, v, 0.8, 0.0, 6, 1e-10)
    assert relerr(x.cpu().numpy(), ref) < FP64_TOL
    for key in ("restarts", "applies", "passes", "prods"):
        assert st[key] == st2[key], (key, st, st2)


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["syk", "xxz"])
def test_ground_state_lanczos_matches_dense(model):
    """The reference's restarted Lanczos (inc/algo.h:180-257) on the GPU:
    energy against the lowest eigenvalue of the oracle's dense matrix, and
    the returned state is an eigenvector."""
    import reapers_b200 as rb
    import torch
    from oracle import oracle as O
    L = 10
    if model == "syk":
        bits, coeff = rb.syk.sparse_syk(2 * L, 8, seed=4)
    else:
        bits, coeff = rb.syk.xxz_chain(L, 1.0, np.random.default_rng(4).uniform(-1, 1, L))
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    E, g = rb.ground_state(ham, krydim=20, eps=1e-9, maxiter=500, seed=3)
    Hd = O.dense_matrix(L, bits, coeff)
    E0 = np.linalg.eigvalsh(Hd)[0]
    assert abs(E - E0) <= 1e-10 * abs(E0), (E, E0)
    gv = g.cpu().numpy()
    assert np.linalg.norm(Hd @ gv - E0 * gv) <= 1e-6
    ham.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("L", [19, 22])
def test_apply_host_pipeline_matches_device_apply(dtype, L):
    """rp_apply_host (host states, copies overlapped with the products) gives
    the device apply's results, bit for bit, for every state of the
    sequence; at 22 qubits each product runs as several launches over output
    ranges whose copies start as each range is written."""
    import reapers_b200 as rb
    bits, coeff = rb.syk.sparse_syk(2 * L, 8, seed=2)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    ins = [rb.random_state(L, dtype, seed=s).cpu().pin_memory() for s in range(5)]
    outs = [torch.empty(1 << L, dtype=tdt).pin_memory() for _ in range(5)]
    ham.apply_host(outs, ins)
    ham.apply_host([], [])
    for x, got in zip(ins, outs):
        y = torch.empty(1 << L, dtype=tdt, device="cuda")
        ham.apply(y, x.cuda())
        assert torch.equal(got, y.cpu())
    ham.close()


@pytest.mark.gpu
def test_dense_path_matches_krylov_on_dense_syk_n24():
    """Exact diagonalisation (inc/algo.h:27-54) on the GPU for the dense SYK
    of 12 qubits (all 10626 quartets of N = 24), through the library's dense
    path (rp_dense_*): V diag(lambda) V^H rebuilds the oracle's matrix, the
    eigenvalues are the oracle's, exp(-iHt) psi equals the oracle's
    restarted Krylov at t = 0.5 .. 5 (tol 1e-12), exponentials are cached
    per exponent, and the ground state is the lowest eigenpair."""
    import reapers_b200 as rb
    from reapers_b200.dense import DenseEvolver
    from oracle import oracle as O
    L = 12
    bits, coeff = rb.syk.dense_syk(24, seed=1)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    ev = DenseEvolver(ham)
    Hd = O.dense_matrix(L, bits, coeff)
    lam = ev.eigenvalues()
    V = ev.eigenvectors().cpu().numpy()
    assert np.abs(lam - np.linalg.eigvalsh(Hd)).max() <= 1e-12 * np.abs(lam).max()
    assert np.abs((V * lam) @ V.conj().T - Hd).max() <= 1e-11 * np.abs(Hd).max()
    rng = np.random.default_rng(7)
    psi0 = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    psi0 /= np.linalg.norm(psi0)
    for t in (0.5, 2.5, 5.0):
        x = torch.from_numpy(psi0).cuda()
        ev.evolve(x, t)
        ref, _ = O.evolve(L, bits, coeff, psi0, t, 0.0, 20, 1e-12)
        assert np.linalg.norm(x.cpu().numpy() - ref) <= 1e-11 * np.linalg.norm(ref)
    x = torch.from_numpy(psi0).cuda()
    ev.evolve(x, 2.5)                      # served from the cache
    assert ev.cache_info()["entries"] == 3 and ev.cache_info()["hits"][(-0.0, -2.5)] == 1
    E0, g = ev.ground_state()
    assert abs(E0 - np.linalg.eigvalsh(Hd)[0]) <= 1e-10
    gv = g.cpu().numpy()
    assert np.linalg.norm(Hd @ gv - E0 * gv) <= 1e-9
    ev.close()
    ham.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["c64", "c128"])
def test_dense_entry_points_small(dtype):
    """rp_dense_* and rp_mat_vec on a random Hermitian Pauli sum of 7 qubits
    (complex and Y-carrying coefficients) against numpy: eigenvalues, the
    exponential exp(c H) for a complex c, and the matrix-vector product;
    FP64 to 1e-12, FP32 to 1e-5 relative."""
    import reapers_b200 as rb
    from reapers_b200.dense import DenseEvolver
    from oracle import oracle as O
    from scipy.linalg import expm
    L = 7
    rng = np.random.default_rng(9)
    bits = np.unique(rng.integers(0, 1 << (2 * L), 40, dtype=np.uint64))
    # Hermitian: a Pauli string times a real number, sigma_y's i carried by
    # the stored coefficient (i^(number of Y factors))
    x = np.array([int(b) & 0x5555 for b in bits], dtype=np.int64)
    z = np.array([(int(b) >> 1) & 0x5555 for b in bits], dtype=np.int64)
    ny = np.array([bin(int(a) & int(c)).count("1") for a, c in zip(x, z)])
    coeff = rng.standard_normal(len(bits)) * (1j ** ny)
    Hd = O.dense_matrix(L, bits, coeff)
    assert np.abs(Hd - Hd.conj().T).max() < 1e-14
    tol = 1e-12 if dtype == "c128" else 1e-5
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    ev = DenseEvolver(ham)
    lam = ev.eigenvalues()
    ref = np.linalg.eigvalsh(Hd)
    assert np.abs(lam - ref).max() <= tol * np.abs(ref).max() * 10
    c = complex(-0.3, -1.7)
    E = ev.matexp(c).cpu().numpy().reshape(1 << L, 1 << L).T
    Er = expm(c * Hd)
    assert np.abs(E - Er).max() <= tol * np.abs(Er).max() * 10
    psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    tdt = torch.complex64 if dtype == "c64" else torch.complex128
    xg = torch.from_numpy(psi).to(tdt).cuda()
    ev.evolve(xg, 1.7, 0.3)
    want = Er @ psi
    assert np.linalg.norm(xg.cpu().numpy() - want) <= tol * np.linalg.norm(want) * 10
    ev.close()
    ham.close()


@pytest.mark.gpu
def test_new_entry_points_reject_bad_arguments():
    """Invalid arguments come back as RPError (status codes), the library
    stays usable."""
    import ctypes as C
    import reapers_b200 as rb
    from reapers_b200 import _lib, stepper as SP
    L = 10
    bits, coeff = rb.syk.sparse_syk(20, 4, seed=1)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    x = rb.random_state(L, "c128", seed=1)
    with pytest.raises(rb.RPError):
        SP.arnoldi(ham, x, 1)                 # m < 2
    with pytest.raises(rb.RPError):
        SP.arnoldi(ham, x, 65)                # m > 64
    with pytest.raises(rb.RPError):
        SP.expm_first_columns(np.eye(2000), [1.0])   # m > 1024
    with pytest.raises(rb.RPError):
        SP.Mlp(0, 2)                          # no inputs
    with pytest.raises(rb.RPError):
        SP.Mlp(4, 9)                          # more than 8 outputs
    with pytest.raises(rb.RPError):
        _lib.call("rp_apply_host", ham.handle, 1, None, None)
    with pytest.raises(rb.RPError):
        _lib.call("rp_arnoldi_combine", None, C.c_void_p(x.data_ptr()))
    # still usable
    y = torch.empty_like(x)
    ham.apply(y, x)
    b = SP.arnoldi(ham, x, 6)
    assert b.m_eff == 6
    ham.close()


@pytest.mark.parametrize("case", range(12))
def test_apply_randomised_sweep(cuda, case):
    """Seeded random draws over the whole kernel choice: state length 1-21
    qubits (direct, bulk-copy tiled and TMA row kernels), 1-200 terms with
    real, imaginary or mixed coefficients, Y-heavy strings (X and Z on the
    same sites), both precisions, overwrite and accumulate."""
    rng = np.random.default_rng(9000 + case)
    L = int(rng.choice([1, 3, 7, 11, 13, 16, 17, 18, 19, 20, 21]))
    dtype = ["c128", "c64"][case % 2]
    kinds = ["mixed", "real", "imag"][case % 3]
    T = int(rng.integers(1, 201))
    bits, coeff = rand_terms(rng, L, T, kinds)
    if case % 4 == 3:   # copy each X mask onto the Z bits: sigma^y on every flipped site
        xm = np.zeros_like(bits)
        for i in range(L):
            xm |= bits & np.uint64(1 << (2 * i))
        bits, idx = np.unique(xm | (xm << np.uint64(1)), return_index=True)
        coeff = coeff[idx]
    v = rand_vec(rng, L)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    x = to_dev(v, dtype)
    out = torch.empty_like(x)
    ham.apply(out, x)
    ref = O.apply(L, bits, coeff, v)
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    got = out.cpu().numpy().astype(np.complex128)
    assert relerr(got, ref) < tol, (L, dtype, kinds, len(bits), ham.info()["kernel"])
    ham.apply(out, x, accumulate=True)
    assert relerr(out.cpu().numpy().astype(np.complex128), 2 * ref) < tol


def _diag_heavy(rng, L):
    """Real Z strings on in-row and high qubits (fused into the diagonal
    factor), an imaginary one and a complex one (its imaginary part stays a
    term), plus X terms on low and high qubits."""
    def zbit(i):
        return 1 << (2 * i + 1)

    def xbit(i):
        return 1 << (2 * i)

    bits, coeff = [], []
    for i in range(L):                      # fields, every qubit
        bits.append(zbit(i))
        coeff.append(rng.uniform(-1, 1))
    for i in range(L - 1):                  # ZZ couplings
        bits.append(zbit(i) | zbit(i + 1))
        coeff.append(rng.uniform(-1, 1))
    bits.append(zbit(0) | zbit(3) | zbit(L - 1))
    coeff.append(0.3j)                      # imaginary diagonal: a plain term
    bits.append(zbit(1) | zbit(L - 2))
    coeff.append(0.2 - 0.4j)                # complex diagonal: split
    for i in (0, 2, 5, L - 3, L - 1):       # X and Y terms, low and high
        bits.append(xbit(i))
        coeff.append(rng.uniform(-1, 1))
        bits.append(xbit(i) | zbit(i))
        coeff.append(1j * rng.uniform(-1, 1))
    return np.array(bits, dtype=np.uint64), np.array(coeff, dtype=np.complex128)


@pytest.mark.parametrize("dtype,L", [("c64", 19), ("c64", 21), ("c128", 18), ("c128", 20)])
@pytest.mark.parametrize("model", ["diag_heavy", "xxz", "fields_only"])
def test_row_kernel_fused_diagonal(cuda, dtype, L, model):
    """Real Z strings summed per row into one diagonal factor (bucketed by
    their in-row Z bits, Walsh-Hadamard over those bits) against the oracle,
    overwrite and accumulate; "fields_only" has no other terms on the
    output's own tile, so the kernel's tile group 0 holds the diagonal alone."""
    rng = np.random.default_rng(L)
    if model == "diag_heavy":
        bits, coeff = _diag_heavy(rng, L)
    elif model == "xxz":
        bits, coeff = rb.syk.xxz_chain(L, 0.8, rng.uniform(-1, 1, L), periodic=True)
    else:
        bits = np.array([1 << (2 * i + 1) for i in range(L)] + [1 << (2 * (L - 1))],
                        dtype=np.uint64)
        coeff = np.concatenate([rng.uniform(-1, 1, L), [0.7]]).astype(np.complex128)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    info = ham.info()
    assert info["kernel"] == 2 and info["diag_terms"] >= 4, info
    v = rand_vec(rng, L)
    x = to_dev(v, dtype)
    out = torch.empty_like(x)
    ham.apply(out, x)
    ref = O.apply(L, bits, coeff, v)
    tol = FP64_TOL if dtype == "c128" else FP32_TOL
    assert relerr(out.cpu().numpy().astype(np.complex128), ref) < tol
    ham.apply(out, x, accumulate=True)
    assert relerr(out.cpu().numpy().astype(np.complex128), 2 * ref) < tol
    ham.close()
