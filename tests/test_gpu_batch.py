"""Batched OTOC (one persistent launch per time step and team size, uneven
qubit counts) against the FP64 CPU oracle and the single-problem mixed path;
teams of 1..16 CTAs (thread-block clusters) per problem give the same answer.

Tolerance: 2e-5 absolute on the OTOC (|F(0)| = 1/4), the FP32 state storage
of the batched form; graph replay and direct launches agree exactly."""
import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_problems(specs, seed=0):
    probs, ref_inputs = [], []
    for i, (N, k) in enumerate(specs):
        L = N // 2
        bits, coeff = rb.syk.sparse_syk(N, k=k, seed=seed + i)
        mb, mc = rb.syk.majoranas(N)
        rng = np.random.default_rng(100 + i)
        psi = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
        psi /= np.linalg.norm(psi)
        psi32 = psi.astype(np.complex64)
        w = (mb[N - 1:N], mc[N - 1:N])
        v = (mb[N - 2:N - 1], mc[N - 2:N - 1])
        probs.append(dict(len=L, bits=bits, coeff=coeff, w=w, v=v,
                          psi0=torch.from_numpy(psi32).cuda()))
        ref_inputs.append((L, bits, coeff, w, v, psi32.astype(np.complex128)))
    return probs, ref_inputs


def test_batched_otoc_matches_oracle_uneven_sizes(cuda):
    specs = [(16, 4), (18, 4), (20, 4), (16, 4)]
    probs, refs = make_problems(specs)
    times = np.array([0.0, 0.6, 1.4])
    b = rb.BatchOTOC(probs, krydim=10, tol=1e-7, max_restarts=16)
    F, ap = b.run(times, use_graph=True)
    F2, ap2 = b.run(times, use_graph=False)
    assert np.array_equal(F, F2) and np.array_equal(ap, ap2)
    for p, (L, bits, coeff, w, v, psi) in enumerate(refs):
        ref = O.otoc(L, bits, coeff, w, v, psi, times, 10, 1e-12)
        assert np.abs(F[p] - ref).max() < 2e-5, (p, F[p], ref)
        assert ap[p, 0] == 0 and ap[p, 1] > 0


def test_batched_matches_single_problem_mixed_path(cuda):
    specs = [(18, 8)]
    probs, refs = make_problems(specs, seed=5)
    times = np.array([0.9])
    b = rb.BatchOTOC(probs, krydim=12, tol=1e-7, max_restarts=16)
    F, ap = b.run(times)
    L, bits, coeff, w, v, psi = refs[0]
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    wh = rb.Hamiltonian(L, *w, "c64")
    vh = rb.Hamiltonian(L, *v, "c64")
    vals, applies = rb.otoc(ham, wh, vh, probs[0]["psi0"], times, 12, 1e-7)
    assert abs(F[0, 0] - vals[0]) < 2e-5
    assert abs(int(ap[0, 0]) - applies) <= 12   # same algorithm; rounding may move a pass


def test_batched_rejects_bad_tile(cuda):
    probs, _ = make_problems([(16, 4)])
    probs[0]["tile"] = 13
    with pytest.raises(rb.RPError):
        rb.BatchOTOC(probs)


@pytest.mark.parametrize("team", [1, 2, 4, 8, 16])
def test_batched_team_sizes_agree(cuda, team):
    """One problem shared by a cluster of `team` CTAs: same OTOC as the oracle
    and as one CTA, within FP32 rounding; same H.psi count."""
    specs = [(20, 4), (18, 4), (16, 4)]
    probs, refs = make_problems(specs, seed=11)
    times = np.array([0.0, 0.8])
    ref_b = rb.BatchOTOC([dict(p, team=1) for p in probs], krydim=10, tol=1e-7, max_restarts=16)
    F1, ap1 = ref_b.run(times)
    ref_b.close()
    b = rb.BatchOTOC([dict(p, team=team) for p in probs], krydim=10, tol=1e-7, max_restarts=16)
    F, ap = b.run(times, use_graph=True)
    F2, _ = b.run(times, use_graph=False)
    b.close()
    assert np.array_equal(F, F2)
    assert np.abs(F - F1).max() < 2e-6
    assert np.abs(ap - ap1).max() <= 10
    for p, (L, bits, coeff, w, v, psi) in enumerate(refs):
        ref = O.otoc(L, bits, coeff, w, v, psi, times, 10, 1e-12)
        assert np.abs(F[p] - ref).max() < 2e-5, (p, F[p], ref)


def test_batched_mixed_team_classes(cuda):
    """Problems of different team sizes in one batch: one launch per class."""
    specs = [(16, 4), (20, 4), (18, 4), (20, 4)]
    probs, refs = make_problems(specs, seed=21)
    for p, t in zip(probs, [1, 16, 4, 8]):
        p["team"] = t
    times = np.array([0.7])
    b = rb.BatchOTOC(probs, krydim=10, tol=1e-7, max_restarts=16)
    F, ap = b.run(times)
    b.close()
    for p, (L, bits, coeff, w, v, psi) in enumerate(refs):
        ref = O.otoc(L, bits, coeff, w, v, psi, times, 10, 1e-12)
        assert np.abs(F[p] - ref).max() < 2e-5, (p, F[p], ref)


def test_batched_rejects_bad_team(cuda):
    probs, _ = make_problems([(16, 4)])
    probs[0]["team"] = 3
    with pytest.raises(rb.RPError):
        rb.BatchOTOC(probs)


@pytest.mark.parametrize("team", [1, 4, 16])
def test_batched_row_tiles_match_tile_loop(cuda, team):
    """The row-tile H.psi loop (2-D TMA swizzled tiles, tile exponent 12)
    against the bulk-copy tile loop (exponent 11) on the same problems."""
    specs = [(24, 8), (28, 8), (32, 4)]
    probs, refs = make_problems(specs, seed=31)
    times = np.array([0.0, 0.9])
    out = {}
    for tile in (11, 12):
        b = rb.BatchOTOC([dict(p, tile=tile, team=team) for p in probs], krydim=12, tol=1e-7,
                         max_restarts=16)
        out[tile] = b.run(times)
        b.close()
    assert np.abs(out[11][0] - out[12][0]).max() < 2e-6
    assert np.abs(out[11][1] - out[12][1]).max() <= 12
    for p, (L, bits, coeff, w, v, psi) in enumerate(refs):
        ref = O.otoc(L, bits, coeff, w, v, psi, times, 12, 1e-12)
        assert np.abs(out[12][0][p] - ref).max() < 2e-5, (p, out[12][0][p], ref)


def test_batch_with_single_path_problems_matches_oracle(cuda):
    """Problems the autotuner sends to the single-problem path (path =
    'single') run one at a time after the batched launches; the batch's
    results keep the problems' order and match the oracle for both kinds."""
    specs = [(16, 4), (20, 4), (18, 4), (20, 4)]
    probs, refs = make_problems(specs, seed=21)
    for i in (1, 3):
        probs[i]["path"] = "single"
    times = np.array([0.0, 0.7])
    b = rb.BatchOTOC(probs, krydim=10, tol=1e-7, max_restarts=16)
    F, ap = b.run(times)
    b.close()
    for p, (L, bits, coeff, w, v, psi) in enumerate(refs):
        ref = O.otoc(L, bits, coeff, w, v, psi, times, 10, 1e-12)
        assert np.abs(F[p] - ref).max() < 2e-5, (p, F[p], ref)
        assert ap[p, 1] > 0


def test_autotuner_picks_a_candidate_per_shape(cuda, tmp_path, monkeypatch):
    """The tuner times one OTOC point for every candidate of a shape (the
    batched launch per tile loop and team size, and the single-problem path)
    and tags the problems with the fastest; a second call reads the cache."""
    from reapers_b200 import autotune
    monkeypatch.setenv("RPB200_TUNE_CACHE", str(tmp_path / "tune.json"))
    specs = [(28, 4)] * 3 + [(32, 4)] * 3
    probs, _ = make_problems(specs, seed=40)
    out = autotune.tune(probs, krydim=8, tol=1e-6, t_probe=0.3, nsingle=2)
    assert len(out) >= 2
    for rec in out.values():
        assert autotune.SINGLE in rec["seconds"]
        assert rec["path"] in ("batched", autotune.SINGLE)
        assert min(rec["seconds"].values()) > 0
    for p in probs:
        assert p["path"] in ("batched", autotune.SINGLE)
    again = autotune.tune(probs, krydim=8, tol=1e-6, t_probe=0.3, nsingle=2)
    assert again == out
