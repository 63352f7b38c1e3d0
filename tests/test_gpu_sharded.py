"""The sharded path on the GPU with 2^k virtual shards in one process
(LocalComm): H.psi and the restarted Krylov evolve over shards against the
single-vector path on the same GPU and against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import reapers_b200 as rb
    rb.init(0)
    return rb


def _models(rb, L):
    rng = np.random.default_rng(L)
    return {"syk": rb.syk.sparse_syk(2 * L, 8, seed=L),
            "xxz": rb.syk.xxz_chain(L, 1.0, rng.uniform(-1, 1, L), periodic=True)}


@pytest.mark.parametrize("k", [1, 2, 3])
@pytest.mark.parametrize("model", ["syk", "xxz"])
def test_sharded_apply_matches_single_vector(rb, k, model):
    from reapers_b200 import sharded as SH
    L = 12
    bits, coeff = _models(rb, L)[model]
    full = rb.random_state(L, "c128", seed=5)
    ref = torch.empty_like(full)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    ham.apply(ref, full)
    comm = SH.LocalComm(1 << k)
    sh = SH.ShardedHamiltonian(L, bits, coeff, comm)
    x = SH.Shards.split(comm, full)
    y = SH.Shards.empty_like(x)
    sh.apply(y, x)
    got = y.gather_local()
    err = (torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)).item()
    assert err <= 1e-14, err
    oracle = O.apply(L, bits, coeff, full.cpu().numpy())
    assert np.linalg.norm(got.cpu().numpy() - oracle) <= 1e-13 * np.linalg.norm(oracle)
    sh.close()
    ham.close()


@pytest.mark.parametrize("k", [1, 2])
def test_sharded_evolve_matches_single_vector(rb, k):
    from reapers_b200 import sharded as SH
    L = 12
    bits, coeff = _models(rb, L)["syk"]
    full = rb.random_state(L, "c128", seed=9)
    psi_ref = full.clone()
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    st_ref = rb.evolve(ham, psi_ref, 1.3, 0.0, 8, 1e-13)
    comm = SH.LocalComm(1 << k)
    sh = SH.ShardedHamiltonian(L, bits, coeff, comm)
    x = SH.Shards.split(comm, full)
    st = SH.sharded_evolve(sh, x, 1.3, 0.0, 8, 1e-13)
    got = x.gather_local()
    err = (torch.linalg.vector_norm(got - psi_ref) / torch.linalg.vector_norm(psi_ref)).item()
    assert err <= 1e-12, (err, st, st_ref)
    # the reference's algorithm in both: same restarts and H.psi count
    assert st["restarts"] == st_ref["restarts"] and st["applies"] == st_ref["applies"]
    ref_o, _ = O.evolve(L, bits, coeff, full.cpu().numpy(), 1.3, 0.0, 8, 1e-13)
    assert np.linalg.norm(got.cpu().numpy() - ref_o) <= 1e-12 * np.linalg.norm(ref_o)
    sh.close()
    ham.close()
