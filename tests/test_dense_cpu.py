"""Host-side argument checks of the exact-diagonalisation path (no GPU):
DenseEvolver refuses states whose precision or length differ from its
Hamiltonian's before any device call, so the dense mat-vec never reads a
matrix of one element size as another."""
import types

import pytest
import torch

from reapers_b200 import RP_C64, RP_C128
from reapers_b200.dense import DenseEvolver


def _ham(length, dtype):
    return types.SimpleNamespace(len=length, dtype=dtype)


def test_too_many_qubits():
    with pytest.raises(ValueError, match="at most 14 qubits"):
        DenseEvolver(_ham(15, RP_C128))


@pytest.mark.parametrize("code,dt", [(RP_C64, torch.complex64), (RP_C128, torch.complex128)])
def test_dtype_follows_hamiltonian(code, dt):
    assert DenseEvolver(_ham(4, code)).dtype == dt


@pytest.mark.parametrize("psi", [torch.zeros(16, dtype=torch.complex64),    # wrong precision
                                 torch.zeros(8, dtype=torch.complex128),    # wrong length
                                 torch.zeros(32, dtype=torch.complex128)])
def test_evolve_rejects_mismatched_state(psi):
    ev = DenseEvolver(_ham(4, RP_C128))
    with pytest.raises(ValueError, match="state must be"):
        ev.evolve(psi, 1.0)
    assert ev.cache_info()["entries"] == 0


def test_evolve_zero_time_is_identity():
    ev = DenseEvolver(_ham(3, RP_C64))
    psi = torch.arange(8, dtype=torch.float32).to(torch.complex64)
    ref = psi.clone()
    assert ev.evolve(psi, 0.0) is psi
    assert torch.equal(psi, ref)
