"""Sharded H.psi host logic on the CPU.

* the per-shard local Hamiltonians H_xh^(r) reassemble the full operator:
  block (r, r ^ xh) of the oracle's dense matrix equals the dense matrix of
  H_xh^(r) on L - k qubits;
* the exchange schedules of ShardedHamiltonian.apply over real gloo process
  groups (world size 2 and 4): one swap with r ^ xh at a time ("copy"), or
  every needed partner shard at once before one full-operator launch
  ("stage"); the gathered result equals the full dense product.  The
  local products here are dense numpy matrices from the oracle (the checker)
  injected through ShardedHamiltonian's `local` argument; on the GPU they
  are the library's kernels (tests/test_gpu_sharded.py).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import oracle as O
from reapers_b200 import sharded as SH
from reapers_b200 import syk as S


def random_terms(L, T, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 1 << (2 * L), T, dtype=np.uint64)
    coeff = rng.standard_normal(T) + 1j * rng.standard_normal(T)
    # a few Y factors carry their i in the stored coefficient
    return bits, coeff


@pytest.mark.parametrize("k", [1, 2, 3])
def test_local_hamiltonians_reassemble_the_operator(k):
    L = 7
    bits, coeff = random_terms(L, 40, seed=k)
    full = O.dense_matrix(L, bits, coeff)
    n = 1 << (L - k)
    for r in range(1 << k):
        parts = SH.shard_terms(L, k, bits, coeff, r)
        got = np.zeros((n, 1 << L), dtype=np.complex128)
        for h, (b, c) in parts.items():
            got[:, (r ^ h) * n:((r ^ h) + 1) * n] += O.dense_matrix(L - k, b, c)
        np.testing.assert_allclose(got, full[r * n:(r + 1) * n, :], atol=1e-13)


class _DenseLocal:
    """Dense numpy stand-in for one shard's local operator (test only)."""

    def __init__(self, length, bits, coeff, dtype):
        self.M = torch.from_numpy(O.dense_matrix(length, bits, coeff))

    def apply(self, out, inp, accumulate=False):
        r = self.M @ inp
        if accumulate:
            out += r
        else:
            out.copy_(r)

    def close(self):
        pass


class _DenseFull:
    """Dense numpy stand-in for the full operator's single-launch sharded
    apply (test only): output shard `rank` from the concatenated shards."""

    def __init__(self, length, bits, coeff, dtype):
        self.M = torch.from_numpy(O.dense_matrix(length, bits, coeff))

    def apply_shard(self, out, shards, rank, accumulate=False):
        n = out.numel()
        r = self.M[rank * n:(rank + 1) * n] @ torch.cat(list(shards))
        if accumulate:
            out += r
        else:
            out.copy_(r)

    def close(self):
        pass


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, L, bits, coeff, vec, out_dir, exchange="copy"):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comm = SH.ProcessGroupComm()
        if exchange == "stage":
            ham = SH.ShardedHamiltonian(L, bits, coeff, comm, exchange="stage", full=_DenseFull)
        else:
            ham = SH.ShardedHamiltonian(L, bits, coeff, comm, local=_DenseLocal)
        x = SH.Shards.split(comm, torch.from_numpy(vec))
        y = SH.Shards.empty_like(x)
        ham.apply(y, x)
        parts = [torch.empty_like(y.t[rank]) for _ in range(world)]
        dist.all_gather(parts, y.t[rank])
        tot = comm.allreduce([float(rank), 1.0])
        if rank == 0:
            np.save(os.path.join(out_dir, "y.npy"), torch.cat(parts).numpy())
            np.save(os.path.join(out_dir, "tot.npy"), tot)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange", ["copy", "stage"])
@pytest.mark.parametrize("world", [2, 4])
def test_sharded_apply_over_gloo_ranks(world, exchange, tmp_path):
    L = 8
    bits, coeff = random_terms(L, 60, seed=10 + world)
    # plus terms whose X masks use the top qubits, so every exchange is exercised
    extra = np.array([(1 << (2 * (L - 1))) | 3, (3 << (2 * (L - 2))), 2 << (2 * (L - 1))],
                     dtype=np.uint64)
    bits = np.concatenate([bits, extra])
    coeff = np.concatenate([coeff, [0.5, -1.25j, 2.0]])
    rng = np.random.default_rng(3)
    vec = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    mp.spawn(_worker, args=(world, _free_port(), L, bits, coeff, vec, str(tmp_path), exchange),
             nprocs=world, join=True)
    y = np.load(tmp_path / "y.npy")
    ref = O.dense_matrix(L, bits, coeff) @ vec
    np.testing.assert_allclose(y, ref, atol=1e-12)
    tot = np.load(tmp_path / "tot.npy")
    assert tot[0] == sum(range(world)) and tot[1] == world


def test_xmask_split_matches_bits():
    L, k = 6, 2
    bits, coeff = random_terms(L, 20, seed=5)
    parts = SH.shard_terms(L, k, bits, coeff, 0)
    assert sorted(parts) == sorted(set((S.xmask(bits) >> np.uint64(L - k)).astype(int).tolist()))
    assert sum(len(b) for b, _ in parts.values()) == len(bits)


class _DenseFullOp(_DenseFull):
    """The dense stand-in with the single-state apply too (test only)."""

    def apply(self, out, inp, accumulate=False):
        r = self.M @ inp
        if accumulate:
            out += r
        else:
            out.copy_(r)


class _WallClock:
    """Host timer standing in for the CUDA events of the GPU run (test only)."""

    def start(self):
        import time
        self.t0 = time.perf_counter()

    def stop(self):
        import time
        return time.perf_counter() - self.t0


def _leg_worker(rank, world, port, L, bits, coeff, vec, out_dir):
    import json
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comm = SH.ProcessGroupComm()
        out = bench.sharded_dist_leg(comm, L, bits, coeff, "c128", steps=2, warmup=1,
                                     modes=("stage",), full=_DenseFullOp,
                                     make_state=lambda: torch.from_numpy(vec.copy()),
                                     clock=_WallClock())
        if rank == 0:
            with open(os.path.join(out_dir, "leg.json"), "w") as f:
                json.dump(out, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_bench_sharded_leg_plumbing_over_gloo(world, tmp_path):
    """bench.py's multi-GPU leg (the reference's high-bit split of one state
    over the ranks) driven over a real gloo process group with the dense
    stand-in operator and a host clock: every rank's output shard equals the
    full product's, the partner shards the terms reach are the ones
    exchanged, and rank 0 reports a time per apply for every rank."""
    import json
    L = 8
    bits, coeff = random_terms(L, 50, seed=20 + world)
    extra = np.array([(1 << (2 * (L - 1))) | 3, (3 << (2 * (L - 2)))], dtype=np.uint64)
    bits = np.concatenate([bits, extra])
    coeff = np.concatenate([coeff, [0.5, -1.25j]])
    rng = np.random.default_rng(4)
    vec = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    mp.spawn(_leg_worker, args=(world, _free_port(), L, bits, coeff, vec, str(tmp_path)),
             nprocs=world, join=True)
    leg = json.load(open(tmp_path / "leg.json"))
    st = leg["modes"]["stage"]
    assert st["bit_identical_to_full_apply"] is True
    assert len(st["ms_per_apply_by_rank"]) == world
    assert st["ms_per_apply"] == max(st["ms_per_apply_by_rank"])
    k = world.bit_length() - 1
    want = sorted(set((S.xmask(bits) >> np.uint64(L - k)).astype(int).tolist()) - {0})
    assert st["partner_offsets"] == want
