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


# --- peer-read applies (rp_apply_shard): one row-kernel launch per output
# shard, every source tile read from the shard that holds it ---------------

@pytest.mark.parametrize("dtype", ["c64", "c128"])
@pytest.mark.parametrize("k", [1, 2, 3])
@pytest.mark.parametrize("model", ["syk", "xxz"])
def test_peer_shard_apply_is_bit_identical_to_full_apply(rb, dtype, k, model):
    L = 20
    bits, coeff = _models(rb, L)[model]
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    assert ham.info()["kernel"] == 2
    full = rb.random_state(L, dtype, seed=11)
    ref = torch.empty_like(full)
    ham.apply(ref, full)
    n = (1 << L) >> k
    shards = [full[s * n:(s + 1) * n].clone() for s in range(1 << k)]
    for r in range(1 << k):
        out = torch.empty_like(shards[0])
        ham.apply_shard(out, shards, rank=r)
        assert torch.equal(out, ref[r * n:(r + 1) * n]), (r, k)
        ham.apply_shard(out, shards, rank=r, accumulate=True)
        assert torch.equal(out, 2 * ref[r * n:(r + 1) * n]), (r, k)
    ham.close()


@pytest.mark.parametrize("exchange", ["peer", "stage"])
def test_single_launch_sharded_hamiltonian_and_evolve(rb, exchange):
    from reapers_b200 import sharded as SH
    L, k = 19, 2
    bits, coeff = _models(rb, L)["syk"]
    full = rb.random_state(L, "c128", seed=21)
    ham = rb.Hamiltonian(L, bits, coeff, "c128")
    ref = torch.empty_like(full)
    ham.apply(ref, full)
    comm = SH.LocalComm(1 << k)
    sh = SH.ShardedHamiltonian(L, bits, coeff, comm, exchange=exchange)
    x = SH.Shards.split(comm, full)
    if exchange == "peer":
        x.share()
    y = SH.Shards.empty_like(x)
    sh.apply(y, x)
    assert torch.equal(y.gather_local(), ref)
    psi_ref = full.clone()
    st_ref = rb.evolve(ham, psi_ref, 0.7, 0.0, 10, 1e-13)
    x = SH.Shards.split(comm, full)
    st = SH.sharded_evolve(sh, x, 0.7, 0.0, 10, 1e-13)
    got = x.gather_local()
    err = (torch.linalg.vector_norm(got - psi_ref) / torch.linalg.vector_norm(psi_ref)).item()
    assert err <= 1e-12, (err, st, st_ref)
    assert st["restarts"] == st_ref["restarts"] and st["applies"] == st_ref["applies"]
    sh.close()
    ham.close()


def test_apply_shard_rejects_bad_arguments(rb):
    import ctypes as C
    from reapers_b200 import _lib
    lib = _lib.load()
    L = 20
    bits, coeff = _models(rb, L)["syk"]
    ham = rb.Hamiltonian(L, bits, coeff, "c64")
    full = rb.random_state(L, "c64", seed=1)
    half = (1 << L) // 2
    a, b = full[:half].clone(), full[half:].clone()
    out = torch.empty_like(a)

    def call(k, rank, ptrs, o):
        arr = (C.c_void_p * len(ptrs))(*ptrs)
        rc = lib.rp_apply_shard(ham._h, k, rank, arr, C.c_void_p(o), 0)
        return rc, lib.rp_last_error().decode()

    good = [a.data_ptr(), b.data_ptr()]
    assert call(1, 0, good, out.data_ptr())[0] == 0
    for k, rank, ptrs, o, msg in [
            (0, 0, good, out.data_ptr(), "2 to 8 shards"),
            (4, 0, good * 8, out.data_ptr(), "2 to 8 shards"),
            (1, 2, good, out.data_ptr(), "shard index"),
            (1, -1, good, out.data_ptr(), "shard index"),
            (1, 0, [a.data_ptr(), 0], out.data_ptr(), "non-null"),
            (1, 0, [a.data_ptr() + 8, b.data_ptr()], out.data_ptr(), "16-byte aligned"),
            (1, 0, good, a.data_ptr(), "output may not be an input shard")]:
        rc, err = call(k, rank, ptrs, o)
        assert rc == -2 and msg in err, (k, rank, rc, err)
    rc = lib.rp_apply_shard(ham._h, 1, 0, None, C.c_void_p(out.data_ptr()), 0)
    assert rc == -2
    ham.close()
    small = rb.Hamiltonian(12, *_models(rb, 12)["syk"], "c128")
    x = rb.random_state(12, "c128", seed=2)
    o = torch.empty(1 << 11, dtype=x.dtype, device=x.device)
    s0, s1 = x[:1 << 11].clone(), x[1 << 11:].clone()
    rc = lib.rp_apply_shard(small._h, 1, 0, (C.c_void_p * 2)(s0.data_ptr(), s1.data_ptr()),
                            C.c_void_p(o.data_ptr()), 0)
    assert rc == -2 and "row kernel" in lib.rp_last_error().decode()
    small.close()


def _ipc_rank(rank, world, port, L, k_seed, q):
    """One rank of the two-process peer-read test: both on cuda:0, each
    owning one shard, the other's opened through CUDA IPC."""
    import datetime
    import torch.distributed as dist
    try:
        import reapers_b200 as rbm
        from reapers_b200 import sharded as SH
        torch.cuda.set_device(0)
        rbm.init(0)
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=60))
        bits, coeff = rbm.syk.sparse_syk(2 * L, 8, seed=k_seed)
        full = rbm.random_state(L, "c64", seed=31)
        ham = rbm.Hamiltonian(L, bits, coeff, "c64")
        ref = torch.empty_like(full)
        ham.apply(ref, full)
        comm = SH.ProcessGroupComm()
        sh = SH.ShardedHamiltonian(L, bits, coeff, comm, dtype="c64", exchange="peer")
        x = SH.Shards.split(comm, full).share()
        y = SH.Shards.empty_like(x)
        sh.apply(y, x)
        n = (1 << L) // world
        ok = torch.equal(y.t[rank], ref[rank * n:(rank + 1) * n])
        x.unshare()
        sh.close()
        ham.close()
        dist.destroy_process_group()
        q.put((rank, bool(ok), ""))
    except Exception as e:  # reported to the parent
        q.put((rank, False, repr(e)))


def test_peer_apply_across_processes_through_ipc(rb):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_ipc_rank, args=(r, 2, port, 20, 40, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = []
    for _ in procs:
        res.append(q.get(timeout=240))
    for p in procs:
        p.join(timeout=60)
    assert all(ok for _, ok, _ in res), res


def test_ipc_entry_points_reject_bad_arguments(rb):
    import ctypes as C
    from reapers_b200 import _lib
    lib = _lib.load()
    # a pointer this process never opened
    rc = lib.rp_ipc_close(C.c_void_p(0x1000))
    assert rc == -2 and "not opened by rp_ipc_open" in lib.rp_last_error().decode()
    # host memory is not a device allocation
    host = (C.c_char * 64)()
    h = _lib.IpcHandle()
    rc = lib.rp_ipc_export(C.cast(host, C.c_void_p), C.byref(h))
    assert rc == -2 and "not a device allocation" in lib.rp_last_error().decode()
    assert lib.rp_ipc_export(None, C.byref(h)) == -2
    assert lib.rp_ipc_open(None, C.byref(C.c_void_p())) == -2
    # a device tensor exports: the handle names its allocation, the offset
    # its place inside it
    t = torch.empty(1 << 20, dtype=torch.complex64, device="cuda")
    view = t[4096:]
    data, off0 = rb.ipc_export(t)
    data2, off1 = rb.ipc_export(view)
    assert data == data2 and off1 - off0 == 4096 * 8
