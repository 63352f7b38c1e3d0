"""A state split over 2^k shards by its top k qubits (one shard per GPU rank).

The reference splits a state over its GPUs by the high index bits and lets
every H.psi read the partner shard it needs (inc/gpuimpl.h:426-432,
src/krnl.cu:96-114).  Here a shard is a contiguous 2^(L-k) slice owned by
one rank; for a Pauli term with X mask x and Z mask z, output element
n = (r, l) (shard r, local index l) reads source (r ^ xh, l ^ xl), xh / xl
the high / low parts of x, with sign (-1)^popc(z & source).  Splitting z the
same way, the high part of the sign depends only on the source shard, so
for every distinct high part xh the terms form a LOCAL Hamiltonian on
L - k qubits,

    H_xh^(r) = sum_{t: xh_t = xh} c_t (-1)^popc(zh_t & (r ^ xh)) P(xl_t, zl_t),

and  (H psi)_r = sum_xh H_xh^(r) psi_{r ^ xh}.  One apply is therefore one
pairwise exchange per distinct xh != 0 (rank r swaps shards with r ^ xh,
both sides take the same steps in the same order), overlapped with the
local products, which run on the single-GPU kernels.  Inner products and
norms are local FP64 sums followed by an all-reduce.  The restarted Krylov
on top is the reference's algorithm (inc/algo.h:267-365) with the
projections of each orthogonalisation pass taken at once (one all-reduce
per pass) and the small matrices on the GPU in FP64, as the single-GPU path.

A process may own several shards (``Shards``), so the same code runs as
2^k ranks with one GPU each (``ProcessGroupComm``: NCCL for GPU tensors,
or gloo) or as 2^k virtual shards on one GPU (``LocalComm``).
"""
from __future__ import annotations

import math

import numpy as np

from . import syk as S

__all__ = ["shard_terms", "LocalComm", "ProcessGroupComm", "Shards", "ShardedHamiltonian",
           "sharded_dot", "sharded_norm", "sharded_evolve"]


def shard_terms(L, k, bits, coeff, rank):
    """{xh: (local bits, local coefficients)} of the local Hamiltonians
    H_xh^(rank) on L - k qubits, xh over the distinct high X parts in
    increasing order."""
    if not 0 <= k < L:
        raise ValueError("k must be in [0, L)")
    Ll = L - k
    b = np.asarray(bits, dtype=np.uint64)
    c = np.asarray(coeff, dtype=np.complex128)
    x = S.xmask(b)
    z = S.zmask(b)
    xh = (x >> np.uint64(Ll)).astype(np.int64)
    zh = (z >> np.uint64(Ll)).astype(np.int64)
    low = np.uint64((1 << (2 * Ll)) - 1)
    out = {}
    for h in sorted(set(xh.tolist())):
        sel = xh == h
        src = rank ^ h
        par = np.array([bin(int(v) & src).count("1") & 1 for v in zh[sel]])
        out[int(h)] = (b[sel] & low, c[sel] * (1.0 - 2.0 * par))
    return out


class LocalComm:
    """Every shard in this process: exchanges are plain reads of the peer
    shard, reductions are sums over the owned shards."""

    def __init__(self, nshards):
        self.world = nshards

    def owned(self):
        return list(range(self.world))

    def allreduce(self, arr):
        return np.asarray(arr, dtype=np.float64)

    def barrier(self):
        pass


class ProcessGroupComm:
    """One shard per rank of a torch.distributed process group."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def owned(self):
        return [self.rank]

    def start_exchange(self, send, peer, recv):
        """Swap `send` with rank `peer` into `recv`; returns the pending requests."""
        return self.start_exchanges([(send, peer, recv)])

    def start_exchanges(self, swaps):
        """Every (send, peer, recv) swap at once; returns the pending requests."""
        d = self.dist
        ops = []
        for send, peer, recv in swaps:
            ops += [d.P2POp(d.isend, send, peer, self.group), d.P2POp(d.irecv, recv, peer, self.group)]
        return d.batch_isend_irecv(ops) if ops else []

    def allreduce(self, arr):
        import torch
        a = np.asarray(arr, dtype=np.float64)
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(a.copy()).to(dev)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def all_gather_object(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out

    def barrier(self):
        """Every rank's device work issued so far is complete when this
        returns (the library stream and torch's are synchronised first)."""
        import torch
        if torch.cuda.is_available():
            from . import synchronize
            synchronize()
            torch.cuda.synchronize()
        self.dist.barrier(group=self.group)
        if self.dist.get_backend(self.group) == "nccl":
            torch.cuda.synchronize()


class Shards:
    """The shards of one vector owned by this process: {shard index: tensor}."""

    def __init__(self, comm, tensors):
        self.comm = comm
        self.t = dict(tensors)

    @classmethod
    def empty_like(cls, other):
        import torch
        return cls(other.comm, {r: torch.empty_like(v) for r, v in other.t.items()})

    @classmethod
    def split(cls, comm, full):
        """Shards of a full vector (every process holds it; for setup and tests)."""
        n = full.numel() // comm.world
        return cls(comm, {r: full[r * n:(r + 1) * n].clone() for r in comm.owned()})

    def gather_local(self):
        """The owned shards in shard order, concatenated."""
        import torch
        return torch.cat([self.t[r] for r in sorted(self.t)])

    peers = None      # device pointers of every shard, for peer-read applies
    _opened = ()

    def share(self):
        """Make every shard readable by every rank (collective): with one
        process per GPU the shards are exported as CUDA IPC handles and the
        peers' opened; in one process the pointers are taken as they are."""
        from . import ipc_export, ipc_open, _ptr
        if isinstance(self.comm, LocalComm):
            self.peers = [_ptr(self.t[r]).value for r in range(self.comm.world)]
            return self
        (r, t), = self.t.items()
        handles = self.comm.all_gather_object(ipc_export(t))
        ptrs, opened = [], []
        for i, h in enumerate(handles):
            if i == r:
                ptrs.append(_ptr(t).value)
            else:
                p = ipc_open(h)
                ptrs.append(p)
                opened.append(p)
        self.peers, self._opened = ptrs, tuple(opened)
        return self

    def unshare(self):
        """Close the peers' mappings (collective; afterwards a rank may free
        its shard)."""
        from . import ipc_close
        for p in self._opened:
            ipc_close(p)
        self.peers, self._opened = None, ()
        self.comm.barrier()


class ShardedHamiltonian:
    """H over 2^k shards of an L-qubit state: the local Hamiltonians
    H_xh^(r) of every owned shard r, on the single-GPU kernels."""

    def __init__(self, L, bits, coeff, comm, dtype="c128", local=None, exchange="copy", full=None):
        """local: the operator class of one shard's terms, called as
        local(length, bits, coeff, dtype) and providing apply(out, inp,
        accumulate) and close(); the library's Hamiltonian unless given.

        exchange: "copy" swaps partner shards into local buffers (NCCL
        send/recv, or plain reads in one process) one at a time, each swap
        in flight while the previous local Hamiltonian is applied; "peer"
        applies the full Hamiltonian in one row-kernel launch per output
        shard that reads every source tile straight from the shard holding
        it (rp_apply_shard: over NVLink for a peer's memory, inputs made
        readable with Shards.share()); "stage" swaps every partner shard the
        terms need at once (each crosses NVLink once) and then runs that same
        single launch over the local copies.

        full: for "peer" / "stage", the class of the full operator, called
        as full(length, bits, coeff, dtype) and providing
        apply_shard(out, shards, rank=r) and close(); the library's
        Hamiltonian unless given."""
        from . import Hamiltonian
        local = local or Hamiltonian
        k = int(round(math.log2(comm.world)))
        if 1 << k != comm.world:
            raise ValueError("the number of shards must be a power of two")
        if exchange not in ("copy", "peer", "stage"):
            raise ValueError("exchange must be 'copy', 'peer' or 'stage'")
        self.L, self.k, self.comm, self.dtype = L, k, comm, dtype
        self.exchange = exchange
        self.parts = {}
        if exchange in ("peer", "stage"):
            if k < 1:
                raise ValueError("a single-launch sharded apply needs at least two shards")
            self.full = (full or Hamiltonian)(L, bits, coeff, dtype)
            if full is None and self.full.info()["kernel"] != 2:
                self.full.close()
                raise ValueError("a single-launch sharded apply needs the row kernel (2^19+ "
                                 "complex64 or 2^18+ complex128 elements)")
            # shard offsets the terms reach (the top k bits of their X masks)
            xs = (S.xmask(np.asarray(bits, dtype=np.uint64)) >> np.uint64(L - k)).astype(np.int64)
            self.offsets = sorted(set(xs.tolist()) - {0})
            self.xhs = []
            self._stage = {}
            return
        for r in comm.owned():
            self.parts[r] = [(h, local(L - k, b, c, dtype))
                             for h, (b, c) in shard_terms(L, k, bits, coeff, r).items()]
        # every shard visits the same high parts in the same order
        self.xhs = [h for h, _ in self.parts[comm.owned()[0]]]

    def apply(self, out, inp):
        """out = H inp (Shards of the same layout)."""
        import torch
        if self.exchange == "peer":
            local = isinstance(self.comm, LocalComm)
            ptrs = inp.peers
            if ptrs is None:
                if not local:
                    raise ValueError("share() the input shards before a peer-read apply")
                ptrs = [inp.t[s] for s in range(self.comm.world)]
            # every shard final before any rank reads it, and read by every
            # rank before any rank goes on to overwrite one
            self.comm.barrier()
            for r in out.t:
                self.full.apply_shard(out.t[r], ptrs, rank=r)
            self.comm.barrier()
            return out
        if self.exchange == "stage":
            if isinstance(self.comm, LocalComm):
                shards = [inp.t[s] for s in range(self.comm.world)]
                for r in out.t:
                    self.full.apply_shard(out.t[r], shards, rank=r)
                return out
            (r, src), = inp.t.items()
            for d in self.offsets:
                buf = self._stage.get(d)
                if buf is None or buf.shape != src.shape or buf.dtype != src.dtype:
                    self._stage[d] = torch.empty_like(src)
            reqs = self.comm.start_exchanges([(src, r ^ d, self._stage[d]) for d in self.offsets])
            for q in reqs:
                q.wait()
            # shards no term reaches are never read: any valid vector stands in
            shards = [src if s == r else self._stage.get(r ^ s, src) for s in range(self.comm.world)]
            self.full.apply_shard(out.t[r], shards, rank=r)
            return out
        if isinstance(self.comm, LocalComm):
            for r, parts in self.parts.items():
                first = True
                for h, ham in parts:
                    ham.apply(out.t[r], inp.t[r ^ h], accumulate=not first)
                    first = False
                if first:
                    out.t[r].zero_()
            return out
        # one shard per rank: exchange with r ^ xh for each xh != 0, the next
        # exchange in flight while the current product runs
        (r, parts), = self.parts.items()
        src = inp.t[r]
        bufs = [torch.empty_like(src), torch.empty_like(src)]
        pending, cur = None, None
        order = list(parts)

        def start(i):
            h = order[i][0]
            if h == 0:
                return None, src
            buf = bufs[i & 1]
            return self.comm.start_exchange(src, r ^ h, buf), buf

        if order:
            pending, cur = start(0)
        first = True
        for i, (h, ham) in enumerate(order):
            if pending is not None:
                for req in pending:
                    req.wait()
            data = cur
            if i + 1 < len(order):
                pending, cur = start(i + 1)
            else:
                pending, cur = None, None
            ham.apply(out.t[r], data, accumulate=not first)
            first = False
        if first:
            out.t[r].zero_()
        return out

    def close(self):
        for parts in self.parts.values():
            for _, h in parts:
                h.close()
        if self.exchange in ("peer", "stage"):
            self.full.close()
            self._stage = {}


def sharded_dot(a, b):
    """<a|b> over all shards: local FP64 sums on the GPU, then an all-reduce."""
    from . import dot
    s = np.zeros(2)
    for r in a.t:
        v = dot(a.t[r], b.t[r])
        s += (v.real, v.imag)
    s = a.comm.allreduce(s)
    return complex(s[0], s[1])


def sharded_norm(a):
    return math.sqrt(max(0.0, sharded_dot(a, a).real))


def _axpy(y, c, x):
    from . import axpy
    for r in y.t:
        axpy(y.t[r], c, x.t[r])


def _scale(v, c):
    from . import scale
    for r in v.t:
        scale(v.t[r], c)


def sharded_evolve(ham, psi, t, beta=0.0, krydim=5, tol=None, max_iters=0):
    """psi <- exp(-(beta + i t) H) psi for a sharded state, in place.

    The reference's restarted Krylov (inc/algo.h:77-173, 267-365): the same
    pass criterion (eta = 1/sqrt 2, at most three passes, the first
    comparison against eta/2), breakdown rule, Hfull growth (Eiermann-Ernst)
    and convergence test ||Hexp0|| < tol; each pass projects on all basis
    vectors at once (one all-reduce).  Returns the counts."""
    from .stepper import expm_first_columns
    if t == 0.0 and beta == 0.0:
        return {"restarts": 0, "applies": 0, "passes": 0}
    if tol is None:
        tol = float(np.finfo(np.float32 if ham.dtype == "c64" else np.float64).eps)
    m = int(krydim)
    beta0 = sharded_norm(psi)
    if beta0 == 0.0:
        return {"restarts": 0, "applies": 0, "passes": 0}
    V = [Shards.empty_like(psi) for _ in range(m + 1)]
    peer = getattr(ham, "exchange", "copy") == "peer"
    if peer:
        for v in V:
            v.share()
    for r in psi.t:
        V[0].t[r].copy_(psi.t[r])
    _scale(V[0], 1.0 / beta0)
    y = Shards.empty_like(psi)
    for r in y.t:
        y.t[r].zero_()
    eta = 1.0 / math.sqrt(2.0)
    f = -(beta + 1j * t)
    Hfull = np.zeros((0, 0), dtype=np.complex128)
    oldbeta = 0.0
    stats = {"restarts": 0, "applies": 0, "passes": 0}
    cycle = 0
    while True:
        cycle += 1
        H = np.zeros((m, m), dtype=np.complex128)
        m_eff, broke, nrm_w = m, False, 0.0
        for j in range(m):
            w = V[j + 1]
            ham.apply(w, V[j])
            stats["applies"] += 1
            old, norm, niter = 1.0, eta / 2, 0
            hacc = np.zeros(j + 1, dtype=np.complex128)
            while niter < 3 and norm != 0.0 and norm < eta * old:
                niter += 1
                loc = np.zeros(2 * (j + 1))
                from . import dot
                for i in range(j + 1):
                    for r in w.t:
                        v = dot(V[i].t[r], w.t[r])
                        loc[2 * i] += v.real
                        loc[2 * i + 1] += v.imag
                tot = psi.comm.allreduce(loc)
                h = tot[0::2] + 1j * tot[1::2]
                hacc += h
                for i in range(j + 1):
                    _axpy(w, -h[i], V[i])
                old, norm = norm, sharded_norm(w)
                stats["passes"] += 1
            H[:j + 1, j] = hacc
            nrm_w = norm
            if not (norm != 0.0 and norm >= eta * old):
                m_eff, broke = j + 1, True
                break
            if j != m - 1:
                H[j + 1, j] = norm
            _scale(w, 1.0 / norm)
        # Hfull = [OldHfull 0; 0..0 oldbeta H] (inc/algo.h:303-328)
        base = Hfull.shape[0]
        Hn = np.zeros((base + m_eff, base + m_eff), dtype=np.complex128)
        Hn[:base, :base] = Hfull
        if cycle > 1:
            Hn[base, base - 1] = oldbeta
        Hn[base:, base:] = H[:m_eff, :m_eff]
        Hfull = Hn
        col = expm_first_columns(Hfull, [f])[0]
        hexp0 = col[base:]
        for i in range(m_eff):
            _axpy(y, beta0 * hexp0[i], V[i])
        nrm = float(np.linalg.norm(hexp0))
        stats["restarts"] = cycle
        if (max_iters and cycle >= max_iters) or broke or nrm < tol:
            break
        V[0], V[m] = V[m], V[0]
        oldbeta = nrm_w
    for r in psi.t:
        psi.t[r].copy_(y.t[r])
    if peer:
        for v in V:
            v.unshare()
    return stats
