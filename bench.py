#!/usr/bin/env python3
"""Benchmark of the REAPERS hot path on B200: Pauli-sum H.psi throughput.

Workload (default, ``--config syk56``): sparse SYK with N = 56 Majoranas on
28 qubits (state of 2^28 complex64 = 2 GiB), k = 8, i.e. 448 quartic terms,
H.psi in FP32.  ``--config syk48``: sparse SYK N = 48 (24 qubits), 384 terms, FP64.

A step is one H.psi product over the whole state.  The metric is H.psi HBM
GB/s: the compulsory DRAM bytes of one apply, (G_w + 1) * 2^L *
sizeof(element), divided by the device time of the kernel.  G_w is the number
of distinct source blocks per block of output tiles in flight (the kernel's
window of 296 tiles of 2^12 elements: distinct x >> 20 for the N = 56
Hamiltonian); every such source block must come from HBM once per window and
the output is written once.  Inputs are larger than L2 (2 GiB vs 126 MB), so
no flush is needed between steps.

Multi-GPU (torchrun): every rank runs an independent replica (its own
disorder realisation); no collective on the data path ("replicas only");
the value is the sum over ranks of bytes / the max over ranks of time.

``--impl reference`` times the reference's own CPU implementation
(oracle/_ref/ref_driver: SpinOp::apply in CPUImpl::apply_ops's loop, OpenMP
over all host threads) on a bounded slice of output rows of the same
workload, in the same unit: the bytes of the whole apply scaled by the
fraction of rows computed, i.e. a rate extrapolated from the row sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("H·psi HBM GB/s; N=56 SYK OTOC pts/s, mixed+batched vs FP64 on B200 @1e-6")

CONFIGS = {
    "syk56": dict(N=56, k=8, dtype="c64", workload="sparse SYK N=56 (28 qubits, 2^28 complex64 = 2 GiB), "
               "k=8, 448 quartic terms, H.psi in FP32"),
    "syk48": dict(N=48, k=8, dtype="c128", workload="sparse SYK N=48 (24 qubits, 2^24 complex128 = 256 MiB), "
               "k=8, 384 quartic terms, H.psi in FP64"),
}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


PROFILE_SUMMARY = {"syk56": "k_apply_rows_sparse_syk_n56_fp32.md"}


def profile_traffic(cfg_name):
    """DRAM bytes (read + write) per launch of the apply kernel, from the
    committed ncu summary of the same kernel and workload (None if absent)."""
    name = PROFILE_SUMMARY.get(cfg_name)
    p = os.path.join(ROOT, "profiles", name) if name else None
    if p and os.path.exists(p):
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clk_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.index)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx = float(parts[1])
                except ValueError:
                    continue
                for n, v in zip(names, parts[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons)}


def on_chip_bound(info, L, cfg, t_step, clocks):
    """The shared-memory gather roofline of the row kernel: every
    element-term reads one element from shared memory and every source tile
    is written into it once; an SM moves 128 bytes per clock."""
    esz = 8 if cfg["dtype"] == "c64" else 16
    D = 1 << L
    smem_bytes = info["smem_bytes"]
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    sms = 148
    peak = 128 * sms * mhz * 1e6 / 1e9
    ach = smem_bytes / t_step / 1e9
    return {"resource": "shared-memory bandwidth (128 B/clk/SM x 148 SMs at the "
                        "measured SM clock)", "bytes_per_launch": smem_bytes,
            "achieved": round(ach, 1), "peak": round(peak, 1), "unit": "GB/s",
            "frac": round(ach / peak, 4)}


def otoc_leg(cfg, bits, coeff, seed, npts=2, krydim=16, last=True):
    """N = 56 OTOC F(t) = <psi0| W(t) V W(t) V |psi0> (W = b_{N-1}, V = b_{N-2},
    the operators of examples/simple-syk-krylov.cc) on a bounded sample of the
    20-point time grid on [0, 15] (t = 0, the first `npts` points and, with
    `last`, the final point t = 15, where the evolves restart most), one
    disorder realisation x one state, m = 16, for the plain FP64 path
    (reference default tol = FP64 epsilon) and the mixed path (FP32 vectors
    and H.psi, FP64 inner products / Hessenberg / expm, tol = FP32 epsilon).
    Error: max |F_mixed - F_fp64| / |F_fp64(0)| over the sampled points, and
    per point; time and H.psi count per point."""
    import torch
    import reapers_b200 as rb
    L = cfg["N"] // 2
    N = cfg["N"]
    grid = np.linspace(0.0, 15.0, 20)
    times = [0.0] + list(grid[1:1 + npts]) + ([float(grid[-1])] if last and npts < 19 else [])
    mb, mc = rb.syk.majoranas(N)
    out = {"workload": f"sparse SYK N={N} (2^{L}), k={cfg['k']}, 1 realisation x 1 state, "
                       f"t in {[float(round(t, 4)) for t in times]} of the 20-point grid on [0, 15], "
                       f"m={krydim}",
           "operators": "W = b_{N-1}, V = b_{N-2} (non-block Majoranas)"}
    psi64 = rb.random_state(L, "c128", seed=seed, normalize=True)
    res = {}
    for name, dt, tol in (("fp64_plain", "c128", float(np.finfo(np.float64).eps)),
                          ("mixed_fp32", "c64", float(np.finfo(np.float32).eps))):
        ham = rb.Hamiltonian(L, bits, coeff, dt)
        w = rb.Hamiltonian(L, mb[N - 1:N], mc[N - 1:N], dt)
        v = rb.Hamiltonian(L, mb[N - 2:N - 1], mc[N - 2:N - 1], dt)
        if dt == "c128":
            psi0 = psi64
        else:
            psi0 = torch.empty(1 << L, dtype=torch.complex64, device="cuda")
            rb.copy(psi0, psi64)
        vals, per_s, per_ap = [], [], []
        for t in times:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            val, ap = rb.otoc(ham, w, v, psi0, [t], krydim, tol)
            torch.cuda.synchronize()
            per_s.append(time.perf_counter() - t0)
            per_ap.append(int(ap))
            vals.append(val[0])
        vals = np.array(vals)
        el = float(sum(per_s))
        res[name] = vals
        npt = len(times) - 1   # t = 0 costs no evolve
        out[name] = {"seconds": round(el, 3), "pts_per_s": round(npt / el, 5),
                     "applies": int(sum(per_ap)), "tol": tol,
                     "seconds_per_point": [round(x, 3) for x in per_s],
                     "applies_per_point": per_ap,
                     "F": [[round(z.real, 10), round(z.imag, 10)] for z in vals]}
        del ham, w, v
        if dt == "c64":
            del psi0
        rb._lib.call("rp_workspace_release")
        torch.cuda.empty_cache()
    f0 = abs(res["fp64_plain"][0])
    per = np.abs(res["mixed_fp32"] - res["fp64_plain"]) / f0
    out["mixed_max_rel_err_vs_fp64"] = float(np.max(per))
    out["mixed_rel_err_per_point"] = [float(x) for x in per]
    out["speedup_mixed_vs_fp64"] = round(out["fp64_plain"]["seconds"] /
                                         out["mixed_fp32"]["seconds"], 3)
    out["speedup_mixed_vs_fp64_per_point"] = [
        round(a / b, 3) if b > 0 else None
        for a, b in zip(out["fp64_plain"]["seconds_per_point"],
                        out["mixed_fp32"]["seconds_per_point"])]
    return out


def otoc_full_leg(cfg, nreal, nstates, krydim=16, npts=20, seed0=1000, first=0, first_state=0):
    """The N = 56 OTOC workload as stated: nreal disorder realisations x
    nstates random states, F(t) at all `npts` points of the grid on [0, 15],
    m = 16, in the plain FP64 path and the mixed path, through otoc_leg's
    sequence (W = b_{N-1}, V = b_{N-2}).  Reports the time of both paths over
    the whole set, the speed-up, and the largest |F_mixed - F_fp64| / |F(0)|
    over every problem and point."""
    import reapers_b200 as rb
    out = {"workload": f"sparse SYK N={cfg['N']} (2^{cfg['N'] // 2}), k={cfg['k']}, {nreal} "
                       f"realisations x {nstates} states, {npts} points on [0, 15], m={krydim}",
           "problems": []}
    tot = {"fp64_plain": 0.0, "mixed_fp32": 0.0}
    err = 0.0
    for r in range(first, first + nreal):
        bits, coeff = rb.syk.sparse_syk(cfg["N"], k=cfg["k"], seed=seed0 + r)
        for st in range(first_state, first_state + nstates):
            leg = otoc_leg(cfg, bits, coeff, seed=7 + 31 * r + st, npts=npts - 1, krydim=krydim,
                           last=False)
            for k in tot:
                tot[k] += leg[k]["seconds"]
            err = max(err, leg["mixed_max_rel_err_vs_fp64"])
            out["problems"].append({"realisation": r, "state": st,
                                    "fp64_seconds": leg["fp64_plain"]["seconds"],
                                    "mixed_seconds": leg["mixed_fp32"]["seconds"],
                                    "fp64_applies": leg["fp64_plain"]["applies"],
                                    "mixed_applies": leg["mixed_fp32"]["applies"],
                                    "max_rel_err": leg["mixed_max_rel_err_vs_fp64"],
                                    "rel_err_per_point": leg["mixed_rel_err_per_point"],
                                    "F_fp64": leg["fp64_plain"]["F"]})
    npoints = nreal * nstates * (npts - 1)
    out["fp64_plain"] = {"seconds": round(tot["fp64_plain"], 2),
                         "pts_per_s": round(npoints / tot["fp64_plain"], 5)}
    out["mixed_fp32"] = {"seconds": round(tot["mixed_fp32"], 2),
                         "pts_per_s": round(npoints / tot["mixed_fp32"], 5)}
    out["speedup_mixed_vs_fp64"] = round(tot["fp64_plain"] / tot["mixed_fp32"], 3)
    out["mixed_max_rel_err_vs_fp64"] = err
    return out


def evolve_leg(seed=0, t=10.0, krydim=30, cpu=True):
    """exp(-iHt) psi for sparse SYK N = 48 (24 qubits, k = 8, 384 terms),
    one random state, m = 30, t = 10: the plain FP64 path (tol = FP64
    epsilon, the reference's default) against the mixed path (FP32 vectors
    and H.psi, FP64 inner products / Hessenberg / expm, tol = FP32 epsilon);
    error = ||psi_mixed - psi_fp64|| / ||psi_fp64||.  The reference CPU
    evolve is estimated from a timed sample of its H.psi (2^18 of 2^24
    output rows, all host threads) times the FP64 H.psi count -- a lower
    bound (its orthogonalisation is not counted), labelled as such."""
    import torch
    import reapers_b200 as rb
    cfg = CONFIGS["syk48"]
    N, L = cfg["N"], cfg["N"] // 2
    bits, coeff = rb.syk.sparse_syk(N, k=cfg["k"], seed=seed + 2000)
    psi64 = rb.random_state(L, "c128", seed=seed + 3, normalize=True)
    out = {"workload": f"exp(-iHt) psi, sparse SYK N={N} (2^{L}), k={cfg['k']}, t={t}, m={krydim}"}
    res = {}
    for name, dt, tol in (("fp64_plain", "c128", float(np.finfo(np.float64).eps)),
                          ("mixed_fp32", "c64", float(np.finfo(np.float32).eps))):
        ham = rb.Hamiltonian(L, bits, coeff, dt)
        x = psi64.clone() if dt == "c128" else torch.empty(1 << L, dtype=torch.complex64,
                                                           device="cuda")
        if dt == "c64":
            rb.copy(x, psi64)
        rb.evolve(ham, x.clone(), 0.05, 0.0, krydim, tol)   # warm-up (workspace, plan)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = rb.evolve(ham, x, t, 0.0, krydim, tol)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        res[name] = x.to(torch.complex128)
        out[name] = {"seconds": round(el, 4), "applies": st["applies"],
                     "restarts": st["restarts"], "tol": tol}
        ham.close()
        rb._lib.call("rp_workspace_release")
        torch.cuda.empty_cache()
    err = (torch.linalg.vector_norm(res["mixed_fp32"] - res["fp64_plain"]) /
           torch.linalg.vector_norm(res["fp64_plain"])).item()
    out["mixed_rel_err_vs_fp64"] = err
    out["speedup_mixed_vs_fp64"] = round(out["fp64_plain"]["seconds"] /
                                         out["mixed_fp32"]["seconds"], 3)
    # the reference's own restarted Krylov on its own GPU backend (GPUImpl,
    # cuBLAS BLAS-1 and krnl_apply_ops, built for sm_100a), same Hamiltonian,
    # t, m and tol, from its own random state
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
    if os.path.exists(drv):
        from oracle import oracle as O
        tf = os.path.join(tempfile.mkdtemp(prefix="rpgpu_"), "terms")
        O.write_terms(tf, L, bits, coeff)
        r = subprocess.run([drv, "evolve", tf, "64", repr(float(t)), str(krydim),
                            repr(float(np.finfo(np.float64).eps))],
                           capture_output=True, text=True, timeout=900)
        if r.returncode == 0:
            g = json.loads(r.stdout.strip().splitlines()[-1])
            out["reference_gpu_evolve"] = {
                "seconds": g["seconds"], "applies": g["applies"],
                "what": "the reference's State::evolve on its GPUImpl backend, sm_100a build"}
            out["speedup_fp64_vs_reference_gpu"] = round(g["seconds"] /
                                                          out["fp64_plain"]["seconds"], 1)
        else:
            out["reference_gpu_evolve"] = {"failed": r.stderr[-300:]}
    if cpu:
        try:
            cb = cpu_sample(cfg, bits, coeff, 0.0, 1 << 18)
            per_apply = cb["seconds"] * ((1 << L) / cb["rows"])
            est = per_apply * out["fp64_plain"]["applies"]
            out["cpu_reference_estimate"] = {
                "seconds_lower_bound": round(est, 2), "cores": cb["threads"],
                "kind": cb["kind"],
                "sample": f"{cb['sample']}: {per_apply:.3f} s per H.psi x "
                          f"{out['fp64_plain']['applies']} H.psi"}
            out["speedup_fp64_vs_cpu_estimate"] = round(est / out["fp64_plain"]["seconds"], 1)
        except Exception as e:   # a reported baseline only
            out["cpu_reference_estimate"] = {"failed": str(e)}
    return out


def shard_leg(ham, x, L, reps=3):
    """The state split by its top k qubits into 2^k shards, k = 1..3, as
    virtual shards on this GPU: every output shard by one peer-read launch
    (rp_apply_shard, the kernel a rank runs on its own GPU with the other
    shards in its peers' memory), all 2^k launches timed against the full
    apply; results bit-identical to it.  peer_tile_fraction: the share of
    source-tile loads a shard takes from other shards (terms whose X mask
    reaches the top k qubits) -- the NVLink share of the loads on 2^k GPUs."""
    import torch
    import reapers_b200 as rb
    st = rb.stream()
    full = torch.empty_like(x)

    def timed(fn):
        fn()
        rb.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    t_full = timed(lambda: ham.apply(full, x))
    xm = rb.syk.xmask(np.asarray(ham.bits, dtype=np.uint64))
    out = {"workload": f"the N=56 H.psi (2^{L} complex64) over 2^k virtual shards on one GPU, "
                       f"one peer-read launch per output shard",
           "full_apply_ms": round(t_full, 3), "shards": {}}
    for k in (1, 2, 3):
        n = x.numel() >> k
        shards = [x[s * n:(s + 1) * n] for s in range(1 << k)]
        outs = [torch.empty(n, dtype=x.dtype, device=x.device) for _ in shards]

        def run():
            for r in range(1 << k):
                ham.apply_shard(outs[r], shards, rank=r)
        t = timed(run)
        same = all(torch.equal(outs[r], full[r * n:(r + 1) * n]) for r in range(1 << k))
        rec = {"ms_all_shards": round(t, 3), "ms_per_shard": round(t / (1 << k), 3),
               "vs_full_apply": round(t_full / t, 4), "bit_identical": bool(same)}
        # source-tile groups (distinct x >> 12) whose shard offset x >> (L - k) is not 0
        xh = np.unique(xm >> np.uint64(12))
        rec["peer_tile_fraction"] = round(float(np.mean((xh >> np.uint64(L - k - 12)) != 0)), 4)
        rec["terms_reaching_top_qubits"] = int(np.count_nonzero(xm >> np.uint64(L - k)))
        out["shards"][f"k{k}"] = rec
        del outs
    del full
    return out


class DeviceClock:
    """CUDA events on the library stream (every apply of a sharded leg ends
    on it; the exchanges before it are ordered ahead through the legacy
    default stream, which the library's blocking stream follows)."""

    def __init__(self):
        import torch
        import reapers_b200 as rb
        self.st = rb.stream()
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def start(self):
        self.e0.record(self.st)

    def stop(self):
        self.e1.record(self.st)
        self.e1.synchronize()
        return self.e0.elapsed_time(self.e1) / 1e3


def sharded_dist_leg(comm, L, bits, coeff, dtype, steps, warmup, modes=("stage", "peer"),
                     full=None, make_state=None, clock=None):
    """The reference's multi-GPU split (inc/gpuimpl.h:426-432, src/krnl.cu:96-114)
    across the ranks of a process group: one state of 2^L elements split by its
    top k qubits over 2^k ranks, one shard per rank, and H.psi through
    reapers_b200.sharded.ShardedHamiltonian in each exchange mode --
    "stage" (every partner shard the terms reach swapped whole by NCCL
    send/recv, then one row-kernel launch) and "peer" (no copy: the launch
    reads the partner shards in the peers' memory over NVLink through CUDA
    IPC mappings, plain loads, no multicast).  Every rank holds the whole
    input (the same seeded state), so it also checks its output shard against
    the single-GPU apply of the full state (bit-identical expected).  Timing:
    `steps` applies after `warmup`, barrier and device synchronisation on
    both sides, device time (clock), the max over ranks.

    full / make_state / clock: the full operator class (the library's
    Hamiltonian unless given), a function making the full input state, and
    the timer (CUDA events on the library stream unless given) -- injectable
    so that a CPU process group (gloo) can drive the same plumbing."""
    from reapers_b200 import sharded as SH
    world = comm.world
    k = world.bit_length() - 1
    r = comm.owned()[0]
    n = 1 << (L - k)
    if full is None:
        import reapers_b200 as rb
        full = rb.Hamiltonian
    xfull = make_state()
    ref_op = full(L, bits, coeff, dtype)
    ref = _full_apply(ref_op, xfull)
    ref_op.close()
    xs = xfull[r * n:(r + 1) * n].clone()
    del xfull
    clock = clock or DeviceClock()
    out = {"workload": f"one state of 2^{L} elements split by its top {k} qubits over {world} "
                       f"ranks (one shard of 2^{L - k} per rank), H.psi per exchange mode",
           "modes": {}}
    for mode in modes:
        ham = SH.ShardedHamiltonian(L, bits, coeff, comm, dtype, exchange=mode, full=full)
        x = SH.Shards(comm, {r: xs})
        y = SH.Shards.empty_like(x)
        if mode == "peer":
            x.share()
        for _ in range(warmup):
            ham.apply(y, x)
        comm.barrier()
        clock.start()
        for _ in range(steps):
            ham.apply(y, x)
        t = clock.stop()
        comm.barrier()
        same = bool((y.t[r] == ref[r * n:(r + 1) * n]).all())
        times = comm.all_gather_object(t)
        oks = comm.all_gather_object(same)
        t_max = max(times)
        out["modes"][mode] = {"ms_per_apply": round(t_max / steps * 1e3, 4),
                              "ms_per_apply_by_rank": [round(v / steps * 1e3, 4) for v in times],
                              "bit_identical_to_full_apply": all(oks),
                              "partner_offsets": list(getattr(ham, "offsets", []))}
        if mode == "peer":
            x.unshare()
        ham.close()
        del x, y
    return out


def _full_apply(op, x):
    y = x.clone()
    op.apply(y, x)
    return y


def _tfim_chain(L, J=1.0, h=0.7):
    """Transverse-field Ising chain: J Z_i Z_{i+1} (open) + h X_i."""
    bits = [(1 << (2 * i + 1)) | (1 << (2 * i + 3)) for i in range(L - 1)]
    bits += [1 << (2 * i) for i in range(L)]
    coeff = [J] * (L - 1) + [h] * L
    return np.array(bits, dtype=np.uint64), np.array(coeff, dtype=np.complex128)


def spin_chain_leg(clocks=None, L=28, reps=10):
    """H.psi on two spin chains of 2^28 complex64 elements -- the XXZ chain
    (open, J = Jz = 1, fields U[-0.5, 0.5]) and the transverse-field Ising
    chain (J = 1, h = 0.7) -- on the row kernel's spin-chain variant (real Z
    strings summed into one per-row diagonal factor, terms with the same X
    mask sharing a row load), with the compulsory-DRAM and shared-memory
    fractions: where the kernel moves from shared-memory bound to HBM bound."""
    import torch
    import reapers_b200 as rb
    peak, _ = measured_peak()
    st = rb.stream()
    models = {"xxz": rb.syk.xxz_chain(L, 1.0, np.random.default_rng(1).uniform(-0.5, 0.5, L)),
              "tfim": _tfim_chain(L)}
    out = {"workload": f"spin chains of L={L} (2^{L} complex64): XXZ (open, fields U[-0.5, 0.5]), "
                       f"transverse-field Ising (J=1, h=0.7)"}
    x = rb.random_state(L, "c64", seed=3)
    y = torch.empty_like(x)
    for name, (bits, coeff) in models.items():
        ham = rb.Hamiltonian(L, bits, coeff, "c64")
        info = ham.info()
        for _ in range(3):
            ham.apply(y, x)
        rb.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            ham.apply(y, x)
        e1.record(st)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        dram = info["alg_bytes_dram"] / t / 1e9
        out[name] = {"terms": info["nterms"], "diag_terms": info["diag_terms"],
                     "source_tile_groups": info["ngroups"], "ms": round(t * 1e3, 4),
                     "compulsory_dram_GBps": round(dram, 1), "dram_frac": round(dram / peak, 4),
                     "on_chip": on_chip_bound(info, L, {"dtype": "c64"}, t, clocks)}
        ham.close()
    del x, y
    return out


def batch_leg(seed=0, points=(1, 2, 20, 39), krydim=16, nreal=64, nstates=8,
              sizes=(32, 36, 40), seq_per_size=2, tune=True):
    """The batched OTOC workload: nreal disorder realisations x nstates random
    states (64 x 8 = 512 problems), sparse SYK k = 8 with N cycling over
    `sizes` (16/18/20 qubits), at the `points` of the 40-point grid on
    [0, 20] (default: t = 0.51, 1.03, 10.26 and 20), m = krydim; one
    persistent launch per time step in a CUDA graph, tile loop and team size
    (or the single-problem path) per size from the autotuner.  Compared with
    the same problems run one at a time through the single-problem mixed path
    (rp_evolve), on seq_per_size problems per size."""
    import torch
    import reapers_b200 as rb
    from reapers_b200 import autotune
    grid = np.linspace(0.0, 20.0, 40)
    times = np.array([grid[i] for i in points])
    problems = []
    for r in range(nreal):
        N = sizes[r % len(sizes)]
        L = N // 2
        bits, coeff = rb.syk.sparse_syk(N, k=8, seed=seed * 100003 + r)
        mb, mc = rb.syk.majoranas(N)
        for s in range(nstates):
            psi = rb.random_state(L, "c64", seed=seed * 7919 + r * 64 + s, normalize=True)
            problems.append(dict(len=L, bits=bits, coeff=coeff, w=(mb[N - 1:N], mc[N - 1:N]),
                                 v=(mb[N - 2:N - 1], mc[N - 2:N - 1]), psi0=psi, N=N))
    tol = float(np.finfo(np.float32).eps)
    t0 = time.perf_counter()
    tuned = autotune.tune(problems, krydim=krydim, tol=tol) if tune else {}
    t_tune = time.perf_counter() - t0
    out = {"workload": f"{nreal} sparse-SYK realisations (k=8, N cycling {list(sizes)}) x "
                       f"{nstates} states = {len(problems)} problems, t in "
                       f"{[float(round(t, 4)) for t in times]} of 40 points on [0, 20], m={krydim}",
           "paths": {k: v.get("path", "batched") for k, v in tuned.items()},
           "tiles": {k: v["tile"] for k, v in tuned.items()},
           "teams": {k: v["team"] for k, v in tuned.items()},
           "tuning_seconds": round(t_tune, 2),
           "tuning_probe_seconds": {k: v["seconds"] for k, v in tuned.items()},
           "per_size": {}}
    tot_batch = tot_seq = tot_best = 0.0
    err = 0.0
    for N in sizes:
        idx = [i for i, p in enumerate(problems) if p["N"] == N]
        sub = [problems[i] for i in idx]
        b = rb.BatchOTOC(sub, krydim=krydim, tol=tol, max_restarts=16)
        b.run(times[:1], use_graph=True)    # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        F, ap = b.run(times, use_graph=True)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        b.close()
        # the same problems one at a time through the single-problem path
        t0 = time.perf_counter()
        for j in range(min(seq_per_size, len(sub))):
            p = sub[j]
            ham = rb.Hamiltonian(p["len"], p["bits"], p["coeff"], "c64")
            w = rb.Hamiltonian(p["len"], *p["w"], "c64")
            v = rb.Hamiltonian(p["len"], *p["v"], "c64")
            vals, _ = rb.otoc(ham, w, v, p["psi0"], times, krydim, tol)
            err = max(err, float(np.abs(vals - F[j]).max()))
        torch.cuda.synchronize()
        el2 = time.perf_counter() - t0
        pts = len(sub) * len(times)
        r_b = pts / el
        r_s = min(seq_per_size, len(sub)) * len(times) / el2
        out["per_size"][f"N{N}"] = {"problems": len(sub), "batched_pts_per_s": round(r_b, 3),
                                    "sequential_pts_per_s": round(r_s, 3),
                                    "batched_seconds": round(el, 3),
                                    "path": sub[0].get("path", "batched"),
                                    "batched_applies": int(ap.sum()),
                                    "applies_per_problem_per_point": [
                                        round(float(v), 1) for v in ap.mean(axis=0)]}
        tot_batch += pts / r_b
        tot_seq += pts / r_s
        tot_best += pts / max(r_b, r_s)
    pts = len(problems) * len(times)
    out["batched_pts_per_s"] = round(pts / tot_batch, 3)
    out["sequential_pts_per_s"] = round(pts / tot_seq, 3)
    out["per_size_best_pts_per_s"] = round(pts / tot_best, 3)
    out["speedup_batched_vs_sequential"] = round(tot_seq / tot_batch, 3)
    out["max_abs_diff_batched_vs_sequential"] = err
    # the whole batch at once, every size in one persistent launch per time
    # step and team size (largest problems first from the shared queue, the
    # smaller ones filling teams as they free up), the single-path shapes
    # after it
    b = rb.BatchOTOC(problems, krydim=krydim, tol=tol, max_restarts=16)
    b.run(times[:1], use_graph=True)    # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F_all, _ = b.run(times, use_graph=True)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    b.close()
    out["whole_batch_one_launch"] = {"seconds": round(el, 3), "pts_per_s": round(pts / el, 3),
                                     "speedup_vs_sequential": round(tot_seq / el, 3)}
    out["launches_per_time_step"] = 1
    out["cuda_graph"] = True
    return out


def step_leg(T=10.0, tol=1e-8, seed=0):
    """Learned (dt, m) step controller vs Expokit's plain step control at
    equal tolerance, on XXZ L=24 (J = Jz = 1, fields U[-W, W], W in {0.5, 3})
    and sparse SYK N=48 (k=8), FP64, exp(-iHT) psi with T = 10.  The network
    is the committed model (trained on the GPU on plain-method traces of
    smaller problems, reapers_b200/data); without it a small model is trained
    here first and the line says so."""
    import torch
    import reapers_b200 as rb
    from reapers_b200 import stepper as SP
    out = {"workload": f"exp(-iHT)psi, T={T}, tol={tol}, FP64; plain = Expokit step control "
                       f"with m=30; plain+stretch = the same, each accepted step extended on its "
                       f"basis when the estimate allows; learned = MLP-proposed (dt, m), m in "
                       f"[{SP.M_MIN}, {SP.M_MAX}], with the same extension",
           "problems": {}}
    if os.path.exists(SP.DEFAULT_MODEL):
        model = SP.StepModel.load()
        out["model"] = dict(model.meta, source="committed")
    else:
        t0 = time.perf_counter()
        runs = []
        for p in SP.training_problems(60, seed=seed + 1):
            runs.extend(SP.generate_traces([p]))
            p["ham"].close()
        X, Y = SP.make_dataset(runs)
        model, loss = SP.train(X, Y, epochs=40)
        out["model"] = dict(model.meta, source="trained in this run",
                            seconds=round(time.perf_counter() - t0, 2))
    rng = np.random.default_rng(seed + 2024)
    cases = [("xxz_L24_W0.5", 24, rb.syk.xxz_chain(24, 1.0, rng.uniform(-0.5, 0.5, 24))),
             ("xxz_L24_W3", 24, rb.syk.xxz_chain(24, 1.0, rng.uniform(-3.0, 3.0, 24))),
             ("sparse_syk_N48", 24, rb.syk.sparse_syk(48, k=8, seed=seed + 1000))]
    tot = {"plain": [0, 0.0], "plain+stretch": [0, 0.0], "learned": [0, 0.0]}
    for name, L, (bits, coeff) in cases:
        ham = rb.Hamiltonian(L, bits, coeff, "c128")
        psi = rb.random_state(L, "c128", seed=seed + 11)
        # warm-up: one small step of each basis size range
        SP.step_evolve(ham, psi.clone(), 1e-3, tol, SP.PlainController(30))
        res, finals = {}, {}
        for ctl in (SP.PlainController(30), SP.PlainController(30, stretch=True),
                    SP.LearnedController(model)):
            ps = psi.clone()
            st = SP.step_evolve(ham, ps, T, tol, ctl)
            st.pop("trace", None)
            rec = {"steps": st["steps"], "applies": st["applies"],
                   "seconds": round(st["seconds"], 4), "rejections": st["rejections"],
                   "err_estimate_sum": st["err_sum"], "modelled_vector_passes": st["cost"],
                   "stretched_steps": st["stretched"]}
            if ctl.name == "learned":
                rec["proposals"] = st["proposals"]
                rec["accepted_fraction"] = round(st["proposals_accepted"] / max(1, st["proposals"]), 4)
                rec["ms_in_mlp"] = round(st["ms_mlp"], 3)
            res[ctl.name] = rec
            finals[ctl.name] = ps
            tot[ctl.name][0] += st["applies"]
            tot[ctl.name][1] += st["seconds"]
        res["final_state_diff"] = float(torch.linalg.vector_norm(finals["plain"] -
                                                                 finals["learned"]).item())
        res["speedup_wall"] = round(res["plain"]["seconds"] / res["learned"]["seconds"], 3)
        res["speedup_wall_vs_stretch"] = round(res["plain+stretch"]["seconds"] /
                                               res["learned"]["seconds"], 3)
        res["applies_ratio"] = round(res["learned"]["applies"] / res["plain"]["applies"], 3)
        out["problems"][name] = res
        del finals, psi
        ham.close()
        torch.cuda.empty_cache()
    model.close()
    out["total_applies"] = {k: v[0] for k, v in tot.items()}
    out["total_seconds"] = {k: round(v[1], 4) for k, v in tot.items()}
    out["speedup_wall_total"] = round(tot["plain"][1] / tot["learned"][1], 3)
    out["speedup_wall_total_vs_stretch"] = round(tot["plain+stretch"][1] / tot["learned"][1], 3)
    return out


def gpu_reference_leg(cfg, bits, coeff, t_ours, reps=3):
    """The reference's own GPU kernel (krnl_apply_ops, one thread per element,
    src/krnl.cu:81-94, launched by GPUImpl::apply_ops, src/krnl.cu:220-257),
    compiled for sm_100a from its sources (oracle/_ref/ref_gpu_driver), timed on
    the same Hamiltonian and state size on this GPU with CUDA events: a
    GPU-side baseline beside the CPU one.  Its results equal the product's
    (tests/test_gpu_ref_kernel.py)."""
    from oracle import oracle as O
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
    if not os.path.exists(drv):
        return {"unavailable": "oracle/_ref/ref_gpu_driver was not built"}
    L = cfg["N"] // 2
    tmp = tempfile.mkdtemp(prefix="rpgpu_")
    tf = os.path.join(tmp, "terms")
    O.write_terms(tf, L, bits, coeff)
    fp = "32" if cfg["dtype"] == "c64" else "64"
    r = subprocess.run([drv, "bench", tf, fp, str(reps)], capture_output=True, text=True,
                       timeout=900)
    if r.returncode != 0:
        return {"failed": r.stderr[-300:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"kernel": "reference krnl_apply_ops (GPUImpl), sm_100a build of src/krnl.cu",
            "ms_per_apply": d["ms_per_apply"], "reps": reps,
            "ours_ms_per_apply": round(t_ours * 1e3, 3),
            "speedup_ours_vs_reference_gpu": round(d["ms_per_apply"] / (t_ours * 1e3), 2)}


def make_terms(cfg, seed):
    import reapers_b200 as rb
    return rb.syk.sparse_syk(cfg["N"], k=cfg["k"], seed=seed)


def cpu_reference(cfg, bits, coeff, alg_bytes, rows, reps):
    """Time the reference CPU apply on a slice of `rows` output rows."""
    from oracle import oracle as O
    L = cfg["N"] // 2
    tmp = tempfile.mkdtemp(prefix="rpbench_")
    tf = os.path.join(tmp, "terms")
    O.write_terms(tf, L, bits, coeff)
    fp = "32" if cfg["dtype"] == "c64" else "64"
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    env.setdefault("OMP_PROC_BIND", "close")
    drv, isa = O.bench_driver()
    r = subprocess.run([drv, "bench_rows", tf, fp, "0", str(rows), str(reps)],
                       capture_output=True, text=True, check=True, env=env)
    d = json.loads(r.stdout)
    D = 1 << L
    return {"value": alg_bytes * (rows / D) / d["seconds"] / 1e9, "seconds": d["seconds"],
            "threads": d["threads"], "rows": rows, "isa": isa}


PORT_ROWS = 1 << 15   # output rows per timed sample of the oracle's port


def port_state(cfg, seed=7):
    """A random state of the workload's size and precision, resident in host
    memory, for the port's timed samples."""
    L = cfg["N"] // 2
    real = np.float32 if cfg["dtype"] == "c64" else np.float64
    v = np.random.default_rng(seed).standard_normal(2 << L, dtype=real)
    return v.view(np.complex64 if real is np.float32 else np.complex128)


def port_reference(cfg, bits, coeff, alg_bytes, rows, state):
    """Time the oracle's restatement of the reference CPU apply (SpinOp::apply
    summed over the terms in list order, inc/ops.h:421-440, as looped by
    CPUImpl::apply_ops, inc/cpuimpl.h:739-754) on the first `rows` output rows
    of `state`: the stand-in for the reference build where oracle/_ref was not
    built.  numpy, one host thread."""
    from oracle import oracle as O
    L = cfg["N"] // 2
    idx = np.arange(rows, dtype=np.uint64)
    t0 = time.perf_counter()
    O.apply_at(bits, coeff, idx, lambda j: state[j])
    dt = time.perf_counter() - t0
    return {"value": alg_bytes * (rows / (1 << L)) / dt / 1e9, "seconds": dt, "threads": 1,
            "rows": rows, "isa": "numpy"}


def cpu_sample(cfg, bits, coeff, alg_bytes, rows, state=None):
    """One timed sample of the reference's CPU apply over `rows` output rows:
    the reference build (oracle/_ref) where it was built, else the oracle's
    port over min(rows, PORT_ROWS) rows of `state` (port_state(cfg) when
    None).  Returns the timing with its 'kind' and a one-line 'sample'."""
    from oracle import oracle as O
    L = cfg["N"] // 2
    if O.ref_available():
        cb = cpu_reference(cfg, bits, coeff, alg_bytes, rows, 1)
        cb["kind"] = "reference"
        cb["sample"] = (f"reference SpinOp::apply (CPUImpl::apply_ops loop) over {rows} of "
                        f"2^{L} output rows, same terms, OpenMP {cb['threads']} threads "
                        f"({cb['isa']} build)")
    else:
        prow = min(rows, PORT_ROWS, 1 << L)
        cb = port_reference(cfg, bits, coeff, alg_bytes, prow,
                            port_state(cfg) if state is None else state)
        cb["kind"] = "port"
        cb["sample"] = (f"the oracle's restatement of SpinOp::apply over {prow} of 2^{L} "
                        f"output rows, same terms, numpy, 1 thread (the reference build "
                        f"oracle/_ref was absent)")
    return cb


def dist_setup(n):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def run_ours(args):
    import torch
    import reapers_b200 as rb

    cfg = CONFIGS[args.config]
    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    rb.init(local)
    L = cfg["N"] // 2
    bits, coeff = make_terms(cfg, seed=1000 + rank)
    ham = rb.Hamiltonian(L, bits, coeff, cfg["dtype"])
    info = ham.info()
    alg = info["alg_bytes"]
    x = rb.random_state(L, cfg["dtype"], seed=7 + rank, normalize=True)
    y = torch.empty_like(x)
    st = rb.stream()

    if args.profile:
        # one apply after a warm-up, for an ncu capture of the kernel
        ham.apply(y, x)
        rb.synchronize()
        ham.apply(y, x)
        rb.synchronize()
        print(json.dumps({"profile": True, "info": info}))
        return

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        ham.apply(y, x)
    torch.cuda.synchronize()
    rb.synchronize()
    clk = Clocks(local)
    clk.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        ham.apply(y, x)
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    t_step = e0.elapsed_time(e1) / 1e3 / args.steps
    t_max = t_step
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([t_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    # the kernel's compulsory DRAM bytes: every distinct source block of the
    # tile window read once per window, plus the write
    alg_dram = info["alg_bytes_dram"]
    value = alg_dram * world / t_max / 1e9
    achieved_dram = alg_dram / t_step / 1e9

    # end to end through the public API with host buffers: every step copies
    # its input state from pinned host memory to the device, applies H and
    # copies the result back (rp_apply_host: the copies of neighbouring steps
    # overlap the product on separate streams)
    esize = 8 if cfg["dtype"] == "c64" else 16
    nbytes = (1 << L) * esize
    hx = torch.empty(1 << L, dtype=x.dtype, pin_memory=True)
    hy = [torch.empty_like(hx, pin_memory=True) for _ in range(2)]
    hx.copy_(x.cpu())
    del y
    torch.cuda.empty_cache()
    k2 = max(3, args.steps)
    ham.apply_host(hy[:1], [hx])   # warm-up (allocates the pipeline buffers)
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(st)
    ham.apply_host([hy[i & 1] for i in range(k2)], [hx] * k2)
    f1.record(st)
    f1.synchronize()
    t_e2e = f0.elapsed_time(f1) / 1e3 / k2
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    rb._lib.call("rp_workspace_release")
    e2e_value = alg_dram * world / t_e2e / 1e9

    peak, peak_kind = measured_peak()
    traffic = profile_traffic(args.config)
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_max * 1e3, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (complex64)" if cfg["dtype"] == "c64" else "f64 (complex128)",
        "data": "synthetic: sparse SYK quartets drawn uniformly without replacement (seeded), "
                "couplings N(0,1) x the reference's SYK scale; i.i.d. complex Gaussian state",
        "config": {"workload": cfg["workload"], "tile_exp": info["tile_exp"],
                   "source_tile_groups": info["ngroups"], "terms": info["nterms"],
                   "hbm_bytes_per_apply": alg_dram,
                   "hbm_bytes_rule": "(G_w + 1) * 2^L * element size: distinct source "
                                     "blocks of the kernel's tile window, plus the write",
                   "staged_tile_bytes_per_apply": alg,
                   "staged_rate_GBps": round(alg / t_step / 1e9, 1),
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (state >> 126 MB), no flush"},
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "ms_per_step": round(t_e2e * 1e3, 3)},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved_dram, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved_dram / peak, 4), "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                                       "one launch, from the committed profile summary of this "
                                       "kernel and workload (not measured in this run)"
                     if traffic else None,
                     "alg_bytes_per_launch": alg_dram,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "on_chip": on_chip_bound(info, L, cfg, t_step, clocks),
                     "term_applications_per_s": info["nterms"] * (1 << L) / t_step},
        "clocks": clocks,
    }
    # the reference's multi-GPU split of one state (N > 1): every rank takes
    # part, so it runs before the single-GPU legs
    if world > 1 and (world & (world - 1)) == 0 and world <= 8 and not args.no_shard:
        from reapers_b200 import sharded as SH
        ham.close()
        del x, ham
        torch.cuda.empty_cache()
        sbits, scoeff = make_terms(cfg, seed=1000)
        # the value above is measured; a failure of this leg (e.g. no peer
        # access between the GPUs) is recorded, not raised, so the line is
        # still printed (a rank's failed collective ends by the process
        # group's timeout on the others)
        try:
            line["sharded_split_syk56"] = sharded_dist_leg(
                SH.ProcessGroupComm(), L, sbits, scoeff, cfg["dtype"], steps=10, warmup=3,
                make_state=lambda: rb.random_state(L, cfg["dtype"], seed=7, normalize=False))
        except Exception as e:   # noqa: BLE001 -- reported in the JSON line
            line["sharded_split_syk56"] = {"failed": f"{type(e).__name__}: {e}"[:400]}
    # the single-GPU characterisation legs run only at N = 1 (under torchrun
    # every rank would repeat them while all GPUs are held)
    legs = world == 1
    if legs and not args.no_refgpu:
        line["gpu_reference_kernel"] = gpu_reference_leg(cfg, bits, coeff, t_step)
    if legs and args.config == "syk56" and not args.no_chains:
        line["hpsi_spin_chains_l28"] = spin_chain_leg(clocks)
    # the sharded leg uses this leg's Hamiltonian and state, so it runs
    # before the OTOC leg frees them
    if legs and args.config == "syk56" and not args.no_shard:
        line["sharded_peer_syk56"] = shard_leg(ham, x, L)
    if legs and args.config == "syk56" and (not args.no_otoc or args.otoc_full):
        ham.close()
        del x, ham
        torch.cuda.empty_cache()
    if legs and args.config == "syk56" and not args.no_otoc:
        line["otoc"] = otoc_leg(cfg, bits, coeff, seed=7 + rank, npts=args.otoc_points)
    if legs and args.config == "syk56" and args.otoc_full:
        spec, _, first = args.otoc_full.partition("+")
        nr, ns = (int(v) for v in spec.split("x"))
        line["otoc_full"] = otoc_full_leg(cfg, nr, ns, first=int(first or 0),
                                          first_state=args.otoc_first_state)
    if legs and args.config == "syk56" and not args.no_evolve:
        line["evolve_syk48"] = evolve_leg(seed=rank, cpu=(rank == 0 and world == 1 and not args.no_cpu))
    if legs and args.config == "syk56" and not args.no_batch:
        line["otoc_batched_syk32_40"] = batch_leg(seed=rank)
    if legs and args.config == "syk56" and not args.no_steps:
        line["learned_steps"] = step_leg(seed=rank)
    if rank == 0 and world == 1 and not args.no_cpu:
        rows = 1 << 20 if cfg["N"] >= 56 else 1 << 18
        try:
            cb = cpu_sample(cfg, bits, coeff, alg_dram, rows)
            line["cpu_baseline"] = {"value": round(cb["value"], 4), "unit": "GB/s",
                                    "cores": cb["threads"], "kind": cb["kind"],
                                    "sample": f"{cb['sample']}, {cb['seconds']:.2f} s; value "
                                              f"= the whole apply's HBM bytes x the row "
                                              f"fraction / time (extrapolated from the "
                                              f"sample)"}
        except Exception as e:   # the baseline is reported, never the target
            line["cpu_baseline"] = {"value": None, "unit": "GB/s", "cores": os.cpu_count(),
                                    "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        if "failed" in line.get("sharded_split_syk56", {}):
            # a collective of the failed leg may have left the communicator
            # aborted: end without the teardown, which could wait on it
            sys.stdout.flush()
            os._exit(0)
        dist.destroy_process_group()


def run_reference(args):
    cfg = CONFIGS[args.config]
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    L = cfg["N"] // 2
    bits, coeff = make_terms(cfg, seed=1000)
    # the bytes are those of our arm's plan (host-side grouping), so both arms
    # report the same unit for the same work
    alg = alg_bytes_host(L, bits, cfg["dtype"])
    rows = 1 << 19 if cfg["N"] >= 56 else 1 << 17
    state = None if O.ref_available() else port_state(cfg)
    times = []
    for i in range(args.warmup + args.steps):
        cb = cpu_sample(cfg, bits, coeff, alg, rows, state)
        if i >= args.warmup:
            times.append(cb["seconds"])
    t = float(np.mean(times))
    value = alg * (cb["rows"] / (1 << L)) / t / 1e9
    sample = (f"{cb['sample']} per step; value = the whole apply's HBM bytes x the row "
              f"fraction / time, i.e. extrapolated from the row sample")
    line = {"metric": METRIC, "value": round(value, 4), "unit": "GB/s", "impl": "reference",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (complex64)" if cfg["dtype"] == "c64" else "f64 (complex128)",
            "data": "synthetic (same generator and seed as our arm)",
            "config": {"workload": cfg["workload"], "sample": sample,
                       "value_is": "extrapolated from a row sample"},
            "cpu_baseline": {"value": round(value, 4), "unit": "GB/s",
                             "cores": cb["threads"], "kind": cb["kind"], "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def alg_bytes_host(L, bits, dtype, sms=148):
    """The row kernel's compulsory DRAM bytes, (G_w + 1) * 2^L * element size,
    computed on the host as the kernel's plan does: tiles of 2^B elements
    (B = 12 for complex64, 11 for complex128), a window of min(tiles, 2 x SMs)
    CTAs, G_w = distinct x >> (B + floor(log2 window))."""
    import reapers_b200.syk as S
    B = 12 if dtype == "c64" else 11
    win = min(1 << max(L - B, 0), 2 * sms)
    lw = 0
    while (2 << lw) <= win:
        lw += 1
    x = S.xmask(bits)
    G_w = len(np.unique(x >> np.uint64(B + lw)))
    return (G_w + 1) * (1 << L) * (8 if dtype == "c64" else 16)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="syk56")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-chains", action="store_true",
                    help="skip the spin-chain H.psi leg (XXZ, transverse-field Ising)")
    ap.add_argument("--no-shard", action="store_true",
                    help="skip the peer-read sharded H.psi leg (virtual shards on one GPU)")
    ap.add_argument("--no-otoc", action="store_true", help="skip the N=56 OTOC leg")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip the reference's own GPU kernel (sm_100a build) timed beside ours")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched OTOC leg (sparse SYK N = 32/36/40)")
    ap.add_argument("--no-evolve", action="store_true", help="skip the N = 48 FP64 vs mixed evolve leg")
    ap.add_argument("--no-steps", action="store_true",
                    help="skip the learned step-controller leg")
    ap.add_argument("--otoc-points", type=int, default=2,
                    help="non-zero time points of the 20-point grid on [0, 15] in the N = 56 OTOC sample")
    ap.add_argument("--otoc-full", default="",
                    help="RxS[+F]: also run the N = 56 OTOC on R realisations (from number F, "
                         "default 0) x S states at all 20 points in both precisions (e.g. 4x2; "
                         "minutes per problem)")
    ap.add_argument("--otoc-first-state", type=int, default=0,
                    help="first random state of --otoc-full (states first .. first + S - 1)")
    ap.add_argument("--profile", action="store_true",
                    help="run two applies and exit (for an ncu capture)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
