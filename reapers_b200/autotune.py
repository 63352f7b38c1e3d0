"""Autotuner for the batched OTOC: tile loop, team size, or the single-problem path.

For every distinct (qubit count, number of source-tile groups, precision,
Krylov dimension) in a batch, the tuner times one whole OTOC point (the
four evolves, the two string products and the inner product, at the batch's
own time `t_probe`) on a sample of the batch's problems of that shape, for
each candidate:

* the persistent batched launch with tile exponent B (12: the 2-D TMA
  row-tile loop; 8..11: the bulk-copy loop, tried below 2^14 elements) and
  team size C (CTAs per problem, a thread-block cluster) in 1, 2, 4, 8, 16
  with C <= 2^(L-B) tiles (see ``candidates``);
* the single-problem path (``reapers_b200.otoc``: each problem alone on the
  whole GPU, the H.psi row kernel on every SM), timed on a few problems and
  scaled to the sample.

A point costs what its Krylov cycles, projections, the team leader's Hfull
exponential and the cluster barriers cost, which a probe of H.psi products
alone does not see.  The winner per shape is cached in a JSON file
(``RPB200_TUNE_CACHE`` or ``~/.cache/reapers_b200/tune.json``) keyed by
``L{len}-G{groups at B=11, to the nearest 32}-c64-m{krydim}-p``, so later
batches of the same shape skip the search.  Problems tuned to the single
path are run one at a time by ``BatchOTOC`` after the batched launches.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import syk as S

SINGLE = "single"


def cache_path():
    return os.environ.get("RPB200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "reapers_b200",
                                       "tune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(d):
    """Write the cache; an unwritable location only costs the next batch a
    new search, so it is not an error."""
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
        return True
    except OSError:
        return False


def shape_key(prob, krydim):
    """Problems of one qubit count whose group counts fall in the same bin of
    32 share a tuning (disorder realisations of one model differ slightly)."""
    L = int(prob["len"])
    g = len(np.unique(S.xmask(prob["bits"]) >> np.uint64(min(11, L))))
    return f"L{L}-G{32 * round(g / 32)}-c64-m{krydim}-p"


def candidates(L):
    """(B, C) pairs of the batched launch tried for L qubits: every tile
    exponent and team size below 2^14 elements; from there the row-tile loop
    (B = 12), and from 2^16 elements teams of 2 to 8 CTAs.  Timed by whole
    OTOC points on the B200 (sparse SYK, 16-20 qubits), teams of 2 won at
    every size; one CTA per problem took 1.7-1.8x longer (a problem's
    vectors stream through one SM) and teams of 16 1.3x (their cluster
    barriers and the leader CTA's expm cost more than the bandwidth they
    add), so those two are not searched there."""
    if L < 14:
        return [(B, C) for B in range(8, min(12, L) + 1) for C in (1, 2, 4, 8, 16)
                if C <= (1 << (L - B))]
    teams = (1, 2, 4, 8, 16) if L < 16 else (2, 4, 8)
    return [(12, C) for C in teams if C <= (1 << (L - 12))]


def _time_batched(probs, krydim, tol, max_restarts, t_probe):
    import torch
    from . import BatchOTOC
    b = BatchOTOC(probs, krydim=krydim, tol=tol, max_restarts=max_restarts)
    try:
        b.run([0.1 * t_probe], use_graph=False)           # warm-up (tables, workspaces)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run([t_probe], use_graph=False)
        torch.cuda.synchronize()
        return time.perf_counter() - t0
    finally:
        b.close()


def _time_single(probs, krydim, tol, t_probe, nsingle):
    import torch
    from . import Hamiltonian, otoc
    sub = probs[:nsingle]
    hams = [(Hamiltonian(p["len"], p["bits"], p["coeff"], "c64"),
             Hamiltonian(p["len"], *p["w"], "c64"), Hamiltonian(p["len"], *p["v"], "c64"))
            for p in sub]
    try:
        h, w, v = hams[0]
        otoc(h, w, v, sub[0]["psi0"], [0.1 * t_probe], krydim, tol)   # warm-up (workspace)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for (h, w, v), p in zip(hams, sub):
            otoc(h, w, v, p["psi0"], [t_probe], krydim, tol)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * len(probs) / len(sub)
    finally:
        for trio in hams:
            for x in trio:
                x.close()


def tune(problems, krydim=16, tol=1.2e-7, max_restarts=16, t_probe=0.3, sample=None,
         nsingle=4, force=False, log=None):
    """Set problems[i]['tile'] / ['team'] to the tuned pair, or
    problems[i]['path'] = 'single'; returns {key: record}."""
    import torch
    cache = {} if force else _load()
    by_key = {}
    for i, p in enumerate(problems):
        by_key.setdefault(shape_key(p, krydim), []).append(i)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = {}
    for key, idx in by_key.items():
        if key not in cache:
            L = int(problems[idx[0]]["len"])
            # the shape's own problems, up to two per SM: a class that needs a
            # second wave of teams (168 problems on 148 two-CTA teams) must be
            # timed with it, or its tail goes unseen
            n = sample or min(len(idx), 2 * sms)
            base = [problems[j] for j in idx[:n]]
            timings = {}
            for B, C in candidates(L):
                probs = [dict(p, tile=B, team=C) for p in base]
                timings[f"B{B}-C{C}"] = _time_batched(probs, krydim, tol, max_restarts, t_probe)
            timings[SINGLE] = _time_single(base, krydim, tol, t_probe, min(nsingle, n))
            best = min(timings, key=timings.get)
            rec = {"seconds": timings, "sample": n, "probe": f"one OTOC point at t={t_probe}"}
            if best == SINGLE:
                rec.update(path=SINGLE, tile=0, team=0)
            else:
                B, C = (int(v[1:]) for v in best.split("-"))
                rec.update(path="batched", tile=B, team=C)
            cache[key] = rec
            if log:
                log(f"autotune {key}: {timings} -> {best}")
        rec = cache[key]
        for j in idx:
            problems[j]["tile"] = int(rec["tile"])
            problems[j]["team"] = int(rec["team"])
            problems[j]["path"] = rec.get("path", "batched")
        out[key] = rec
    _save(cache)
    return out
