"""Autotuner for the batched OTOC kernel's tile exponent and team size.

For every distinct (qubit count, number of source-tile groups, precision,
Krylov dimension) in a batch, the tuner times one persistent launch doing
two H.psi products per problem (rp_batch_probe) on a sample of the batch's
own problems of that size (up to one per SM, so the memory system is loaded
as in the real run), for each tile exponent B in 8..min(12, L) (12: the
row-tile loop) and each
team size (CTAs per problem, a thread-block cluster) C in 1, 2, 4, 8, 16
with C <= 2^(L-B) tiles, and keeps the fastest pair.  Results are cached in
a JSON file (``RPB200_TUNE_CACHE`` or ``~/.cache/reapers_b200/tune.json``)
keyed by ``L{len}-G{groups at B=11, to the nearest 32}-c64-m{krydim}-t``, so
later batches of the same shape skip the search.
"""
from __future__ import annotations

import json
import os


import numpy as np

from . import syk as S


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
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def shape_key(prob, krydim):
    """Problems of one qubit count whose group counts fall in the same bin of
    32 share a tuning (disorder realisations of one model differ slightly)."""
    L = int(prob["len"])
    g = len(np.unique(S.xmask(prob["bits"]) >> np.uint64(min(11, L))))
    return f"L{L}-G{32 * round(g / 32)}-c64-m{krydim}-t"


def tune(problems, krydim=16, tol=1.2e-7, max_restarts=16, sample=None,
         force=False, log=None):
    """Set problems[i]['tile'] and ['team'] to the tuned pair; returns {key: record}."""
    import torch
    from . import BatchOTOC
    cache = {} if force else _load()
    by_key = {}
    for i, p in enumerate(problems):
        by_key.setdefault(shape_key(p, krydim), []).append(i)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = {}
    for key, idx in by_key.items():
        if key not in cache:
            L = int(problems[idx[0]]["len"])
            n = sample or min(len(idx), sms)
            timings = {}
            for B in range(8, min(12, L) + 1):
                for C in (1, 2, 4, 8, 16):
                    if C > (1 << (L - B)):
                        continue
                    probs = [dict(problems[j], tile=B, team=C) for j in idx[:n]]
                    b = BatchOTOC(probs, krydim=krydim, tol=tol, max_restarts=max_restarts)
                    b.probe(1)                                   # warm-up
                    timings[f"B{B}-C{C}"] = b.probe(2) / 1e3     # two H.psi per problem
                    b.close()
            best = min(timings, key=timings.get)
            B, C = (int(v[1:]) for v in best.split("-"))
            cache[key] = {"tile": B, "team": C, "seconds": timings, "sample": n,
                          "probe": "2 H.psi"}
            if log:
                log(f"autotune {key}: {timings} -> {best}")
        for j in idx:
            problems[j]["tile"] = int(cache[key]["tile"])
            problems[j]["team"] = int(cache[key]["team"])
        out[key] = cache[key]
    _save(cache)
    return out
