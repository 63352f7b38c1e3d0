"""bench.py's host-side figures on the CPU: the compulsory DRAM bytes the
`value` metric divides by, for the two configured workloads (the reference
arm computes its value with the same function)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import reapers_b200.syk as S  # noqa: E402


def test_compulsory_bytes_of_the_n56_workload():
    """(G_w + 1) * 2^28 * 8 with G_w = 42 distinct x >> 20 (tiles of 2^12
    complex64 elements, a window of 296 tiles): 92.34 GB per apply."""
    bits, _ = S.sparse_syk(56, k=8, seed=1000)
    b = bench.alg_bytes_host(28, bits, "c64")
    gw = len(np.unique(S.xmask(bits) >> np.uint64(20)))
    assert gw == 42
    assert b == (gw + 1) * (1 << 28) * 8
    assert abs(b - 92.34e9) < 0.01e9


def test_compulsory_bytes_window_follows_the_tile_count():
    """complex128 rows hold 8 elements (tiles of 2^11); the window is
    min(tiles, 2 x SMs) CTAs and its log2 rounds down."""
    bits, _ = S.sparse_syk(48, k=8, seed=2000)
    b = bench.alg_bytes_host(24, bits, "c128")
    # 2^13 tiles, window 296 -> 8 bits: x >> (11 + 8)
    gw = len(np.unique(S.xmask(bits) >> np.uint64(19)))
    assert b == (gw + 1) * (1 << 24) * 16
    # a state of fewer tiles than the window: the window is the state
    small = bench.alg_bytes_host(19, bits & np.uint64((1 << 38) - 1), "c64", sms=148)
    gw_small = len(np.unique(S.xmask(bits & np.uint64((1 << 38) - 1)) >> np.uint64(12 + 7)))
    assert small == (gw_small + 1) * (1 << 19) * 8
