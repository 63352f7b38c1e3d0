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


SMALL = dict(N=28, k=8, dtype="c64", workload="sparse SYK N=28 (14 qubits), k=8")


def test_port_sample_computes_the_apply_it_times(monkeypatch):
    """Where the reference build is absent the CPU baseline times the
    oracle's port on a row sample; the rows it computes are those of the
    full oracle apply, and the rate is extrapolated from the sample."""
    from oracle import oracle as O
    monkeypatch.setattr(O, "ref_available", lambda: False)
    bits, coeff = bench.make_terms(SMALL, seed=3)
    state = bench.port_state(SMALL)
    assert state.dtype == np.complex64 and state.size == 1 << 14
    cb = bench.cpu_sample(SMALL, bits, coeff, 1e9, 1 << 18, state)
    assert cb["kind"] == "port" and cb["threads"] == 1
    assert cb["rows"] == 1 << 14             # the whole state when it is smaller
    assert cb["value"] == 1e9 * 1.0 / cb["seconds"] / 1e9
    idx = np.arange(100, dtype=np.uint64)
    full = O.apply(14, bits, coeff, state.astype(np.complex128))
    part = O.apply_at(bits, coeff, idx, lambda j: state[j])
    np.testing.assert_allclose(part, full[:100], rtol=1e-12, atol=1e-12)


def test_reference_arm_falls_back_to_the_port(monkeypatch, capsys):
    import json
    from oracle import oracle as O
    monkeypatch.setattr(O, "ref_available", lambda: False)
    monkeypatch.setitem(bench.CONFIGS, "small", SMALL)
    monkeypatch.delenv("RANK", raising=False)
    args = bench.argparse.Namespace(config="small", steps=2, warmup=1)
    bench.run_reference(args)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" not in line
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 == line["e2e"]["d2h_bytes_per_step"]
    assert line["config"]["value_is"] == "extrapolated from a row sample"


def test_compulsory_bytes_of_a_state_smaller_than_one_tile():
    """Below one tile (2^12 complex64 elements) the window is the one tile:
    G_w counts distinct x >> 12 and the formula stays (G_w + 1) * D * 8."""
    bits, _ = S.sparse_syk(20, k=8, seed=3)
    gw = len(np.unique(S.xmask(bits) >> np.uint64(12)))
    assert bench.alg_bytes_host(10, bits, "c64") == (gw + 1) * (1 << 10) * 8
