"""The autotuner's host logic on the CPU: the candidate set per qubit count
and the shape key that groups disorder realisations of one model."""
import numpy as np

from reapers_b200 import autotune as AT
from reapers_b200 import syk as S


def test_candidates_cover_every_tile_loop_below_2_14():
    for L in (8, 10, 12, 13):
        c = AT.candidates(L)
        tiles = sorted({B for B, _ in c})
        assert tiles == list(range(8, min(12, L) + 1))
        # a team never has more CTAs than the problem has tiles
        assert all(C <= (1 << (L - B)) for B, C in c)


def test_candidates_from_2_14_use_row_tiles():
    assert AT.candidates(14) == [(12, 1), (12, 2), (12, 4)]
    assert AT.candidates(15) == [(12, 1), (12, 2), (12, 4), (12, 8)]
    for L in (16, 18, 20, 24):
        assert AT.candidates(L) == [(12, 2), (12, 4), (12, 8)]


def test_shape_key_groups_realisations_by_size_and_group_count():
    keys = set()
    for seed in range(6):
        bits, _ = S.sparse_syk(40, k=8, seed=seed)
        keys.add(AT.shape_key({"len": 20, "bits": bits}, 16))
    assert all(k.startswith("L20-G") and k.endswith("-c64-m16-p") for k in keys)
    assert len(keys) <= 2          # bins of 32 source-tile groups
    bits, _ = S.sparse_syk(32, k=8, seed=0)
    assert AT.shape_key({"len": 16, "bits": bits}, 16).startswith("L16-")
    g = len(np.unique(S.xmask(bits) >> np.uint64(11)))
    assert AT.shape_key({"len": 16, "bits": bits}, 12) == f"L16-G{32 * round(g / 32)}-c64-m12-p"


def test_cache_round_trip_and_unwritable_location(tmp_path, monkeypatch):
    monkeypatch.setenv("RPB200_TUNE_CACHE", str(tmp_path / "sub" / "tune.json"))
    rec = {"L20-G64-c64-m16-p": {"path": "batched", "tile": 12, "team": 2}}
    assert AT._save(rec)
    assert AT._load() == rec
    # a path under a regular file cannot be created: the save reports it and
    # the load falls back to an empty cache instead of raising
    blocker = tmp_path / "file"
    blocker.write_text("x")
    monkeypatch.setenv("RPB200_TUNE_CACHE", str(blocker / "tune.json"))
    assert AT._save(rec) is False
    assert AT._load() == {}
