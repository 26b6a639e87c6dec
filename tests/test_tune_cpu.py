"""CPU checks of the float64 sweep's layout table and the autotuner's host logic (no GPU:
the library's layout entry points make no CUDA call)."""
import pytest

from adamixture_b200 import _lib, tune


def test_layout_counts():
    assert [tune.tiles(k) for k in range(1, 17)] == [2] * 8 + [1] * 8
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        tune.tiles(0)


def test_layout_table_set_get_and_limits():
    before = tune.get_tile(5, 3)
    try:
        tune.set_tile(5, 1, 3)
        assert tune.get_tile(5, 3) == 1
        assert tune.get_tile(5, 2) == 0          # per device
        tune.set_tile(5, 0, 3)
        assert tune.get_tile(5, 3) == 0
    finally:
        tune.set_tile(5, before, 3)
    for K, tile, dev in ((12, 1, 0), (4, 2, 0), (4, -1, 0), (17, 0, 0), (4, 0, 64), (4, 0, -1)):
        with pytest.raises(_lib.AdxError, match="invalid argument"):
            tune.set_tile(K, tile, dev)


def test_pick_prefers_the_default_on_a_tie():
    assert tune.pick({0: 10.0, 1: 7.0}) == 1
    assert tune.pick({0: 10.0, 1: 9.95}) == 0     # within 1 %
    assert tune.pick({0: 8.0, 1: 9.0}) == 0


def test_timed_blocks_cover_whole_waves():
    from adamixture_b200 import ops

    for M, N, K in ((500_000, 200_000, 8), (100_000, 20_000, 3), (10_000, 1_000, 3), (200, 300, 2)):
        spb, n_blocks, per_block = ops.em_sweep_blocks_info(M, N, K)
        nb = tune.timed_blocks(M, N, K, 148)
        assert 1 <= nb <= n_blocks
        assert nb == n_blocks or nb * per_block >= 4 * 2 * 148


def test_batch_groups_follow_the_table():
    before = {k: tune.get_tile(k, 1) for k in (2, 6, 10)}
    try:
        for k in (2, 6, 10):
            tune.set_tile(k, 0, 1)
        assert tune.batch_groups([2, 6, 10, 2], 1) == [[0, 1, 2, 3]]
        tune.set_tile(2, 1, 1)
        assert tune.batch_groups([2, 6, 10, 2], 1) == [[1, 2], [0, 3]]
    finally:
        for k, t in before.items():
            tune.set_tile(k, t, 1)


def test_autotune_switch(monkeypatch):
    monkeypatch.setenv("ADX_AUTOTUNE", "0")
    assert not tune.enabled()
    monkeypatch.setenv("ADX_AUTOTUNE", "1")
    assert tune.enabled()


def test_cache_file_round_trip(tmp_path, monkeypatch):
    f = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("ADX_TUNE_CACHE", str(f))
    monkeypatch.setattr(tune, "_CACHE", {"B200|M=10|N=20|K=3": {"tile": 1, "ms": {"0": 2.0, "1": 1.5}, "blocks": 4}})
    monkeypatch.setattr(tune, "_LOADED", True)
    tune._save_cache()
    assert f.exists()
    monkeypatch.setattr(tune, "_CACHE", {})
    monkeypatch.setattr(tune, "_LOADED", False)
    tune._load_cache()
    assert tune.choices() == {"B200|M=10|N=20|K=3": {"tile": 1, "ms": {"0": 2.0, "1": 1.5}, "blocks": 4}}


def test_unreadable_cache_file_is_ignored(tmp_path, monkeypatch):
    f = tmp_path / "tune.json"
    f.write_text("{not json")
    monkeypatch.setenv("ADX_TUNE_CACHE", str(f))
    monkeypatch.setattr(tune, "_CACHE", {})
    monkeypatch.setattr(tune, "_LOADED", False)
    tune._load_cache()
    assert tune.choices() == {}
