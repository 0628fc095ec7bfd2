"""The autotuner's host logic (no GPU): candidate sets, cache entries with
and without an algorithm, and the size buckets."""
import json

from winding_b200 import _lib, autotune


class _Cloud:
    def __init__(self, count):
        self.count = count


def test_one_cta_candidates_only_for_small_jobs():
    small = [(_Cloud(100), None), (_Cloud(_lib.ONE_CTA_MAX), None)]
    big = small + [(_Cloud(_lib.ONE_CTA_MAX + 1), None)]
    algos = {c[3] for c in autotune.candidates_for(small)}
    assert algos == {_lib.ALGO_PHASES, _lib.ALGO_ONE_RADIX, _lib.ALGO_ONE_COUNT}
    assert {c[3] for c in autotune.candidates_for(big)} == {_lib.ALGO_PHASES}
    assert {c[3] for c in autotune.candidates_for([])} == {_lib.ALGO_PHASES}


def test_cache_entries_old_and_new():
    assert autotune._full((2048, 1, 1)) == (2048, 1, 1, _lib.ALGO_PHASES)
    assert autotune._full([2048, 1, 1, 2]) == (2048, 1, 1, 2)
    assert autotune._valid([2048, 1, 1]) and autotune._valid([2048, 1, 1, 1])
    assert not autotune._valid([0, 1, 1]) and not autotune._valid([2048, 1]) and not autotune._valid("x")


def test_load_reads_both_entry_forms(tmp_path, monkeypatch):
    installed = {}
    monkeypatch.setattr(autotune, "install", lambda ctx, table: installed.update(table))
    monkeypatch.setattr(autotune, "gpu_name", lambda device=0: "gpu")

    class Ctx:
        device = 0

    path = tmp_path / "tuning.json"
    path.write_text(json.dumps({"gpu": {"13": [2048, 1, 1, 2], "20": [8192, 1, 1], "7": [0, 1, 1]}}))
    table = autotune.load(Ctx(), str(path))
    assert table == {13: (2048, 1, 1, 2), 20: (8192, 1, 1, 0)}
    assert installed == table


def test_buckets():
    assert autotune.bucket(1) == 0 and autotune.bucket(16384) == 14 and autotune.bucket(16385) == 14
    assert autotune.bucket(25_000_000) == 24
