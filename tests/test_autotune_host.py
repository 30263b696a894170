"""Host side of the autotuner (no GPU): the flag encodings of the tuning
knobs, the candidate sets it times, and its cache file."""
from __future__ import annotations

import json

import pytest

from quantem.gpu_b200 import _lib, autotune


def test_flag_bits_do_not_overlap():
    assert _lib.flag_variant(3) == 3 << 8
    assert _lib.flag_chunks(5) == 5 << 16
    every = _lib.flag_variant(_lib.QSSB_FLAG_VARIANT_MAX) | _lib.flag_chunks(_lib.QSSB_FLAG_CHUNKS_MAX)
    low = _lib.QSSB_FLAG_CHI_FP64 | _lib.QSSB_FLAG_FULL_PLANE | _lib.QSSB_FLAG_QUADRATIC
    assert every & low == 0
    assert (_lib.flag_variant(15) & _lib.flag_chunks(1)) == 0
    for bad in (-1, 16):
        with pytest.raises(ValueError):
            _lib.flag_variant(bad)


def test_object_options_cover_tiles_only_on_the_quadratic_path():
    opts = autotune.object_options(128, 1781, quadratic=True)
    assert {v for _, v in opts} == {0, 1, 3}
    assert {c for c, _ in opts} == {64, 128, 192, 256}
    assert {v for _, v in autotune.object_options(128, 1781, quadratic=False)} == {0}
    # chunk counts never exceed the BF count
    assert max(c for c, _ in autotune.object_options(256, 20, True)) == 20


def test_loss_chunk_options_fill_whole_waves():
    opts = autotune.loss_chunk_options(1781, 64, 148)
    assert opts == sorted(set(opts)) and all(1 <= c <= 1781 for c in opts)
    # 148 SMs, 64 candidates: 2 chunks fill 128 CTAs (one wave with room), 3 spill over
    assert 2 in opts and 3 in opts


def test_cache_round_trips_through_its_file(tmp_path, monkeypatch):
    path = tmp_path / "tuning.json"
    monkeypatch.setenv("QSSB_TUNING_CACHE", str(path))
    monkeypatch.setattr(autotune, "_CACHE", None)
    autotune._store("gather:dev:128:128:16384:1781", 3)
    assert json.loads(path.read_text()) == {"gather:dev:128:128:16384:1781": 3}
    monkeypatch.setattr(autotune, "_CACHE", None)
    assert autotune._cache()["gather:dev:128:128:16384:1781"] == 3
