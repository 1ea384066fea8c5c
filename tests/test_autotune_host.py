"""Host logic of the autotuner's batched geometry stage: the per-length
device times it reads from the timeline the library prints."""
from __future__ import annotations

import json

from piculator_b200 import autotune


def _lines(marks):
    return "\n".join(json.dumps(m) for m in marks)


def test_timeline_ms_by_k_takes_the_last_computation():
    first = [{"timeline": "bsr_level_ntt", "k": 14, "ms": 99.0}, {"timeline_alloc": {"calls": 1}}]
    second = [
        {"timeline": "bsr_level_school", "ms": 5.0},
        {"timeline": "bsr_level_ntt", "k": 14, "ms": 10.0},
        {"timeline": "bsr_level_ntt", "k": 15, "ms": 20.0},
        {"timeline": "top_merge_chunk", "k": 15, "ms": 7.5},
        {"timeline": "pi_phase", "ms": 3.0},
        {"timeline_alloc": {"calls": 2}},
    ]
    text = "noise\n" + _lines(first) + "\n" + _lines(second) + "\n"
    assert autotune._timeline_ms_by_k(text) == {14: 10.0, 15: 27.5}


def test_timeline_ms_by_k_empty():
    assert autotune._timeline_ms_by_k("") == {}


def test_committed_tuning_table_is_well_formed():
    """The table init() applies: every NTT length 2^10..2^27 with a geometry
    the library accepts (row bits 8..13, column width 0..6, radix 2..4) and
    the product and binary-splitting thresholds."""
    import os

    import piculator_b200 as P
    assert os.path.exists(P.TUNING_FILE)
    with open(P.TUNING_FILE) as f:
        t = json.load(f)
    for k in range(10, 28):
        g = t["ntt"][str(k)]
        assert 8 <= g["row_bits"] <= 13
        assert 0 <= g["col_width_log2"] <= 6
        assert 2 <= g["radix_log2"] <= 4
    assert t["products"]["school_max_words"] >= 0
    assert t["products"]["fft_max_words"] >= 0
    assert t["bsr"]["bsr_school_max_words"] > 0


def test_table_write_replaces_the_file_whole(tmp_path):
    """The tuner writes its table beside the destination and renames it over
    it: the old table stays until the new one is complete, and no temporary
    file is left behind."""
    from piculator_b200 import autotune
    out = tmp_path / "tuning.json"
    out.write_text('{"old": 1}')
    autotune._write_table(str(out), {"ntt": {"20": {"row_bits": 11}}})
    assert autotune._read_table(str(out)) == {"ntt": {"20": {"row_bits": 11}}}
    assert sorted(p.name for p in tmp_path.iterdir()) == ["tuning.json"]


def test_table_write_failure_keeps_the_old_table(tmp_path):
    from piculator_b200 import autotune
    out = tmp_path / "tuning.json"
    out.write_text('{"old": 1}')
    import pytest
    with pytest.raises(TypeError):
        autotune._write_table(str(out), {"bad": object()})  # not serialisable
    assert autotune._read_table(str(out)) == {"old": 1}
