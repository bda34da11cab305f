"""The tuning table's reader (no device needed): entries counted, malformed lines refused, and the
tuner's merge keeps other GPUs' and sizes' entries."""
import json

import pytest

from totem_b200 import capi, tune


def test_load_tuning_counts_entries_and_rejects_bad_lines(tmp_path):
    good = tmp_path / "t.jsonl"
    good.write_text('{"device": "NVIDIA B200", "n": 512, "row_variant": 5, "col_variant": 1, "batch_mib": 4096}\n'
                    '\n{"device": "Other GPU", "n": 1024, "row_variant": 4, "col_variant": 5, "batch_mib": 2048.5}\n')
    try:
        assert capi.load_tuning(str(good)) == 2
        bad = tmp_path / "bad.jsonl"
        bad.write_text('{"n": 512, "row_variant": 5}\n')
        with pytest.raises(capi.TotemError) as e:
            capi.load_tuning(str(bad))
        assert e.value.code == capi.ERR_INVALID_ARG and "device" in str(e.value)
        with pytest.raises(capi.TotemError):
            capi.load_tuning(str(tmp_path / "missing.jsonl"))
        assert capi.load_tuning(None) == 0
    finally:
        capi.load_tuning(capi.TUNING_FILE)


def test_committed_table_parses():
    n = capi.load_tuning(capi.TUNING_FILE)
    rows = [json.loads(line) for line in open(capi.TUNING_FILE) if line.strip()]
    assert n == len(rows) > 0
    for r in rows:
        assert r["row_variant"] in (1, 3, 4, 5) and r["col_variant"] in (1, 2, 3, 5, 6) and r["batch_mib"] > 0
        assert r["us_per_probe_slice"] <= r["default_us_per_probe_slice"] * 1.0001


def test_merge_keeps_other_entries(tmp_path):
    path = tmp_path / "t.jsonl"
    path.write_text(json.dumps({"device": "A", "n": 512, "row_variant": 1}) + "\n" +
                    json.dumps({"device": "B", "n": 512, "row_variant": 4}) + "\n")
    tune.merge(str(path), "A", [{"n": 512, "row_variant": 5, "col_variant": 2, "batch_mib": 1024},
                                {"n": 1024, "row_variant": 3, "col_variant": 1, "batch_mib": 4096}])
    rows = [json.loads(line) for line in open(path)]
    assert [(r["device"], r["n"], r["row_variant"]) for r in rows] == [("A", 512, 5), ("A", 1024, 3), ("B", 512, 4)]


def test_candidate_sets():
    assert tune.col_variants(1024) == [1, 2, 3, 5]
    assert tune.row_variants(512) == [1, 4, 5] and tune.row_variants(2048) == [1, 3, 4]
