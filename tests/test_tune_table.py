"""The autotuner's JSON choice table (host logic, no GPU)."""
import json

import pytest

from mustard_b200 import tune_table


def test_missing_file_is_an_empty_table(tmp_path):
    t = tune_table.load(str(tmp_path / "none.json"))
    assert t == tune_table.empty()
    assert tune_table.lookup(t, "B200", 0, 512) is None


def test_record_lookup_missing_and_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    t = tune_table.empty()
    tune_table.record(t, "B200", 0, 512, 384, 128)
    tune_table.record(t, "B200", 2, 512, 512, 0)
    tune_table.record(t, "H100", 0, 512, 256, 64)
    assert tune_table.lookup(t, "B200", 0, 512) == (384, 128)
    assert tune_table.lookup(t, "B200", 2, 512) == (512, 0)
    assert tune_table.lookup(t, "B200", 1, 512) is None  # per precision
    assert tune_table.missing(t, "B200", 0, [512, 64, 512, 96]) == [1, 3]
    tune_table.save(t, path)
    again = tune_table.load(path)
    assert again == t
    assert json.load(open(path))["devices"]["B200"]["fp64"]["512"] == {"tile": 384, "nest": 128}
    assert [p.name for p in tmp_path.iterdir()] == ["tune.json"]  # no temporary file left


def test_wrong_version_is_rejected(tmp_path):
    path = tmp_path / "old.json"
    path.write_text(json.dumps({"version": 0, "devices": {}}))
    with pytest.raises(ValueError):
        tune_table.load(str(path))
