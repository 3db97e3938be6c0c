"""CPU checks of the autotuner's bookkeeping (no kernel runs here)."""
import json

import numpy as np

from quantom_loits_b200 import tuning


def test_shape_key_buckets_by_powers_of_two():
    k = tuning.shape_key(np.array([0, 100, 1100]), np.array([1000, 3000]), False)
    assert k == "d1-g10-n12-all"
    assert tuning.shape_key(np.array([0, 1024]), np.array([4096]), True) == "d0-g10-n12-cut"
    # same bucket for a slightly different batch
    assert tuning.shape_key(np.array([0, 90, 1000]), np.array([1500, 2500]), False) == k


def test_candidates_are_valid_geometries():
    for threads, blocks, scan in tuning.CANDIDATES:
        assert threads in (256, 512, 1024)
        assert blocks in (2, 4, 8, 16)
        assert 1 <= scan <= 64


def test_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "t.json"
    path.write_text(json.dumps({"d1-g10-n12-all": {"threads": 512, "blocks_per_item": 8,
                                                   "scan_knots": 8}}))
    monkeypatch.setenv("LOITS_TUNE_CACHE", str(path))
    t = tuning.Autotuner("cpu")
    assert t.table["d1-g10-n12-all"]["threads"] == 512
    t.table["x"] = {"threads": 256, "blocks_per_item": 16, "scan_knots": 8}
    t._save()
    assert json.loads(path.read_text())["x"]["threads"] == 256
