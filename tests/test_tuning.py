"""The per-shape-class tuning file of the batched global DP (CPU only)."""
import json

import numpy as np

from protlocus_b200 import tuning as T


def test_shape_class_buckets():
    assert T.shape_class([20000, 30000, 25000], [300, 400, 350]) == "al256_nl32768_n4"  # nearest powers of two
    assert T.shape_class([], []) == "empty"
    # similar batches share a class, different lengths do not
    a = T.shape_class(np.full(8192, 24000), np.full(8192, 350))
    b = T.shape_class(np.full(8000, 26000), np.full(8000, 330))
    c = T.shape_class(np.full(8192, 2000), np.full(8192, 350))
    assert a == b != c


def test_round_trip(tmp_path):
    p = tmp_path / "sub" / "tuning.json"
    f = T.TuningFile(str(p))
    assert f.get("al256_nl16384_n8192") is None
    f.put("al256_nl16384_n8192", 1536, 0.5, device="test")
    f.save()
    g = T.TuningFile(str(p))
    assert g.get("al256_nl16384_n8192") == {"r4_rows": 1536, "coop_ratio": 0.5}
    data = json.loads(p.read_text())
    assert data["version"] == 1 and data["classes"]["al256_nl16384_n8192"]["device"] == "test"


def test_unreadable_file_is_empty(tmp_path):
    p = tmp_path / "tuning.json"
    p.write_text("{not json")
    assert T.TuningFile(str(p)).classes == {}
