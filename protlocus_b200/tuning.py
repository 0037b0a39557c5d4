"""Tuning of the batched global DP per shape class, kept in a JSON file.

pl_engine_autotune picks, for one batch, the rows-per-lane bin boundary (jobs with
at most r4_rows DP rows take 4 rows per lane, the rest 8) and the cooperative-job
ratio (a job takes a whole CTA when it holds more than coop_ratio times a warp's
share of its wave's cells).  The best point depends on the batch's shape: the
protein lengths, the window lengths and the number of jobs.  A shape class puts
batches of similar shape together (log2 buckets of the median protein length,
of the median window length and of the job count), and the JSON file maps each
class to the point the autotuner chose, so a later batch of that class is tuned
without a search:

    {"version": 1, "classes": {"al256_nl16384_n8192": {"r4_rows": 0, "coop_ratio": 0.7,
                                                      "jobs": 8192, "device": "NVIDIA B200"}}}

The file is read and written whole; writers replace it atomically.
"""
from __future__ import annotations

import json
import math
import os
import tempfile

import numpy as np

DEFAULT_PATH = os.path.join(os.path.expanduser("~"), ".cache", "protlocus_b200", "tuning.json")


def _bucket(x: float) -> int:
    return 1 << max(0, int(round(math.log2(max(float(x), 1.0)))))


def shape_class(nl, al) -> str:
    """Class key of a batch from its window lengths nl and protein lengths al."""
    nl = np.asarray(nl, dtype=np.int64)
    al = np.asarray(al, dtype=np.int64)
    if nl.size == 0:
        return "empty"
    return f"al{_bucket(np.median(al))}_nl{_bucket(np.median(nl))}_n{_bucket(nl.size)}"


class TuningFile:
    """The JSON map from shape class to tuning point."""

    def __init__(self, path: str | None = None):
        self.path = path or os.environ.get("PLGPU_TUNING_JSON") or DEFAULT_PATH
        self.classes = {}
        try:
            with open(self.path) as f:
                data = json.load(f)
            if data.get("version") == 1:
                self.classes = dict(data.get("classes", {}))
        except (OSError, ValueError):
            pass

    def get(self, key: str):
        v = self.classes.get(key)
        if not v or "r4_rows" not in v or "coop_ratio" not in v:
            return None
        return {"r4_rows": int(v["r4_rows"]), "coop_ratio": float(v["coop_ratio"])}

    def put(self, key: str, r4_rows: int, coop_ratio: float, **extra):
        self.classes[key] = {"r4_rows": int(r4_rows), "coop_ratio": float(coop_ratio), **extra}

    def save(self):
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(prefix=".tuning.", dir=d or ".")
        with os.fdopen(fd, "w") as f:
            json.dump({"version": 1, "classes": self.classes}, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)
