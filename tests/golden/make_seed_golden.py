"""Regenerate the golden fixture of the coarse mapper's seeding from the reference's own steps.

map.c's mp_sketch_query, mp_cal_max_occ, mp_collect_anchors and the anchor sort
(map.c:304-397, :565-572; sketch.c:18-37) are compiled from the reference's sources
by `make -C oracle seedref` into oracle/_ref/libseed_ref.so (a copy of map.c with
oracle/seed_ref_hook.c appended).  This script runs them on a seeded synthetic index
in the mapper's layout (tests/oracle_lib.seed_index) and seeded proteins
(tests/test_seed.seed_proteins) under several option sets, and writes, per case, the
options, the generators' seeds, a SHA-256 of the regenerated index and proteins, and
every protein's sorted anchors, to tests/golden/seed_golden.json.  The tests
regenerate the inputs from the seeds (and check the digests), so the fixture pins the
restatement (oracle/seed_port.c) and the device seeding on machines without the
reference tree.

Cases: the default cap (max_occ 20000), a low cap, no sampling (mod_bit 0), and the
accuracy mode's repeat rescue with a budget that scales the shares and hands out the
rest from the query names' hashes, on an index with 5 % repeat buckets.

Usage: python tests/golden/make_seed_golden.py [out.json]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

CASES = [
    # name, index (kmer, mod_bit, mean_occ, hot, hot_occ, seed), proteins (n, seed), max_occ, repeat_cap, budget
    ("default", (5, 1, 2.0, 64, 2000, 601), (10, 611), 20000, 0, 0),
    ("low_cap", (5, 1, 2.0, 64, 2000, 602), (10, 612), 6, 0, 0),
    ("no_sampling", (5, 0, 1.0, 64, 2000, 603), (8, 613), 200, 0, 0),
    ("rescue_round_robin", (5, 1, 2.0, 1 << 15, 300, 604), (10, 614), 20, 5, 7),
    ("rescue_scaled", (5, 1, 2.0, 1 << 15, 300, 605), (10, 615), 20, 64, 300),
]


def case_inputs(index, prots):
    import oracle_lib as O
    from test_seed import seed_proteins
    kmer, mod_bit, mean_occ, hot, hot_occ, iseed = index
    ki, kb = O.seed_index(np.random.default_rng(iseed), kmer=kmer, mod_bit=mod_bit, mean_occ=mean_occ,
                          n_block=50_000, hot=hot, hot_occ=hot_occ)
    n, pseed = prots
    ps = [p[:160] for p in seed_proteins(np.random.default_rng(pseed), n)]
    names = [b"q%d" % q for q in range(n)]
    return ki, kb, ps, names


def digest(ki, kb, ps) -> str:
    h = hashlib.sha256()
    h.update(ki.tobytes())
    h.update(kb.tobytes())
    for p in ps:
        h.update(p)
        h.update(b"|")
    return h.hexdigest()


def main(out: str):
    import oracle_lib as O
    if O.seed_ref_lib() is None:
        raise SystemExit("oracle/_ref/libseed_ref.so not built (make -C oracle seedref)")
    cases = []
    for name, index, prots, max_occ, cap, budget in CASES:
        ki, kb, ps, names = case_inputs(index, prots)
        anchors = []
        for p, nm in zip(ps, names):
            if cap > 0:
                a = O.seed_anchors_acc(ki, kb, index[0], index[1], max_occ, cap, budget, nm, p, use_ref=True)
            else:
                a = O.seed_anchors(ki, kb, index[0], index[1], max_occ, p, use_ref=True)
            anchors.append([int(x) for x in a])
        cases.append({"name": name, "index": list(index), "proteins": list(prots), "max_occ": max_occ,
                      "repeat_cap": cap, "budget": budget, "digest": digest(ki, kb, ps), "anchors": anchors})
    with open(out, "w") as f:
        json.dump({"source": "the reference's map.c seeding steps (oracle/_ref/libseed_ref.so)", "cases": cases}, f)
    print(f"wrote {out}: {len(cases)} cases, {sum(len(a) for c in cases for a in c['anchors'])} anchors")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "seed_golden.json"))
