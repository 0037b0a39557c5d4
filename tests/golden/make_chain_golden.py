"""Regenerate the golden fixture of anchor chaining from the reference's own mp_chain.

mp_chain (chain.c:160) is compiled from the reference's sources by `make -C oracle
extra` into oracle/_ref/libchain_ref.so (behind oracle/ref_chain.c).  This script
runs it on seeded synthetic queries (protlocus_b200.workload.chain_anchors) under
several argument sets and writes, per case, the arguments, the generator's seed and
parameters, a SHA-256 of the regenerated anchors, and the chain words u[] and the
chained anchors a[] mp_chain returns, to tests/golden/chain_golden.json.  The tests
regenerate the anchors from the seeds (and check the digests), so the fixture pins
the restatement (tests/chain_ref.py), the library's host half and the device DP on
machines without the reference tree.

Cases: the coarse mapping's main-chain and pre-chain arguments, nucleotide
coordinates (bbit 0, kmer 5), tight max_iter / max_skip, and two random argument
sets (non-spliced penalties, min_sc, min_cnt).

Usage: python tests/golden/make_chain_golden.py [out.json]
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

from protlocus_b200 import workload as W  # noqa: E402
from protlocus_b200.abi import chain_opt  # noqa: E402

CASES = [
    ("main", chain_opt("main"), dict(n_q=12, seed=501, al_median=200.0)),
    ("pre", chain_opt("pre"), dict(n_q=12, seed=502, al_median=200.0)),
    ("nucleotide", chain_opt("main", max_intron=5000, bbit=0, kmer=5),
     dict(n_q=10, seed=503, genome_len=2_000_000, bbit=0, al_median=150.0)),
    ("tight", dict(chain_opt("main"), max_iter=5, max_skip=2), dict(n_q=10, seed=504, hit_rate=0.5, al_median=150.0)),
    ("random_a", dict(max_dist_x=9000, max_dist_y=400, bw=7000, max_skip=6, max_iter=300, min_cnt=2, min_sc=15,
                      coef=0.5, is_spliced=0, kmer=5, bbit=4), dict(n_q=10, seed=505, al_median=180.0)),
    ("random_b", dict(max_dist_x=30000, max_dist_y=1500, bw=20000, max_skip=40, max_iter=4000, min_cnt=4, min_sc=0,
                      coef=1.2, is_spliced=1, kmer=7, bbit=8), dict(n_q=10, seed=506, al_median=250.0)),
]


def case_queries(gen: dict):
    g = dict(gen)
    n_q, seed = g.pop("n_q"), g.pop("seed")
    return W.chain_anchors(n_q, seed=seed, **g)


def digest(queries) -> str:
    h = hashlib.sha256()
    for q in queries:
        h.update(np.asarray(q, np.uint64).tobytes())
        h.update(b"|")
    return h.hexdigest()


def main(out: str):
    import oracle_lib as O
    if O.chain_lib() is None:
        raise SystemExit("oracle/_ref/libchain_ref.so is not built (make -C oracle extra)")
    cases = []
    for name, opt, gen in CASES:
        qs = case_queries(gen)
        res = []
        for a in qs:
            u, a_out = O.ref_chain(opt, a)
            res.append({"u": [int(x) for x in u], "a": [int(x) for x in a_out]})
        cases.append({"name": name, "opt": opt, "gen": gen, "sha256": digest(qs), "chains": res})
    with open(out, "w") as f:
        json.dump({"generator": "tests/golden/make_chain_golden.py", "cases": cases}, f, separators=(",", ":"))
    print(f"wrote {out}: {len(cases)} cases, {sum(len(c['chains']) for c in cases)} queries")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "chain_golden.json"))
