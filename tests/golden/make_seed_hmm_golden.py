"""Regenerate the golden fixture of HMM-profile queries' seeds from the reference's own code.

sketch.c's mp_sketch_hmm, map.c's mp_sketch_query with a profile and mp_map_coarse's
seeding steps, and hmm.c's parser (oracle/_ref/libseed_ref.so, `make -C oracle seedref`)
run on
  * emission tables regenerated from seeds (tests/test_seed_hmm.emission_table: Dirichlet
    profiles, ties, unreadable entries, flat rows) under several parameter sets: the
    profile-derived seeds in the reference's order (with a pos_loss that lets losses over
    32767 into the lists, which the reference keeps in 16 bits);
  * synthetic HMMER3 profiles (protlocus_b200.hmm.synthetic_profiles) read by the
    reference's parser: the query's merged seeds and its anchors on a seeded synthetic index
    (tests/oracle_lib.seed_index).
Per case the fixture keeps the generators' seeds, a SHA-256 of the regenerated input, the
number of outputs, their SHA-256 (little-endian uint64) and the first few, so it stays
small and still pins every value.  Written to tests/golden/seed_hmm_golden.json.

Usage: python tests/golden/make_seed_hmm_golden.py [out.json]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

# emission table (kind, n, seed) x (kmer, mod_bit, pos_loss, win_loss, max_per_win)
TABLES = [("dirichlet", 300, 901), ("ties", 120, 902), ("stars", 150, 903), ("flat", 40, 904), ("wide", 200, 905)]
TABLE_PARAMS = [(6, 1, 6, 8, 16), (5, 0, 6, 8, 16), (6, 2, 12, 20, 64), (4, 0, 100, 1000, 300),
                (6, 1, 40000, 40000, 16)]  # the last: losses over 32767 kept in 16 bits
# profiles (n, seed) x index (kmer 6, mod_bit 1, seed) x (pos_loss, win_loss, seed_max, max_occ)
PROFILES = (4, 911)
INDEX_SEED = 912
QUERY_PARAMS = [(6, 8, 16, 20000), (12, 20, 64, 40), (6, 8, 0, 20000)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def summary(a: np.ndarray) -> dict:
    return {"n": int(a.size), "sha256": sha(a), "head": [int(x) for x in a[:4]]}


def profile_texts():
    from protlocus_b200.hmm import synthetic_profiles
    texts, _ = synthetic_profiles(PROFILES[0], seed=PROFILES[1], m_min=40, m_max=250)
    return texts


def main(out: str):
    import oracle_lib as O
    from test_seed_hmm import emission_table
    if O.seed_ref_lib() is None:
        raise SystemExit("oracle/_ref/libseed_ref.so not built (make -C oracle seedref)")
    tables = []
    for kind, n, seed in TABLES:
        e = emission_table(np.random.default_rng(seed), n, kind)
        for kmer, mod_bit, pos_loss, win_loss, mx in TABLE_PARAMS:
            s = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=True)
            tables.append({"kind": kind, "n": n, "seed": seed, "digest": hashlib.sha256(e.tobytes()).hexdigest(),
                           "params": [kmer, mod_bit, pos_loss, win_loss, mx], "seeds": summary(s)})
    ki, kb = O.seed_index(np.random.default_rng(INDEX_SEED), kmer=6, mod_bit=1, n_block=200_000)
    queries = []
    with tempfile.TemporaryDirectory() as tmp:
        for q, text in enumerate(profile_texts()):
            path = os.path.join(tmp, f"p{q}.hmm")
            with open(path, "w") as f:
                f.write(text)
            for pos_loss, win_loss, mx, max_occ in QUERY_PARAMS:
                s = O.ref_hmm_query(path, 6, 1, pos_loss, win_loss, mx)
                a = O.ref_hmm_query(path, 6, 1, pos_loss, win_loss, mx, ki=ki, kb=kb, max_occ=max_occ)
                queries.append({"profile": q, "text_sha256": hashlib.sha256(text.encode()).hexdigest(),
                                "params": [pos_loss, win_loss, mx, max_occ], "seeds": summary(s),
                                "anchors": summary(a)})
    with open(out, "w") as f:
        json.dump({"source": "the reference's sketch.c / map.c / hmm.c (oracle/_ref/libseed_ref.so)",
                   "profiles": list(PROFILES), "index_seed": INDEX_SEED, "tables": tables, "queries": queries}, f,
                  indent=0)
    print(f"wrote {out}: {len(tables)} tables, {len(queries)} queries")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "seed_hmm_golden.json"))
