"""The seeds of HMM-profile queries, restated (oracle/seed_port.c: sp_sketch_hmm,
sp_seeds_hmm_query, sp_anchors_hmm) against the reference's own functions
(oracle/_ref/libseed_ref.so: sketch.c's mp_sketch_hmm, map.c's mp_sketch_query with a
profile, hmm.c's parser and mp_map_coarse's seeding steps).

mp_sketch_hmm (sketch.c:40-118): for every window of kmer match states, the 13-letter
k-mers whose summed emission loss against each state's best group stays within
win_loss, each state offering at most four groups within pos_loss of its best, the
first max_per_win of them in the enumeration order; a seed where the k-mer's hash
passes the sampling.  mp_sketch_query (map.c:332-343) merges them with the consensus's
own seeds, sorts and removes duplicates.

Emission tables: Dirichlet profiles in the parser's units (2 ln p, the best residue at
+4), ties (small integers: many groups at equal loss), unreadable entries (INT16_MIN,
whole rows of them) and flat rows (every group at loss 0, so the window budget and
max_per_win cut the enumeration)."""
import numpy as np
import pytest

import oracle_lib as O

need_ref = pytest.mark.skipif(O.seed_ref_lib() is None, reason="oracle/_ref/libseed_ref.so not built")

BG = np.array([0.0787945, 0.0151600, 0.0535222, 0.0668298, 0.0397062, 0.0695071, 0.0229198, 0.0590092, 0.0594422,
               0.0963728, 0.0237718, 0.0414386, 0.0482904, 0.0395639, 0.0540978, 0.0683364, 0.0540687, 0.0673417,
               0.0114135, 0.0304133])

# kmer, mod_bit, pos_loss, win_loss, max_per_win: the coarse stage's defaults (options.c:112-114,
# kmer 6, mod_bit 1), the refine stage's (kmer2 5, mod_bit 0), wider budgets, consensus-like
# budgets, one k-mer per window, none, and very short and very long k-mers
PARAMS = [(6, 1, 6, 8, 16), (5, 0, 6, 8, 16), (7, 1, 6, 8, 16), (6, 2, 12, 20, 64), (6, 1, 0, 0, 16),
          (6, 1, 6, 8, 1), (6, 1, 6, 8, 0), (1, 0, 6, 8, 16), (4, 0, 100, 1000, 300)]


# budgets past 16 bits: a state's losses over 32767 are kept wrapped to 16 bits, as the
# reference's alt_loss keeps them; window budgets at the int32 limits and below 0
WIDE_PARAMS = [(6, 1, 40000, 40000, 16), (6, 1, 70000, 2 ** 31 - 1, 16), (5, 0, 100000, -5, 16),
               (6, 1, 32767, 65534, 16), (4, 0, 65535, 0, 300), (3, 0, 2 ** 31 - 1, -(2 ** 31), 64)]


def emission_table(rng, n: int, kind: str) -> np.ndarray:
    """n match states x 20 columns of int16 emissions of the given kind."""
    if kind == "dirichlet":
        p = rng.dirichlet(BG * 20.0, size=n)
        v = np.rint(2.0 * np.log(np.maximum(p, 1e-300))).clip(-32767, 32767).astype(np.int64)
        e = v - v.max(axis=1, keepdims=True) + 4
    elif kind == "ties":
        e = rng.integers(-3, 5, size=(n, 20))
    elif kind == "stars":
        e = rng.integers(-12, 5, size=(n, 20))
        e[rng.random((n, 20)) < 0.3] = -32768
        if n:
            e[rng.integers(0, n, size=max(1, n // 10))] = -32768  # rows the parser read as all '*'
    elif kind == "wide":  # one to three columns high, the rest far below: losses over 32767 kept
        e = rng.integers(-32767, 0, size=(n, 20))
        for i in range(n):
            e[i, rng.choice(20, size=int(rng.integers(1, 4)), replace=False)] = rng.integers(20000, 32768)
        e[rng.random((n, 20)) < 0.05] = -32768
    elif kind == "flat":
        e = np.full((n, 20), 4)
        if n > 4:
            e[n // 2] = rng.integers(-40, 5, size=20)
    else:
        raise ValueError(kind)
    return ((e + 32768) % 65536 - 32768).astype(np.int16)  # int16 as the parser stores them


@need_ref
@pytest.mark.parametrize("kind", ["dirichlet", "ties", "stars", "flat"])
def test_sketch_hmm_port_equals_reference(kind):
    """The profile-derived seeds, in the reference's order (window by window, each window's
    k-mers in its enumeration order), for every parameter set and for tables shorter than,
    as long as, and much longer than a window."""
    rng = np.random.default_rng({"dirichlet": 11, "ties": 12, "stars": 13, "flat": 14}[kind])
    total = 0
    for kmer, mod_bit, pos_loss, win_loss, mx in PARAMS:
        for n in sorted({0, 1, kmer - 1, kmer, 37, 400}):
            e = emission_table(rng, n, kind)
            ref = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=True)
            port = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=False)
            assert np.array_equal(ref, port), (kind, kmer, mod_bit, pos_loss, win_loss, mx, n, ref.size, port.size)
            total += ref.size
    assert total > 0


def test_sketch_hmm_hand_case():
    """One flat state (every group at loss 0) repeated: each window offers the four lowest
    groups 0, 1, 2, 3 per position, and with mod_bit 0 and no loss budget beyond 0 the first
    max_per_win k-mers are the lexicographic ones 0000, 0001, 0002, ... (kmer 4)."""
    e = np.full((4, 20), 4, np.int16)
    seeds = O.sketch_hmm(e, 4, 0, 0, 0, 6, use_ref=False)
    assert seeds.size == 6 and np.all((seeds & 0xFFFFFFFF) == 3)
    mask = (1 << 16) - 1

    def h(x):  # sketch.c:7-16
        x = (x + ~(x << 15)) & mask
        x ^= x >> 10
        x = (x + (x << 3)) & mask
        x ^= x >> 6
        x = (x + ~(x << 11)) & mask
        x ^= x >> 16
        return x
    want = [h(c0 << 12 | c1 << 8 | c2 << 4 | c3) for c0, c1, c2, c3 in
            [(0, 0, 0, 0), (0, 0, 0, 1), (0, 0, 0, 2), (0, 0, 0, 3), (0, 0, 1, 0), (0, 0, 1, 1)]]
    assert [int(s) >> 32 for s in seeds] == want
    # state 2 with groups 0-3 (A; S T; R K; H) one below the best: its four closest groups are
    # then 4-7 (N D; Q E; C; P) at loss 0, so the first k-mer is 0 0 4 0
    e[2, [0, 15, 16, 14, 8, 6]] = 3
    first = O.sketch_hmm(e, 4, 0, 1, 0, 1, use_ref=False)
    assert [int(s) >> 32 for s in first] == [h(0 << 12 | 0 << 8 | 4 << 4 | 0)]
    # every window then has 4^4 k-mers at loss 0, so max_per_win (64) ends each window
    assert O.sketch_hmm(e, 4, 0, 1, 1, 64, use_ref=False).size == 64
    # no windows: shorter than kmer, or max_per_win 0
    assert O.sketch_hmm(e[:3], 4, 0, 6, 8, 16, use_ref=False).size == 0
    assert O.sketch_hmm(e, 4, 0, 6, 8, 0, use_ref=False).size == 0


def _profiles(tmp_path, n, seed):
    from protlocus_b200.hmm import synthetic_profiles
    texts, _ = synthetic_profiles(n, seed=seed, m_min=20, m_max=300)
    paths = []
    for q, t in enumerate(texts):
        if q % 3 == 2:  # some emissions the file gives as '*' (probability 0)
            lines = t.split("\n")
            for k, line in enumerate(lines):
                tok = line.split()
                if len(tok) == 25 and tok[0].isdigit() and int(tok[0]) % 7 == 0:  # index, 20 emissions, 4 more
                    tok[1 + int(tok[0]) % 20] = "*"
                    lines[k] = "{:>7} ".format(tok[0]) + " ".join(tok[1:])
            t = "\n".join(lines)
            assert " * " in t
        p = tmp_path / f"p{q}.hmm"
        p.write_text(t)
        paths.append(str(p))
    return paths


@need_ref
def test_hmm_query_seeds_equal_reference(tmp_path):
    """A profile file through the reference's parser and mp_sketch_query (consensus seeds
    plus the profile-derived ones, sorted, duplicates removed) against the restatement on
    the parser's consensus and emissions; the consensus is the first best column per state."""
    from protlocus_b200.hmm import parse_hmmer3
    for path in _profiles(tmp_path, 9, 41):
        cons, emit = O.ref_hmm_tables(path)
        ours = parse_hmmer3(open(path).read())[0]["emit"]
        assert np.array_equal(emit, ours)
        assert cons == O.hmm_consensus(emit)
        for kmer, mod_bit, pos_loss, win_loss, mx in PARAMS:
            ref = O.ref_hmm_query(path, kmer, mod_bit, pos_loss, win_loss, mx)
            port = O.seeds_hmm_query(cons, emit, kmer, mod_bit, pos_loss, win_loss, mx)
            assert np.array_equal(ref, port), (path, kmer, mod_bit, mx, ref.size, port.size)
            assert np.all(port[1:] > port[:-1])  # sorted, no duplicates


@need_ref
@pytest.mark.parametrize("max_occ", [20000, 40])
def test_hmm_query_anchors_equal_reference(tmp_path, max_occ):
    """mp_map_coarse's seeding of an HMM-profile query (the merged seeds, the occurrence cap
    over them and the collected anchors, sorted) on a synthetic index."""
    rng = np.random.default_rng(77 + max_occ)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=200_000)
    for path in _profiles(tmp_path, 6, 43 + max_occ):
        cons, emit = O.ref_hmm_tables(path)
        for pos_loss, win_loss, mx in [(6, 8, 16), (12, 20, 64), (6, 8, 0)]:
            ref = O.ref_hmm_query(path, 6, 1, pos_loss, win_loss, mx, ki=ki, kb=kb, max_occ=max_occ)
            port = O.anchors_hmm(ki, kb, 6, 1, max_occ, cons, emit, pos_loss, win_loss, mx)
            assert np.array_equal(ref, port), (path, pos_loss, win_loss, mx, ref.size, port.size)


def _golden():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "seed_hmm_golden.json")) as f:
        return json.load(f)


def test_seed_hmm_port_equals_golden():
    """The restatement against the reference's outputs in tests/golden/seed_hmm_golden.json
    (tests/golden/make_seed_hmm_golden.py): the inputs regenerated from their seeds (their
    digests checked), every output's count and SHA-256 equal; no reference tree needed.
    The profiles' emissions come from this package's parser, the consensus from them."""
    import hashlib
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_seed_hmm_golden import profile_texts, sha
    from protlocus_b200.hmm import parse_hmmer3
    g = _golden()
    for t in g["tables"]:
        e = emission_table(np.random.default_rng(t["seed"]), t["n"], t["kind"])
        assert hashlib.sha256(e.tobytes()).hexdigest() == t["digest"]
        s = O.sketch_hmm(e, *t["params"], use_ref=False)
        assert s.size == t["seeds"]["n"] and sha(s) == t["seeds"]["sha256"], (t["kind"], t["params"])
    ki, kb = O.seed_index(np.random.default_rng(g["index_seed"]), kmer=6, mod_bit=1, n_block=200_000)
    texts = profile_texts()
    for q in g["queries"]:
        text = texts[q["profile"]]
        assert hashlib.sha256(text.encode()).hexdigest() == q["text_sha256"]
        emit = parse_hmmer3(text)[0]["emit"]
        cons = O.hmm_consensus(emit)
        pos_loss, win_loss, mx, max_occ = q["params"]
        s = O.seeds_hmm_query(cons, emit, 6, 1, pos_loss, win_loss, mx)
        a = O.anchors_hmm(ki, kb, 6, 1, max_occ, cons, emit, pos_loss, win_loss, mx)
        assert s.size == q["seeds"]["n"] and sha(s) == q["seeds"]["sha256"], q["params"]
        assert a.size == q["anchors"]["n"] and sha(a) == q["anchors"]["sha256"], q["params"]


@pytest.mark.parametrize("kind", ["dirichlet", "ties", "stars", "flat"])
def test_device_functions_host_build_equal_restatement_and_reference(kind):
    """protlocus_b200/csrc/seed_hmm.cuh, the functions the device kernel runs per state and
    per window, built for the host: the same seeds in the same order as the restatement and,
    when built, the reference's mp_sketch_hmm, for every parameter set and table length."""
    rng = np.random.default_rng({"dirichlet": 21, "ties": 22, "stars": 23, "flat": 24}[kind])
    ref_lib = O.seed_ref_lib()
    for kmer, mod_bit, pos_loss, win_loss, mx in PARAMS:
        for n in sorted({0, 1, kmer - 1, kmer, 53, 300}):
            e = emission_table(rng, n, kind)
            dev = O.device_seed_fns_host(e, kmer, mod_bit, pos_loss, win_loss, mx)
            port = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=False)
            assert np.array_equal(dev, port), (kind, kmer, mod_bit, pos_loss, win_loss, mx, n)
            if ref_lib is not None:
                ref = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=True)
                assert np.array_equal(dev, ref)


@pytest.mark.parametrize("kind", ["wide", "stars", "dirichlet"])
def test_sketch_hmm_losses_past_16_bits(kind):
    """pos_loss over 32767 lets losses over 32767 into a state's list, where the reference
    keeps them in 16 bits (wrapped): the restatement and the device functions' host build
    follow it, checked against the reference where it is built (else the two against each
    other); window budgets at the int32 limits and negative."""
    rng = np.random.default_rng({"wide": 31, "stars": 32, "dirichlet": 33}[kind])
    ref_lib = O.seed_ref_lib()
    total = 0
    for kmer, mod_bit, pos_loss, win_loss, mx in WIDE_PARAMS:
        for n in (kmer, 60, 250):
            e = emission_table(rng, n, kind)
            port = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=False)
            dev = O.device_seed_fns_host(e, kmer, mod_bit, pos_loss, win_loss, mx)
            assert np.array_equal(dev, port), (kind, kmer, mod_bit, pos_loss, win_loss, mx, n)
            if ref_lib is not None:
                ref = O.sketch_hmm(e, kmer, mod_bit, pos_loss, win_loss, mx, use_ref=True)
                assert np.array_equal(ref, port), (kind, kmer, mod_bit, pos_loss, win_loss, mx, n, ref.size, port.size)
            total += port.size
    assert total > 0


@need_ref
@pytest.mark.parametrize("cap,budget", [(5, 7), (64, 300), (20, 0)])
def test_hmm_query_rescue_equals_reference(tmp_path, cap, budget):
    """An HMM-profile query with the accuracy mode's repeat rescue (map.c:360-384): the budget
    handed out over the merged seeds in their sorted order, from the hash of the query's name
    (the profile's name, as mp_map_hmm_file names the query); an index with 5 % repeat buckets."""
    from protlocus_b200.hmm import parse_hmmer3
    rng = np.random.default_rng(501 + cap)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, mean_occ=2.0, n_block=50_000, hot=1 << 15, hot_occ=300)
    for path in _profiles(tmp_path, 5, 503 + cap):
        cons, emit = O.ref_hmm_tables(path)
        name = parse_hmmer3(open(path).read())[0]["name"].encode()
        for pos_loss, win_loss, mx in [(6, 8, 16), (12, 20, 64)]:
            ref = O.ref_hmm_query(path, 6, 1, pos_loss, win_loss, mx, ki=ki, kb=kb, max_occ=20, repeat_cap=cap,
                                  budget=budget)
            port = O.anchors_hmm(ki, kb, 6, 1, 20, cons, emit, pos_loss, win_loss, mx, repeat_cap=cap, budget=budget,
                                 qname=name)
            assert np.array_equal(ref, port), (path, cap, budget, mx, ref.size, port.size)


@need_ref
def test_package_consensus_equals_reference_parser(tmp_path):
    """protlocus_b200.hmm.consensus, the query an HMM-profile mapping seeds from, equals the
    consensus the reference's parser stores (hmm.c:181-189), '*' emissions included."""
    from protlocus_b200.hmm import consensus
    for path in _profiles(tmp_path, 6, 71):
        cons, emit = O.ref_hmm_tables(path)
        assert consensus(emit) == cons == O.hmm_consensus(emit)
