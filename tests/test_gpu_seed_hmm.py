"""Seeding of HMM-profile queries on the device (seed.cu: k_seed_hmm_alts, k_seed_hmm_enum,
k_seed_unique; pl_seed_anchors_hmm_host / _device) against the restatement
(oracle/seed_port.c sp_anchors_hmm, itself checked against the reference's mp_sketch_hmm,
mp_sketch_query and mp_map_coarse steps in tests/test_seed_hmm.py and pinned by
tests/golden/seed_hmm_golden.json): the same sorted anchors per query, bit for bit.

Queries: the consensus of each profile (the parser's, hmm.c:181-189) with its match
emissions; Dirichlet profiles written as HMMER3 text and read by this package's parser,
tables with ties, unreadable entries, flat rows and losses past 16 bits; profiles shorter
than a k-mer and empty ones; the defaults (options.c:112-114) and wider budgets, one k-mer
per window, the rescue, the golden fixture's queries, and the anchors left on the device."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L
from test_seed_hmm import emission_table

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def _device_u64(ptr: int, n: int) -> np.ndarray:
    """n uint64 at a device address, read through torch (the engine's stream synchronised by
    the entry point before it returns)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False), "version": 2}
    return torch.as_tensor(_View(), device="cuda").cpu().numpy().view(np.uint64)


def hmm_queries(rng, n: int):
    """n (consensus, emissions) pairs of mixed kinds and lengths, some empty or shorter than a k-mer."""
    from protlocus_b200.hmm import parse_hmmer3, synthetic_profiles
    texts, _ = synthetic_profiles(max(n // 3, 1), seed=int(rng.integers(1 << 30)), m_min=20, m_max=400)
    tabs = [parse_hmmer3(t)[0]["emit"] for t in texts]
    kinds = ["dirichlet", "ties", "stars", "flat", "wide"]
    while len(tabs) < n:
        k = len(tabs)
        m = [0, 3, 6][k % 3] if k % 7 == 0 else int(rng.integers(7, 500))
        tabs.append(emission_table(rng, m, kinds[k % len(kinds)]))
    return [(O.hmm_consensus(e), e) for e in tabs[:n]]


@pytest.mark.parametrize("pos_loss,win_loss,seed_max,max_occ",
                         [(6, 8, 16, 20000), (12, 20, 64, 40), (6, 8, 1, 20000), (100, 1000, 300, 500),
                          (40000, 40000, 16, 20000)])
def test_hmm_seed_anchors_match_oracle(engine, pos_loss, win_loss, seed_max, max_occ):
    rng = np.random.default_rng(300 + seed_max + max_occ % 97)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=300_000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        qs = hmm_queries(rng, 90)
        got = L.seed_anchors(engine, idx, [c for c, _ in qs], max_occ, profiles=[e for _, e in qs],
                             pos_loss=pos_loss, win_loss=win_loss, seed_max=seed_max)
        for q, (cons, emit) in enumerate(qs):
            want = O.anchors_hmm(ki, kb, 6, 1, max_occ, cons, emit, pos_loss, win_loss, seed_max)
            assert np.array_equal(got[q], want), (q, len(cons), got[q].size, want.size)
    finally:
        idx.close()


def test_hmm_seed_max_zero_is_the_default_path(engine):
    """seed_max 0: the query's own seeds only, the anchors of the default mode."""
    rng = np.random.default_rng(17)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=100_000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        qs = hmm_queries(rng, 30)
        prots = [c for c, _ in qs]
        a = L.seed_anchors(engine, idx, prots, 20000, profiles=[e for _, e in qs], seed_max=0)
        b = L.seed_anchors(engine, idx, prots, 20000)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
    finally:
        idx.close()


@pytest.mark.parametrize("cap,budget", [(5, 7), (64, 300)])
def test_hmm_seed_rescue_matches_oracle(engine, cap, budget):
    rng = np.random.default_rng(600 + cap)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, mean_occ=2.0, n_block=50_000, hot=1 << 15, hot_occ=300)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        qs = hmm_queries(rng, 40)
        names = [b"prof%d" % q for q in range(len(qs))]
        got = L.seed_anchors(engine, idx, [c for c, _ in qs], 20, repeat_cap=cap, budget=budget, names=names,
                             profiles=[e for _, e in qs])
        for q, (cons, emit) in enumerate(qs):
            want = O.anchors_hmm(ki, kb, 6, 1, 20, cons, emit, 6, 8, 16, repeat_cap=cap, budget=budget,
                                 qname=names[q])
            assert np.array_equal(got[q], want), (q, got[q].size, want.size)
    finally:
        idx.close()


def test_hmm_seed_device_equals_golden(engine):
    """The device against the anchors the reference's own steps wrote for synthetic profiles
    (tests/golden/seed_hmm_golden.json: counts and SHA-256 digests)."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_seed_hmm_golden import profile_texts, sha
    from protlocus_b200.hmm import parse_hmmer3
    from test_seed_hmm import _golden
    g = _golden()
    ki, kb = O.seed_index(np.random.default_rng(g["index_seed"]), kmer=6, mod_bit=1, n_block=200_000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        texts = profile_texts()
        for q in g["queries"]:
            emit = parse_hmmer3(texts[q["profile"]])[0]["emit"]
            pos_loss, win_loss, mx, max_occ = q["params"]
            a = L.seed_anchors(engine, idx, [O.hmm_consensus(emit)], max_occ, profiles=[emit], pos_loss=pos_loss,
                               win_loss=win_loss, seed_max=mx)[0]
            assert a.size == q["anchors"]["n"] and sha(a) == q["anchors"]["sha256"], q["params"]
    finally:
        idx.close()


def test_hmm_seed_anchors_left_on_device(engine):
    """pl_seed_anchors_hmm_device: the same offsets and anchors as the host entry point, in
    device memory; a profile range past the emission table is refused with the reason."""
    rng = np.random.default_rng(23)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=100_000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        qs = hmm_queries(rng, 25)
        prots = [c for c, _ in qs]
        want = L.seed_anchors(engine, idx, prots, 20000, profiles=[e for _, e in qs])
        n = len(qs)
        lens = np.array([len(p) for p in prots], np.int32)
        offs = np.zeros(n, np.int64)
        offs[1:] = np.cumsum(lens[:-1])
        seq = np.frombuffer(b"".join(prots), np.uint8).copy()
        e_len = np.array([e.shape[0] for _, e in qs], np.int32)
        e_off = np.zeros(n, np.int64)
        e_off[1:] = np.cumsum(e_len[:-1])
        emit = np.ascontiguousarray(np.concatenate([e for _, e in qs]).astype(np.int16))
        h = L.SeedHmm(emit.ctypes.data, int(e_len.sum()), e_off.ctypes.data, e_len.ctypes.data, 6, 8, 16, 0)
        o = L.SeedOpt(20000, 0, 0, None)
        a_off = np.zeros(n + 1, np.int64)
        a_dev = C.c_void_p()
        tot = engine.lib.pl_seed_anchors_hmm_device(engine.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                                    lens.ctypes.data, C.byref(o), C.byref(h), a_off.ctypes.data,
                                                    C.byref(a_dev))
        assert tot == sum(w.size for w in want) and list(np.diff(a_off)) == [w.size for w in want]
        if tot > 0:
            got = _device_u64(a_dev.value, int(tot))
            assert np.array_equal(got, np.concatenate(want))
        # a profile past the table: refused before any device work
        bad = np.array(e_off)
        bad[-1] = int(e_len.sum())
        h2 = L.SeedHmm(emit.ctypes.data, int(e_len.sum()), bad.ctypes.data, e_len.ctypes.data, 6, 8, 16, 0)
        if e_len[-1] > 0:
            assert engine.lib.pl_seed_anchors_hmm_host(engine.h, idx.h, n, seq.ctypes.data, seq.size,
                                                       offs.ctypes.data, lens.ctypes.data, C.byref(o), C.byref(h2),
                                                       a_off.ctypes.data, None, 0) == -1
            assert "profile" in L.error()
    finally:
        idx.close()
