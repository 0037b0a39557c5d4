"""Seeding on the device (seed.cu, pl_seed_anchors_host) against the reference's own
steps (map.c's mp_sketch_query, mp_cal_max_occ, mp_collect_anchors and the anchor sort,
oracle/_ref/libseed_ref.so; the restatement oracle/seed_port.c where that is not built):
the same sorted anchors per protein, bit for bit, on synthetic indexes in the mapper's
layout with hot (repeat) buckets, for several sampling rates and occurrence caps;
proteins with stops, X, lowercase letters, residue codes, repeats, and fewer than 8 seeds.
Also: an empty batch, an empty index, and the capacity rule (a_off filled, anchors not)."""
import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L
from test_seed import seed_proteins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("mod_bit,max_occ", [(1, 20000), (1, 40), (2, 500), (0, 200)])
def test_seed_anchors_match_reference(engine, mod_bit, max_occ):
    rng = np.random.default_rng(200 + mod_bit * 7 + max_occ)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=mod_bit, n_block=300_000)
    idx = L.SeedIndex(ki, kb, 6, mod_bit)
    try:
        prots = seed_proteins(rng, 300)
        got = L.seed_anchors(engine, idx, prots, max_occ)
        for q, seq in enumerate(prots):
            want = O.seed_anchors(ki, kb, 6, mod_bit, max_occ, seq)
            assert np.array_equal(got[q], want), (q, len(seq), got[q].size, want.size)
    finally:
        idx.close()


def test_seed_edges(engine):
    rng = np.random.default_rng(7)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=1000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    lib = engine.lib
    import ctypes as C
    try:
        assert L.seed_anchors(engine, idx, [], 100) == []
        prots = seed_proteins(rng, 20)
        want = [O.seed_anchors(ki, kb, 6, 1, 20000, s) for s in prots]
        # the capacity rule: a too small array gets the offsets only
        n = len(prots)
        lens = np.array([len(p) for p in prots], np.int32)
        offs = np.zeros(n, np.int64)
        offs[1:] = np.cumsum(lens[:-1])
        seq = np.frombuffer(b"".join(prots), np.uint8).copy()
        a_off = np.zeros(n + 1, np.int64)
        a = np.zeros(1, np.uint64)
        tot = lib.pl_seed_anchors_host(engine.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                       lens.ctypes.data, 20000, a_off.ctypes.data, a.ctypes.data, 0)
        assert tot == sum(w.size for w in want) and list(np.diff(a_off)) == [w.size for w in want]
        # a protein span past the sequence is refused
        bad = lens.copy()
        bad[-1] += 5
        assert lib.pl_seed_anchors_host(engine.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                        bad.ctypes.data, 20000, a_off.ctypes.data, a.ctypes.data, 0) == -1
    finally:
        idx.close()
    empty = L.SeedIndex(np.zeros(1 << 23, np.int64), np.zeros(0, np.uint32), 6, 1)
    try:
        got = L.seed_anchors(engine, empty, [b"ARNDCQEGHILK" * 5], 100)
        assert got[0].size == 0
    finally:
        empty.close()


@pytest.mark.parametrize("max_occ,cap,budget", [(40, 64, 250000), (40, 64, 300), (20, 200, 50), (20, 5, 7), (20, 5, 0)])
def test_seed_rescue_matches_reference(engine, max_occ, cap, budget):
    """The accuracy mode's repeat rescue on an index with 5 % repeat buckets: evenly spaced
    blocks of the over-cap buckets, the budget's scaled shares and round-robin from the query
    name's hash, over the seeds in their sorted order."""
    from test_seed import rescue_index
    rng = np.random.default_rng(400 + cap + budget)
    ki, kb = rescue_index(rng)
    idx = L.SeedIndex(ki, kb, 5, 1)
    try:
        prots = seed_proteins(rng, 200)
        names = [b"query_%d" % q for q in range(len(prots))]
        assert all(engine.lib.pl_seed_qname_hash(nm) == O.seed_qname_hash(nm) for nm in names)
        got = L.seed_anchors(engine, idx, prots, max_occ, cap, budget, names)
        for q, seq in enumerate(prots):
            want = O.seed_anchors_acc(ki, kb, 5, 1, max_occ, cap, budget, names[q], seq)
            assert np.array_equal(got[q], want), (q, len(seq), got[q].size, want.size)
    finally:
        idx.close()


def test_seed_anchors_on_device_feed_chaining(engine):
    """pl_seed_anchors_opt_device leaves the anchors on the device with the same offsets; the
    chaining DP runs on them in place (pl_chain_fill_device) and, finished on the host, gives the
    chains pl_chain_host gives from the host anchors."""
    import ctypes as C
    import torch
    from protlocus_b200.abi import chain_opt, chain_opt_struct
    rng = np.random.default_rng(77)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=1, n_block=4000)
    idx = L.SeedIndex(ki, kb, 6, 1)
    try:
        prots = seed_proteins(rng, 120)
        host = L.seed_anchors(engine, idx, prots, 20000)
        n = len(prots)
        lens = np.array([len(p) for p in prots], np.int32)
        offs = np.zeros(n, np.int64)
        offs[1:] = np.cumsum(lens[:-1])
        seq = np.frombuffer(b"".join(prots), np.uint8).copy()
        a_off = np.zeros(n + 1, np.int64)
        a_dev = C.c_void_p()
        so = L.SeedOpt(20000, 0, 0, None)
        tot = engine.lib.pl_seed_anchors_opt_device(engine.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                                    lens.ctypes.data, C.byref(so), a_off.ctypes.data, C.byref(a_dev))
        assert tot == sum(h.size for h in host) > 0 and list(np.diff(a_off)) == [h.size for h in host]
        opt = chain_opt("main")
        o = chain_opt_struct(opt)
        off, nq = a_off[:-1].copy(), np.diff(a_off).astype(np.int32)
        d_f, d_p, d_v = (torch.zeros(int(tot), dtype=torch.int32, device="cuda") for _ in range(3))
        assert engine.lib.pl_chain_fill_device(engine.h, C.byref(o), n, off.ctypes.data, nq.ctypes.data, a_dev.value,
                                               int(tot), d_f.data_ptr(), d_p.data_ptr(), d_v.data_ptr(), None), L.error()
        torch.cuda.synchronize()
        f, p = d_f.cpu().numpy(), d_p.cpu().numpy()
        want = engine.chain(opt, host)
        for q in range(n):
            s = slice(int(off[q]), int(off[q]) + int(nq[q]))
            u, a_out = L.chain_finish(opt, host[q], f[s], p[s])
            assert np.array_equal(u, want[q][0]) and np.array_equal(a_out, want[q][1]), q
    finally:
        idx.close()


def test_seed_device_equals_golden(engine):
    """The device against the anchors the reference's own steps wrote (tests/golden/seed_golden.json)."""
    import json
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_seed_golden as G
    with open(os.path.join(os.path.dirname(__file__), "golden", "seed_golden.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        ki, kb, ps, names = G.case_inputs(tuple(c["index"]), tuple(c["proteins"]))
        assert G.digest(ki, kb, ps) == c["digest"], c["name"]
        idx = L.SeedIndex(ki, kb, c["index"][0], c["index"][1])
        try:
            got = L.seed_anchors(engine, idx, ps, c["max_occ"], c["repeat_cap"], c["budget"], names)
        finally:
            idx.close()
        for q in range(len(ps)):
            assert [int(x) for x in got[q]] == c["anchors"][q], (c["name"], q)
