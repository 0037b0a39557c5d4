"""The seeding restatement (oracle/seed_port.c) against the reference's own steps
(map.c's mp_sketch_query, mp_cal_max_occ, mp_collect_anchors and the anchor sort,
map.c:304-397 and :565-572, sketch.c:18-37; oracle/_ref/libseed_ref.so built from the
reference's sources with oracle/seed_ref_hook.c): the same sorted anchors, on
synthetic indexes in the reference's layout.  Proteins: random residues, repeats of a
short motif (hot buckets), stop and X runs (k-mer restarts), lowercase letters,
residue codes, very short ones (fewer than 8 seeds: the option's cap alone)."""
import numpy as np
import pytest

import oracle_lib as O

need_ref = pytest.mark.skipif(O.seed_ref_lib() is None, reason="oracle/_ref/libseed_ref.so not built")
AA = b"ARNDCQEGHILKMFPSTWYV"


def seed_proteins(rng, n):
    out = []
    for q in range(n):
        L = int(rng.integers(1, 1200))
        s = bytearray(AA[int(x)] for x in rng.integers(0, 20, size=L))
        kind = q % 6
        if kind == 1 and L > 40:  # a repeated motif: the same k-mers many times
            m = bytes(s[:7])
            for p in range(0, L - 7, 9):
                s[p:p + 7] = m
        elif kind == 2:  # stops and X restart the k-mer
            for p in rng.integers(0, L, size=max(1, L // 30)):
                s[p] = ord("*") if rng.random() < 0.5 else ord("X")
        elif kind == 3:
            s = bytearray(s.lower())
        elif kind == 4:  # residue codes 0-21 instead of letters
            s = bytearray(int(x) for x in rng.integers(0, 22, size=L))
        elif kind == 5:
            s = s[: int(rng.integers(1, 12))]
        out.append(bytes(s))
    return out


@need_ref
@pytest.mark.parametrize("mod_bit,max_occ", [(1, 20000), (1, 40), (2, 20000), (0, 200)])
def test_seed_port_equals_reference(mod_bit, max_occ):
    rng = np.random.default_rng(100 + mod_bit * 7 + max_occ)
    ki, kb = O.seed_index(rng, kmer=6, mod_bit=mod_bit, n_block=200_000)
    for seq in seed_proteins(rng, 60):
        ref = O.seed_anchors(ki, kb, 6, mod_bit, max_occ, seq, use_ref=True)
        port = O.seed_anchors(ki, kb, 6, mod_bit, max_occ, seq, use_ref=False)
        assert np.array_equal(ref, port), (len(seq), ref.size, port.size)


def test_seed_port_hand_case():
    """ARNDCQ (six residues, kmer 6): one k-mer, a seed iff its hash has mod_bit zero low bits;
    with mod_bit 0 every k-mer is a seed, and a bucket of three blocks gives three anchors."""
    kmer, mod_bit = 6, 0
    n_bucket = 1 << (kmer * 4)
    ki = np.zeros(n_bucket, dtype=np.int64)
    kb = np.zeros(0, dtype=np.uint32)
    a = O.seed_anchors(ki, kb, kmer, mod_bit, 100, b"ARNDCQ", use_ref=False)
    assert a.size == 0  # empty index
    # the seed's bucket, from the port's sketch: give it three blocks
    import ctypes as C
    lib = O.port_lib()
    lib.sp_sketch.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    sd = np.zeros(8, np.uint64)
    assert lib.sp_sketch(b"ARNDCQ", 6, kmer, mod_bit, sd.ctypes.data) == 1
    b = int(sd[0] >> np.uint64(32))
    ki[b + 1:] = 3
    kb = np.array([7, 5, 9], dtype=np.uint32)
    a = O.seed_anchors(ki, kb, kmer, mod_bit, 100, b"ARNDCQ", use_ref=False)
    assert [int(x >> np.uint64(32)) for x in a] == [5, 7, 9] and all(int(x) & 0xffffffff == 5 for x in a)


@need_ref
@pytest.mark.parametrize("max_occ,cap,budget", [(40, 64, 250000), (40, 64, 300), (20, 200, 50), (20, 5, 7),
                                                (20, 5, 0)])
def test_seed_port_rescue_equals_reference(max_occ, cap, budget):
    """The accuracy mode's repeat rescue: evenly spaced blocks of the over-cap buckets, and with
    a small budget the scaled shares plus the round-robin from the query name's hash."""
    rng = np.random.default_rng(300 + cap + budget)
    ki, kb = rescue_index(rng)
    lib = O.seed_ref_lib()
    import ctypes as C
    lib.ref_seed_qname_hash.argtypes = [C.c_char_p]
    lib.ref_seed_qname_hash.restype = C.c_uint32
    rescued = 0
    for q, seq in enumerate(seed_proteins(rng, 60)):
        name = b"query_%d" % q
        assert O.seed_qname_hash(name) == lib.ref_seed_qname_hash(name)
        ref = O.seed_anchors_acc(ki, kb, 5, 1, max_occ, cap, budget, name, seq, use_ref=True)
        port = O.seed_anchors_acc(ki, kb, 5, 1, max_occ, cap, budget, name, seq, use_ref=False)
        assert np.array_equal(ref, port), (q, len(seq), ref.size, port.size)
        rescued += ref.size != O.seed_anchors(ki, kb, 5, 1, max_occ, seq, use_ref=False).size
    assert rescued >= 10 if budget > 0 else rescued == 0  # a zero budget takes nothing (map.c:365-383)


def rescue_index(rng):
    """kmer 5 (2^19 buckets) with 5 % repeat buckets of 150-300 blocks, so that proteins meet
    buckets over the occurrence cap"""
    return O.seed_index(rng, kmer=5, mod_bit=1, n_block=100_000, hot=1 << 19 >> 4, hot_occ=300)


def test_seed_boundary_host_checks():
    """The library's host logic for seeding, no device touched: the query-name hash equals the
    reference's mp_hash_qname (and the restatement's), and an index of the wrong shape or a
    missing engine is refused with a reason."""
    import ctypes as C
    from protlocus_b200 import lib as L
    lib = L.load()
    ref = O.seed_ref_lib()
    for name in [b"", b"q", b"sp|P12345|TITIN_HUMAN", bytes(range(1, 200))]:
        h = lib.pl_seed_qname_hash(name)
        assert h == O.seed_qname_hash(name)
        if ref is not None:
            ref.ref_seed_qname_hash.argtypes = [C.c_char_p]
            ref.ref_seed_qname_hash.restype = C.c_uint32
            assert h == ref.ref_seed_qname_hash(name)
    ki = np.zeros(8, np.int64)
    kb = np.zeros(1, np.uint32)
    # 8 buckets do not fit kmer 6, mod_bit 1 (2^23 buckets); kmer 9 is over the 32-bit k-mer
    assert not lib.pl_seed_index_create(0, ki.ctypes.data, 8, kb.ctypes.data, 1, 6, 1)
    assert "buckets" in L.error()
    assert not lib.pl_seed_index_create(0, ki.ctypes.data, 8, kb.ctypes.data, 1, 9, 33)
    # kmer 8: the reference's mask (1U << 32) - 1 is an undefined shift, so no parity to keep
    assert not lib.pl_seed_index_create(0, ki.ctypes.data, 8, kb.ctypes.data, 1, 8, 29)
    assert "kmer 1-7" in L.error()
    a_off = np.zeros(2, np.int64)
    so = L.SeedOpt(100, 0, 0, None)
    assert lib.pl_seed_anchors_opt_host(None, None, 1, None, 0, None, None, C.byref(so), a_off.ctypes.data, None, 0) == -1


def _golden():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "seed_golden.json")) as f:
        return json.load(f)["cases"]


def test_seed_port_equals_golden():
    """The restatement against the anchors the reference's own steps wrote
    (tests/golden/make_seed_golden.py); no reference tree needed."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_seed_golden as G
    rescued = 0
    for c in _golden():
        ki, kb, ps, names = G.case_inputs(tuple(c["index"]), tuple(c["proteins"]))
        assert G.digest(ki, kb, ps) == c["digest"], c["name"]
        kmer, mod_bit = c["index"][0], c["index"][1]
        for q, (p, nm) in enumerate(zip(ps, names)):
            if c["repeat_cap"] > 0:
                a = O.seed_anchors_acc(ki, kb, kmer, mod_bit, c["max_occ"], c["repeat_cap"], c["budget"], nm, p,
                                       use_ref=False)
                rescued += a.size != O.seed_anchors(ki, kb, kmer, mod_bit, c["max_occ"], p, use_ref=False).size
            else:
                a = O.seed_anchors(ki, kb, kmer, mod_bit, c["max_occ"], p, use_ref=False)
            assert [int(x) for x in a] == c["anchors"][q], (c["name"], q)
    assert rescued >= 10
