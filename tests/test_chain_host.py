"""The host half of batched chaining (pl_chain_finish: backtrack, compaction and the
reference's radix sort) against the reference's own mp_chain, on the CPU.

The fill (f, p) comes from the Python restatement of chain.c:160-208
(tests/chain_ref.py); the library turns it into chains; the reference's mp_chain
(oracle/_ref/libchain_ref.so, compiled from chain.c where it lies) must give the
same chain words and anchors.  Cases: the synthetic coarse-mapping anchors under
the pre-chain and main-chain arguments, nucleotide coordinates (bbit 0), a small
max_iter and max_skip, more than 64 chains (the radix sort path of the
compaction), score ties, and empty and one-anchor queries.
"""
import numpy as np
import pytest

import chain_ref as CR
import oracle_lib as O
from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import chain_opt

need = pytest.mark.skipif(O.chain_lib() is None, reason="oracle/_ref/libchain_ref.so not built")


def _check(opt, a):
    f, p, _v = CR.fill(a, opt)
    got_u, got_a = L.chain_finish(opt, a, f, p)
    want_u, want_a = O.ref_chain(opt, a)
    assert np.array_equal(got_u, want_u), (got_u[:8], want_u[:8])
    assert np.array_equal(got_a, want_a)
    return len(want_u)


@need
@pytest.mark.parametrize("kind", ["main", "pre"])
def test_synthetic_queries(kind):
    opt = chain_opt(kind)
    n_chains = 0
    for a in W.chain_anchors(24, seed=3, al_median=200):
        n_chains += _check(opt, a)
    assert n_chains > 24


@need
def test_nucleotide_coordinates_and_limits():
    opt = chain_opt("main", max_intron=5000, bbit=0, kmer=5)
    for a in W.chain_anchors(12, seed=4, genome_len=2_000_000, bbit=0, al_median=150):
        _check(opt, a)
    tight = dict(chain_opt("main"), max_iter=5, max_skip=2)
    for a in W.chain_anchors(12, seed=5, al_median=150, hit_rate=0.5):
        _check(tight, a)


@need
def test_many_chains_and_ties():
    rng = np.random.default_rng(6)
    # 120 separate clusters of 3-5 collinear anchors with equal scores: >64 chains
    anchors = []
    for c in range(120):
        b0, q0 = 1000 * c, int(rng.integers(0, 50))
        for k in range(int(rng.integers(3, 6))):
            anchors.append((b0 + k) << 32 | (q0 + 3 * k))
    a = np.unique(np.array(anchors, np.uint64))
    assert _check(chain_opt("main", max_intron=2000), a) > 64
    # one long diagonal with duplicated query positions: many equal f values
    a = np.unique(np.array([(k // 2) << 32 | (k % 7 + 6 * (k // 2)) for k in range(300)], np.uint64))
    _check(chain_opt("main"), a)


@need
def test_empty_and_single():
    opt = chain_opt("main")
    for a in (np.zeros(0, np.uint64), np.array([5 << 32 | 7], np.uint64),
              np.array([5 << 32 | 7, 5 << 32 | 13], np.uint64)):
        _check(opt, a)


def test_corrupt_predecessors_are_an_error():
    """The host backtrack refuses a predecessor array with a forward or self link (it
    would otherwise walk forever) instead of looping."""
    opt = chain_opt("main")
    a = np.array([(k // 3) << 32 | (5 * k) for k in range(40)], np.uint64)
    f = np.arange(10, 50, dtype=np.int32)
    p = np.arange(-1, 39, dtype=np.int32)
    p[20] = 25  # a forward link
    with pytest.raises(RuntimeError):
        L.chain_finish(opt, a, f, p)
    p[20] = 20  # a self link
    with pytest.raises(RuntimeError):
        L.chain_finish(opt, a, f, p)


@need
@pytest.mark.parametrize("seed", range(6))
def test_random_arguments(seed):
    """mp_chain's arguments drawn at random (non-spliced penalties and max_drop = bw,
    positive min_sc, min_cnt, small bw and max_dist_y, bbit 0 / 4 / 8, kmer, coefficient):
    the restated fill plus the library's host half equal the reference."""
    rng = np.random.default_rng(100 + seed)
    bbit = int(rng.choice([0, 4, 8]))
    opt = dict(max_dist_x=int(rng.integers(200, 40000)), max_dist_y=int(rng.integers(50, 2000)),
               bw=int(rng.integers(100, 40000)), max_skip=int(rng.integers(1, 40)),
               max_iter=int(rng.integers(3, 5000)), min_cnt=int(rng.integers(1, 5)), min_sc=int(rng.integers(0, 40)),
               coef=float(rng.uniform(0.2, 1.5)), is_spliced=int(rng.integers(0, 2)), kmer=int(rng.integers(4, 8)),
               bbit=bbit)
    glen = 5_000_000 if bbit == 0 else 100_000_000
    for a in W.chain_anchors(10, seed=200 + seed, genome_len=glen, bbit=bbit, al_median=180):
        _check(opt, a)


def _golden_cases():
    import json
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_chain_golden as G
    with open(os.path.join(here, "golden", "chain_golden.json")) as f:
        data = json.load(f)
    for case in data["cases"]:
        qs = G.case_queries(case["gen"])
        assert G.digest(qs) == case["sha256"], case["name"]  # the generator still makes the same anchors
        yield case, qs


def test_golden_fixture():
    """The restated fill plus the library's host half reproduce the fixture the
    reference's mp_chain wrote (tests/golden/make_chain_golden.py); no reference
    build needed."""
    for case, qs in _golden_cases():
        for a, want in zip(qs, case["chains"]):
            f, p, _v = CR.fill(a, case["opt"])
            u, out = L.chain_finish(case["opt"], a, f, p)
            assert [int(x) for x in u] == want["u"], case["name"]
            assert [int(x) for x in out] == want["a"], case["name"]
