"""Batched anchor chaining on the device (chain.cu + plchain.c) against the reference's
own mp_chain (chain.c:160, oracle/_ref/libchain_ref.so) and, for the fill arrays
themselves, against the restatement in tests/chain_ref.py.

* pl_chain_host over batches of synthetic coarse-mapping queries under the main-chain
  and pre-chain arguments, nucleotide coordinates (bbit 0), tight max_iter/max_skip,
  empty and one-anchor queries and one dense query of 20000 anchors: chain words and
  chained anchors equal the reference's for every query;
* pl_chain_fill_device: f, p and v of every anchor equal the restatement's.
"""
import ctypes as C

import numpy as np
import pytest

import chain_ref as CR
import oracle_lib as O
from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import chain_opt, chain_opt_struct

pytestmark = pytest.mark.gpu
need = pytest.mark.skipif(O.chain_lib() is None, reason="oracle/_ref/libchain_ref.so not built")


def _batch(eng, opt, queries):
    got = eng.chain(opt, queries)
    n_chains = 0
    for q, a in enumerate(queries):
        want_u, want_a = O.ref_chain(opt, a)
        assert np.array_equal(got[q][0], want_u), (q, got[q][0][:6], want_u[:6])
        assert np.array_equal(got[q][1], want_a), q
        n_chains += len(want_u)
    return n_chains


@need
@pytest.mark.parametrize("kind", ["main", "pre"])
def test_batch_matches_reference(kind):
    eng = L.Engine(0)
    try:
        qs = W.chain_anchors(600, seed=11)
        qs += [np.zeros(0, np.uint64), np.array([3 << 32 | 1], np.uint64)]
        assert _batch(eng, chain_opt(kind), qs) > 600
    finally:
        eng.close()


@need
def test_nucleotide_coordinates_tight_limits_and_dense():
    eng = L.Engine(0)
    try:
        _batch(eng, chain_opt("main", max_intron=5000, bbit=0, kmer=5),
               W.chain_anchors(200, seed=12, genome_len=2_000_000, bbit=0, al_median=150))
        _batch(eng, dict(chain_opt("main"), max_iter=5, max_skip=2), W.chain_anchors(200, seed=13, hit_rate=0.5))
        rng = np.random.default_rng(14)
        dense = np.unique(((rng.integers(0, 4000, 20000).astype(np.uint64)) << np.uint64(32)) |
                          rng.integers(0, 2500, 20000).astype(np.uint64))
        _batch(eng, chain_opt("main"), [dense] + W.chain_anchors(50, seed=15))
    finally:
        eng.close()


@need
def test_fill_arrays_match_restatement():
    torch = pytest.importorskip("torch")
    eng = L.Engine(0)
    try:
        opt = chain_opt("main")
        qs = W.chain_anchors(40, seed=16, al_median=250)
        off, n, a = L.chain_pack(qs)
        d_a = torch.from_numpy(a.view(np.int64).copy()).cuda()
        d_f, d_p, d_v = (torch.zeros(len(a), dtype=torch.int32, device="cuda") for _ in range(3))
        o = chain_opt_struct(opt)
        assert eng.lib.pl_chain_fill_device(eng.h, C.byref(o), len(qs), off.ctypes.data, n.ctypes.data, d_a.data_ptr(),
                                            len(a), d_f.data_ptr(), d_p.data_ptr(), d_v.data_ptr(), None), L.error()
        torch.cuda.synchronize()
        f, p, v = d_f.cpu().numpy(), d_p.cpu().numpy(), d_v.cpu().numpy()
        for q, x in enumerate(qs):
            wf, wp, wv = CR.fill(x, opt)
            s = slice(int(off[q]), int(off[q]) + len(x))
            assert np.array_equal(f[s], wf) and np.array_equal(p[s], wp) and np.array_equal(v[s], wv), q
    finally:
        eng.close()


@need
@pytest.mark.parametrize("seed", range(4))
def test_random_arguments_match_reference(seed):
    """The device DP plus host half under random mp_chain arguments (non-spliced
    penalties, positive min_sc, small bw and max_dist_y, bbit 0 / 4 / 8, kmer, coefficient)."""
    rng = np.random.default_rng(300 + seed)
    bbit = int(rng.choice([0, 4, 8]))
    opt = dict(max_dist_x=int(rng.integers(200, 40000)), max_dist_y=int(rng.integers(50, 2000)),
               bw=int(rng.integers(100, 40000)), max_skip=int(rng.integers(1, 40)),
               max_iter=int(rng.integers(3, 5000)), min_cnt=int(rng.integers(1, 5)), min_sc=int(rng.integers(0, 40)),
               coef=float(rng.uniform(0.2, 1.5)), is_spliced=int(rng.integers(0, 2)), kmer=int(rng.integers(4, 8)),
               bbit=bbit)
    glen = 5_000_000 if bbit == 0 else 100_000_000
    eng = L.Engine(0)
    try:
        _batch(eng, opt, W.chain_anchors(150, seed=400 + seed, genome_len=glen, bbit=bbit, al_median=180))
    finally:
        eng.close()


def test_golden_fixture_on_device():
    """Device DP plus host half against the fixture the reference's mp_chain wrote."""
    from test_chain_host import _golden_cases
    eng = L.Engine(0)
    try:
        for case, qs in _golden_cases():
            got = eng.chain(case["opt"], qs)
            for (u, out), want in zip(got, case["chains"]):
                assert [int(x) for x in u] == want["u"], case["name"]
                assert [int(x) for x in out] == want["a"], case["name"]
    finally:
        eng.close()
