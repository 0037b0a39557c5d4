"""GPU parity of the integer profile-HMM DP (mp_hmm_dp_score, hmm.c:252-291;
exact int32 scores) against the reference's golden vectors and the oracle.

The reference's own coverage is test/test_gpu.c:222-290 (two LCG profiles, one
3000-nt buffer and a five-region batch with an empty region); those cases are
in the fixture, and the reference test program itself runs against this
library in test_gpu_dropin.py.  Added here: profiles of one to three 256-column
tiles, regions with ambiguous codes, stop codons, lengths 0-5 and many regions
per batch.
"""
import ctypes

import numpy as np
import pytest

from protlocus_b200 import hmm as H
from protlocus_b200 import lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def test_hmm_golden(engine, hmm_golden):
    ca = H.codon_alpha()
    for p in hmm_golden["profiles"]:
        prof = L.HmmProfile(p["emit"], p["trans"], ca)
        regions = [np.frombuffer(bytes.fromhex(r), dtype=np.uint8) for r in p["regions"]]
        assert engine.hmm_score(prof, regions) == p["scores"], p["source"]
        assert engine.lib.pl_hmm_last_cells(engine.h) == sum(len(r) // 3 for r in regions) * p["m"]
        prof.close()


def test_hmm_sweep(engine, oracle):
    """Synthetic profiles of 1 to 5 tiles (m up to 1200), 40 regions each, against the restatement."""
    ca = H.codon_alpha()
    texts, probs = H.synthetic_profiles(6, seed=21, m_min=30, m_max=1200)
    rng = np.random.default_rng(4)
    for prof_t, pr in zip(H.parse_hmmer3("".join(texts)), probs):
        prof = L.HmmProfile(prof_t["emit"], prof_t["trans"], ca)
        regions = H.regions(rng, pr, 40, 0, 1500)
        got = engine.hmm_score(prof, regions)
        want = [oracle.port_hmm(prof_t["m"], prof_t["emit"], prof_t["trans"], ca, r) for r in regions]
        assert got == want
        prof.close()


def test_hmm_reference_entry_without_hmm_c():
    """mp_hmm_dp_score_gpu reports "not taken" (INT32_MIN) when the program links no hmm.c accessors."""
    nt = np.zeros(30, dtype=np.uint8)
    assert L.load().mp_hmm_dp_score_gpu(None, nt.ctypes.data, 30) == -2 ** 31


def test_hmm_many_profiles_equal_one_by_one(engine):
    """pl_hmm_score_many_device (the region set planned and translated once, the profiles'
    launches side by side on the engine's HMM streams) gives every profile's per-call scores:
    nine profiles of 1-4 tiles (more than there are streams, so streams are reused), one
    with another codon table (the rows are translated again), 60 regions of 0-2500 nt."""
    ca = H.codon_alpha()
    texts, probs = H.synthetic_profiles(9, seed=31, m_min=20, m_max=1000)
    tabs = H.parse_hmmer3("".join(texts))
    ca2 = ca.copy()
    ca2[[3, 7, 11]] = 20  # three more codons without emission
    profs = [L.HmmProfile(t["emit"], t["trans"], ca2 if k == 5 else ca) for k, t in enumerate(tabs)]
    rng = np.random.default_rng(32)
    regions = H.regions(rng, probs[0], 60, 0, 2500)
    try:
        many = engine.hmm_score_many(profs, regions)
        lens = np.array([len(r) for r in regions], dtype=np.int32)
        offs = np.concatenate([[0], np.cumsum(lens[:-1])]).astype(np.int32)
        nt = np.ascontiguousarray(np.concatenate(regions).astype(np.uint8))
        host = np.zeros((len(profs), len(regions)), dtype=np.int32)
        handles = (ctypes.c_void_p * len(profs))(*[p.h for p in profs])
        assert engine.lib.pl_hmm_score_many_host(engine.h, handles, len(profs), len(regions), nt.ctypes.data, nt.size,
                                                 offs.ctypes.data, lens.ctypes.data, host.ctypes.data), L.error()
        assert np.array_equal(host, many)
        for k, prof in enumerate(profs):
            assert many[k].tolist() == engine.hmm_score(prof, regions), k
        assert engine.lib.pl_hmm_last_cells(engine.h) == sum(len(r) // 3 for r in regions) * tabs[-1]["m"]
    finally:
        for prof in profs:
            prof.close()
