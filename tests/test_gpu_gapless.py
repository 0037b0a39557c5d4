"""GPU parity of the gapless X-drop candidate prefilter (ns_gapless_xdrop_batch,
nasw-cuda.cu:1151-1295; int32 scores, bit-exact).

The fixture holds the reference kernel's own scores (run from the reference's
nasw-cuda.cu, tests/golden/make_gapless_golden.py), including its edge cases
(invalid query ends, no anchors, more than 32 anchors, blocks past the contig
end, runs of N).  The sweeps compare against the C restatement: other seeds,
x-drop values, k-mer sizes and block widths, and both entry points (the
reference's ns_gpu_gapless_score_batch with its genome cache, and the bulk
pl_gapless_score_host).
"""
import numpy as np
import pytest

from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import BLOSUM62, make_tables, set_stop_sc

pytestmark = pytest.mark.gpu

MAT = set_stop_sc(BLOSUM62, 23)
CODON = make_tables()[2]


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def test_gapless_golden(engine, gapless_golden):
    g, G = gapless_golden
    for k, c in enumerate(g["cases"]):
        w = G.case_inputs(k)
        assert {n: G.digest(w[n]) for n in G.INPUTS} == c["sha256"]
        got = engine.gapless_score(w, c["block_width"], c["kmer"], c["xdrop"], MAT, CODON)
        want = np.array(c["scores"], dtype=np.int32)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"case {k}: {bad.size} mismatches, first {bad[:5]} {got[bad[:5]]} vs {want[bad[:5]]}"


@pytest.mark.parametrize("seed,xdrop,kmer,bbit", [(31, 40, 6, 8), (32, 25, 5, 7), (33, 200, 6, 9), (34, 40, 3, 8)])
def test_gapless_sweep(engine, oracle, seed, xdrop, kmer, bbit):
    w = W.gapless_workload(60, 600_000, 4000, seed=seed, n_contigs=16, al=400, kmer=kmer, bbit=bbit,
                           anchors_per_cand=12)
    got = engine.gapless_score(w, 1 << bbit, kmer, xdrop, MAT, CODON)
    want = oracle.port_gapless(w, 1 << bbit, kmer, xdrop, MAT, CODON)
    assert (got == want).all(), np.nonzero(got != want)[0][:5]


def test_gapless_reference_entry_and_cache(oracle):
    """ns_gpu_gapless_score_batch: needs ns_gpu_init, caches the genome by pointer, counts work."""
    assert L.gpu_init(0)
    w = W.gapless_workload(30, 300_000, 2000, seed=41, n_contigs=8, al=300)
    want = oracle.port_gapless(w, 256, 6, 40, MAT, CODON)
    prof0 = np.zeros(4, dtype=np.uint64)
    L.load().ns_gpu_gapless_profile(prof0.ctypes.data)
    a = L.gapless_reference_entry(w, 256, 6, 40, MAT, CODON)
    b = L.gapless_reference_entry(w, 256, 6, 40, MAT, CODON)   # genome resident: same pointer and length
    w2 = dict(w, packed=w["packed"].copy())
    w2["packed"][:] = 0x44                                      # all N at a new address: re-uploaded
    c = L.gapless_reference_entry(w2, 256, 6, 40, MAT, CODON)
    assert (a == want).all() and (b == want).all()
    assert (c == oracle.port_gapless(w2, 256, 6, 40, MAT, CODON)).all()  # scored on the new genome, not the cached one
    assert (c != a).any()
    prof1 = np.zeros(4, dtype=np.uint64)
    L.load().ns_gpu_gapless_profile(prof1.ctypes.data)
    d = prof1 - prof0
    assert d[0] == 3 and d[1] == 3 * len(w["candidates"]) and d[3] == 3 * len(w["anchors"]) * 256
