"""Host logic of the learned prefilter on the CPU: the candidate generator's shapes,
the CIGAR span rule that makes the training targets, window tightening, the
decision thresholds, the shipped model file, and the feature restatement on a
hand-built case."""
import numpy as np
import pytest

from protlocus_b200 import prefilter as P
from protlocus_b200.abi import SpliceResult, make_tables


def _res(counts):
    out = np.zeros(len(counts), P.RES_DTYPE)
    out["n_cigar"] = counts
    out["cigar_off"] = np.concatenate([[0], np.cumsum(counts)[:-1]])
    return out


def test_result_record_matches_the_c_struct():
    import ctypes as C
    assert P.RES_DTYPE.itemsize == C.sizeof(SpliceResult)
    for name, _ in SpliceResult._fields_:
        assert P.RES_DTYPE.fields[name][1] == getattr(SpliceResult, name).offset


OPS = {"M": 0, "I": 1, "D": 2, "N": 3, "F": 10, "G": 11, "U": 12, "V": 13}  # nasw.h:33-41


def w(n, op):
    return (n << 4) | OPS[op]


def test_candidate_shapes():
    c = P.make_candidates(5, n_prot=16)
    j = c["jobs"]
    assert len(j) == 16 * 8 and (c["kind"][::8] == P.KIND_OWN_PLUS).all()
    assert (j["nl"] >= 3).all() and (j["nt_off"] + j["nl"] <= len(c["nt"])).all()
    assert (j["aa_off"] + j["al"] <= len(c["aa"])).all()
    # the own window on both strands: the minus copy is the reverse complement
    a = c["nt"][j["nt_off"][0]: j["nt_off"][0] + j["nl"][0]].tobytes()
    b = c["nt"][j["nt_off"][1]: j["nt_off"][1] + j["nl"][1]].tobytes()
    assert b == a[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    # deterministic per seed
    assert np.array_equal(P.make_candidates(5, n_prot=16)["jobs"], j)


def test_cigar_bounds_skip_short_terminal_runs():
    # 1M 692U 2D 55M 336V 320M 2356N 2M : the core is 55M..320M
    cig = np.array([w(1, "M"), w(692, "U"), w(2, "D"), w(55, "M"), w(336, "V"), w(320, "M"), w(2356, "N"), w(2, "M"),
                    w(12, "M"), w(3, "I"), w(40, "M")], np.uint32)
    s, e = P.cigar_bounds(cig, _res([8, 3]))
    assert s[0] == 3 + 692 + 6 and e[0] == 3 + 692 + 6 + 165 + 336 + 960
    assert s[1] == 0 and e[1] == 36 + 120


def test_tightened_windows():
    cand = {"jobs": np.zeros(3, P.JOB_DTYPE)}
    cand["jobs"]["nt_off"] = [0, 1000, 5000]
    cand["jobs"]["nl"] = [1000, 4000, 10]
    cand["jobs"]["al"] = [100, 200, 3]
    pipe = P.Pipeline.__new__(P.Pipeline)
    pipe.cand = cand
    out = np.array([[5.0, 0.2, 0.5], [5.0, 0.9, 0.1], [5.0, 0.4, 0.5]], np.float32)
    chain = np.array([[400, 600, 10, 50], [-1, -1, -1, -1], [-1, -1, -1, -1]], np.int32)
    jobs = pipe.tightened(np.arange(3), out, chain, 50)
    # union of [200, 500] and the chain's implied [400 - 32, 600 + 3*49 + 1] plus 50 each side
    assert jobs["nt_off"][0] == 150 and jobs["nl"][0] == 748 + 50 - 150
    # swapped prediction is ordered; 400..3600 plus 50
    assert jobs["nt_off"][1] == 1000 + 350 and jobs["nl"][1] == 3650 - 350
    # a window shorter than 3 nt after cutting keeps the full window
    assert jobs["nt_off"][2] == 5000 + 0 or jobs["nl"][2] >= 3


def test_logit_edges():
    assert P._logit(0.0) == -np.inf and P._logit(1.0) == np.inf
    assert abs(P._logit(0.5)) < 1e-12


def test_shipped_model_file():
    z = np.load(P.__file__.replace("prefilter.py", "data/prefilter.npz"))
    n = 256 * 576 + 256 + 2 * (256 * 256 + 256) + 16 * 256 + 16
    assert z["params"].shape == (n,) and np.isfinite(z["params"]).all()
    assert 0.0 < float(z["tau"]) < 1.0 and 0.0 < float(z["tau_fb"]) <= 1.0 and int(z["margin"]) >= 0


def test_feature_restatement_hand_case():
    import sys
    import os
    sys.path.insert(0, os.path.dirname(__file__))
    import pf_ref
    nt4, aa20, codon = make_tables()
    prot = b"MKVLAWHEPQ"
    # codons of MKVLAWHEPQ followed by the same protein again 30 nt later
    cds = b"ATGAAAGTTCTTGCTTGGCATGAACCTCAA"
    win = b"CC" + cds + b"T" * 30 + cds
    F, chain, na, length = pf_ref.features(win, prot, nt4, aa20, codon)
    # every 5-mer of the protein occurs twice in frame: 6 + 6 anchors, one chain of 6
    assert na == 12 and length == 6
    assert chain == [2 + 14, 2 + 29, 4, 9]
    assert F[512 + 17] == 1.0 and F[512 + 18] == 1.0


def test_query_span_counts_residues_like_extra_cal():
    # 2I 5M 300N 3G... residues: I 2, M 5, N 0, G 1, U 1 (split codon), M 4
    cig = np.array([w(2, "I"), w(5, "M"), w(300, "N"), w(4, "G"), w(80, "U"), w(4, "M"), w(6, "D"),
                    w(3, "I"), w(1, "M")], np.uint32)
    qs, qe = P.query_span(cig, _res([7, 2]))
    assert qs[0] == 2 and qe[0] == 2 + 5 + 1 + 1 + 4
    assert qs[1] == 3 and qe[1] == 4          # 3I 1M
    qs, qe = P.query_span(np.array([w(4, "I")], np.uint32), _res([1]))
    assert qs[0] == 0 and qe[0] == 0          # no codon match: empty span


def test_output_set_follows_the_reference_rule():
    # protein 0: best 1000; 995 >= 0.99*1000 passes, 986 does not; protein 1: all scores <= 0
    score = np.array([1000, 995, 986, 0, -5, -1], np.int32)
    prot = np.array([0, 0, 0, 0, 1, 1])
    qlen = np.array([100] * 6)
    qs = np.zeros(6, np.int64)
    qe = np.array([100, 100, 100, 100, 100, 100])
    out = P.output_set(score, qs, qe, prot, qlen)
    assert out.tolist() == [True, True, False, False, False, False]
    # a short aligned span fails out_cov (< 0.1 x 100 residues)
    qe2 = qe.copy()
    qe2[1] = 9
    assert P.output_set(score, qs, qe2, prot, qlen).tolist()[:2] == [True, False]
    # a candidate without a result neither passes nor sets the best score (986 >= 0.99*995)
    aligned = np.array([False, True, True, True, True, True])
    out = P.output_set(score, qs, qe, prot, qlen, aligned)
    assert out.tolist()[:3] == [False, True, True]
    # out_n limits the ranks examined
    assert P.output_set(score, qs, qe, prot, qlen, out_n=1).tolist()[:2] == [True, False]


def test_loci_reported_needs_a_candidate_on_the_gene():
    kind = np.array([P.KIND_OWN_PLUS, P.KIND_OWN_MINUS, P.KIND_PARTIAL, P.KIND_OTHER] * 2, np.int8)
    prot = np.repeat([0, 1], 4)
    out = np.array([False, False, True, False, False, False, False, True])
    assert P.loci_reported(out, prot, kind, 2).tolist() == [True, False]


def test_decision_thresholds_in_c():
    """pl_pf_decide keeps logit >= logit(tau) and marks fallback at logit >= logit(tau_fb)."""
    from protlocus_b200 import lib as L
    jobs = np.zeros(4, P.JOB_DTYPE)
    jobs["nt_off"] = [0, 100, 200, 300]
    jobs["nl"] = [90, 90, 90, 90]
    jobs["al"] = [10, 10, 10, 10]
    z = np.array([P._logit(0.2) - 1e-3, P._logit(0.2), P._logit(0.9), 5.0], np.float32)
    out = np.zeros((4, 3), np.float32)
    out[:, 0], out[:, 1], out[:, 2] = z, 0.1, 0.9
    keep = np.zeros(4, np.uint8)
    fb = np.zeros(4, np.uint8)
    tight = np.zeros(4, P.JOB_DTYPE)
    assert L.load().pl_pf_decide(4, jobs.ctypes.data, out.ctypes.data, 3, None, 0.2, 5, 0.0, 0.9, keep.ctypes.data,
                                 fb.ctypes.data, tight.ctypes.data)
    # float32 rounding of the logits decides the borderline case exactly as the comparison in C does
    assert keep.tolist() == [int(np.float64(x) >= P._logit(0.2)) for x in z]
    assert fb.tolist() == [int(np.float64(x) >= P._logit(0.9)) for x in z]
    assert tight["nt_off"][3] == 300 + 4 and tight["nl"][3] == 81 + 5 - 4   # [9 - 5, 81 + 5] of 90
    assert tight["nt_off"][0] == 0 and tight["nl"][0] == 90                 # dropped: copied unchanged
