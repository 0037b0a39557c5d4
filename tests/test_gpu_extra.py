"""Alignment statistics and exon features from the CIGAR on the device (extra.cu)
against the reference's own mp_extra_cal (align.c:148-269), compiled from its
sources behind oracle/ref_extra.c.

Alignments are the exact global DP's (the oracle's CIGARs are the reference's) over
planted spliced genes on both strands, random pairs, windows with N bases and
planted stop codons, with and without position-specific scores, the stop-codon
feature, and CIGARs whose span does not match the region.
"""
import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import BLOSUM62, NS_F_CIGAR, Options, make_tables

need_ref = pytest.mark.skipif(O.extra_lib() is None, reason="oracle/_ref/libextra_ref.so not built")
NT4, AA20, CODON = make_tables()
GO, GE, FS = 11, 1, 23
MAT = np.asarray(BLOSUM62, dtype=np.int8).reshape(-1)


def _alignments(seed, n_planted=12, n_random=40):
    rng = np.random.default_rng(seed)
    opt = Options(flag=NS_F_CIGAR)
    out = []
    pairs = []
    for q in range(n_planted):
        nt, aa = W.single_locus(seed=seed * 100 + q, al=int(rng.integers(60, 300)), window=int(rng.integers(1500, 5000)),
                                n_intron=int(rng.integers(0, 4)), n_frameshift=int(rng.integers(0, 3)))
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    pairs += [W.random_pair(rng, max_al=60, n_rate=0.03) for _ in range(n_random)]
    for nt, aa in pairs:
        score, ntl, aal, cig = O.run("gs_auto", nt, aa, opt)
        nt4 = NT4[np.frombuffer(nt, np.uint8)]
        out.append({"cigar": list(cig), "nt4": nt4, "aa": aa, "vs": 0, "ve": len(nt), "qs": 0, "qe": len(aa),
                    "has_stop": bool(rng.random() < 0.3)})
    return out, rng


def _compare(alns, got):
    for a, (res, feats) in zip(alns, got):
        stats, want = O.ref_extra(a["cigar"], a["nt4"], a["aa"], a["vs"], a["ve"], a["qs"], a["qe"], a["has_stop"],
                                  GO, GE, FS, MAT, a.get("pssm"))
        assert res.ok == stats[8], (res.ok, stats)
        if not stats[8]:
            continue
        mine = [res.blen, res.n_iden, res.n_plus, res.n_fs, res.n_stop, res.dp_max, res.n_exon, res.n_feat]
        assert mine == stats[:8], (mine, stats)
        assert len(feats) == len(want)
        for f, g in zip(feats, want):
            for k in ("vs", "ve", "qs", "qe", "type", "phase", "n_fs", "n_stop", "score", "n_iden", "blen"):
                assert getattr(f, k) == getattr(g, k), (k, getattr(f, k), getattr(g, k))
            assert bytes(f.donor) == bytes(g.donor) and bytes(f.acceptor) == bytes(g.acceptor)


@need_ref
def test_reference_extra_hand_case():
    """The reference wrapper on a 3-codon match: ATG AAA CCC against MKP."""
    stats, feats = O.ref_extra([3 << 4], NT4[np.frombuffer(b"ATGAAACCC", np.uint8)], b"MKP", 0, 9, 0, 3, False,
                               GO, GE, FS, MAT)
    s_m, s_k, s_p = (int(BLOSUM62[i][i]) for i in (12, 11, 14))  # ARNDCQEGHILKMFPSTWYV: M 12, K 11, P 14
    assert stats == [9, 3, 3, 0, 0, s_m + s_k + s_p, 1, 1, 1]
    assert (feats[0].vs, feats[0].ve, feats[0].qs, feats[0].qe, feats[0].blen) == (0, 9, 0, 3, 9)


@pytest.mark.gpu
@need_ref
def test_extra_matches_reference():
    alns, rng = _alignments(7)
    # planted in-frame stops and N runs inside a few windows (the CIGARs stay as the DP made them)
    for a in alns[:6]:
        nt4 = a["nt4"].copy()
        for p in rng.integers(0, len(nt4) - 3, size=3):
            nt4[p: p + 3] = (3, 0, 0)  # TAA
        nt4[rng.integers(0, len(nt4))] = 4
        a["nt4"] = nt4
    eng = L.Engine(0)
    try:
        _compare(alns, eng.extra_cal(alns, GO, GE, FS, MAT, CODON, AA20))
    finally:
        eng.close()


@pytest.mark.gpu
@need_ref
def test_extra_pssm_and_span_mismatch():
    alns, rng = _alignments(8, n_planted=6, n_random=20)
    for a in alns[::2]:
        a["pssm"] = rng.integers(-6, 10, size=(a["qe"] - a["qs"], 22)).astype(np.int8)
    # sub-regions: the same CIGAR against a shorter region span (the reference drops the features)
    for a in alns[1::5]:
        a["ve"] = a["ve"] - 1
    eng = L.Engine(0)
    try:
        _compare(alns, eng.extra_cal(alns, GO, GE, FS, MAT, CODON, AA20))
    finally:
        eng.close()


@pytest.mark.gpu
def test_extra_device_entry_equals_host_entry():
    """pl_extra_cal_device on device-resident buffers gives the host entry point's records."""
    import ctypes as C
    from protlocus_b200.abi import ExtraResult, Feat
    alns, rng = _alignments(9, n_planted=6, n_random=20)
    for a in alns[::3]:
        a["pssm"] = rng.integers(-6, 10, size=(a["qe"] - a["qs"], 22)).astype(np.int8)
    eng = L.Engine(0)
    try:
        pk = eng.extra_run(eng.extra_pack(alns), GO, GE, FS, MAT, CODON, AA20)
        d = eng.extra_upload(pk)
        eng.extra_run_device(pk, d, GO, GE, FS, MAT, CODON, AA20)
        res = (ExtraResult * max(pk["n"], 1)).from_buffer_copy(d["res"].cpu().numpy().tobytes())
        feats = (Feat * max(pk["n_feat"], 1)).from_buffer_copy(d["feats"].cpu().numpy().tobytes())
        assert bytes(res)[: C.sizeof(ExtraResult) * pk["n"]] == bytes(pk["res"])[: C.sizeof(ExtraResult) * pk["n"]]
        for q in range(pk["n"]):
            J, r = pk["jobs"][q], pk["res"][q]
            for k in range(min(r.n_feat, J.feat_cap)):  # field by field: the struct's tail padding is not written
                f, g = feats[J.feat_off + k], pk["feats"][J.feat_off + k]
                assert [bytes(getattr(f, m)) if m in ("donor", "acceptor") else getattr(f, m) for m, _ in Feat._fields_] \
                    == [bytes(getattr(g, m)) if m in ("donor", "acceptor") else getattr(g, m) for m, _ in Feat._fields_], \
                    (q, k)
    finally:
        eng.close()
