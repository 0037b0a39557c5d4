"""The oracle is pinned before it is trusted (CPU only).

* The restatement (oracle/ns_port.c) reproduces every golden vector the
  reference produced (tests/golden/splice_golden.json): known answers of
  test/test_dp32.c and test/test_gpu.c, random and planted global DPs with
  and without a splice-score track, 16- and 32-bit widths, extensions.
* The reference's own assertions (test/test_dp32.c) hold for it.
* Where the reference build is present (oracle/_ref), a fresh seeded sweep
  is compared directly, and the scoring tables of protlocus_b200.abi equal
  the reference's.
"""
import ctypes as C

import numpy as np
import pytest

from protlocus_b200 import workload as W
from protlocus_b200.abi import (AA_I2C, BLOSUM62, NS_CIGAR_STR, NS_F_CIGAR, NS_F_EXT_LEFT, NS_F_EXT_RIGHT,
                                Options)

FN = {"ns_global_gs16b": "gs16b", "ns_global_gs32b": "gs32b", "ns_global_gs_auto": "gs_auto"}


def _golden_cases(golden, groups=None):
    for c in golden["cases"]:
        if groups is None or c["group"] in groups:
            yield c


def test_port_matches_golden(oracle, golden):
    avx2 = golden["host_avx2"]
    n = 0
    for c in _golden_cases(golden):
        opt = oracle.make_options(c["opt"])
        ss = bytes.fromhex(c["ss"]) if c["ss"] else None
        got = oracle.port_run(FN[c["fn"]], c["nt"].encode(), c["aa"].encode(), opt, ss, avx2=avx2)
        assert got == (c["score"], c["nt_len"], c["aa_len"], c["cigar"]), (c["group"], c["fn"], len(c["nt"]))
        n += 1
    assert n == len(golden["cases"]) and n > 400


def test_port_matches_ext_golden(oracle, ext_golden):
    """The restatement reproduces every extension golden vector of the reference (both stripe widths)."""
    for c in ext_golden["cases"]:
        opt = oracle.make_ext_options(c["opt"])
        ss = bytes.fromhex(c["ss"]) if c["ss"] else None
        got = oracle.port_run("gs16b", c["nt"].encode(), c["aa"].encode(), opt, ss, avx2=c["width"] == 16)
        assert got[:3] == (c["score"], c["nt_len"], c["aa_len"]), c


def test_port_matches_hmm_golden(oracle, hmm_golden):
    """The restatement of mp_hmm_dp_score reproduces every reference score of the HMM fixture."""
    import numpy as np
    from protlocus_b200 import hmm as H
    ca = H.codon_alpha()
    for p in hmm_golden["profiles"]:
        for r, s in zip(p["regions"], p["scores"]):
            nt = np.frombuffer(bytes.fromhex(r), dtype=np.uint8)
            assert oracle.port_hmm(p["m"], p["emit"], p["trans"], ca, nt) == s


def test_hmm_parser_matches_reference_tables(hmm_golden):
    """parse_hmmer3 gives the reference parser's int16 tables for the fixture's synthetic profiles."""
    import numpy as np
    from protlocus_b200 import hmm as H
    g = hmm_golden["synthetic"]
    texts, _ = H.synthetic_profiles(g["n"], seed=g["seed"], m_min=g["m_min"], m_max=g["m_max"])
    mine = H.parse_hmmer3("".join(texts))
    ref = [p for p in hmm_golden["profiles"] if p["source"].startswith("synthetic")]
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a["m"] == b["m"]
        assert (a["emit"].reshape(-1) == np.array(b["emit"], dtype=np.int16)).all()
        assert (a["trans"].reshape(-1) == np.array(b["trans"], dtype=np.int16)).all()


def test_port_matches_gapless_golden(oracle, gapless_golden):
    """The gapless restatement reproduces the reference CUDA kernel's scores on every fixture case
    (inputs regenerated from their seeds and checked against the recorded digests)."""
    import numpy as np
    from protlocus_b200.abi import BLOSUM62, make_tables, set_stop_sc
    g, G = gapless_golden
    _, _, codon = make_tables()
    mat = set_stop_sc(BLOSUM62, 23)
    for k, c in enumerate(g["cases"]):
        w = G.case_inputs(k)
        assert {n: G.digest(w[n]) for n in G.INPUTS} == c["sha256"], f"case {k}: inputs do not regenerate"
        got = oracle.port_gapless(w, c["block_width"], c["kmer"], c["xdrop"], mat, codon)
        assert (got == np.array(c["scores"], dtype=np.int32)).all(), k


def test_dp32_known_answers(oracle):
    """test/test_dp32.c assertions, on the restatement."""
    opt = Options.nasw_defaults(flag=NS_F_CIGAR, go=3, ge=1, io=100, fs=100, sp_model=0)
    a = oracle.port_run("gs16b", b"ATGAAAACTTGG", b"MKQTW", opt)
    b = oracle.port_run("gs32b", b"ATGAAAACTTGG", b"MKQTW", opt)
    assert a[0] == b[0] and a[3] == b[3]
    assert any((w & 0xf) == 1 for w in a[3])  # has an insertion
    ww = int(BLOSUM62[AA_I2C.index("W"), AA_I2C.index("W")])
    for flag in (NS_F_EXT_LEFT, NS_F_EXT_RIGHT):
        for n in (7, 19):
            o = Options.nasw_defaults(flag=flag)
            s, ntl, aal, _ = oracle.port_run("gs16b", b"TGG" * n, b"W" * n, o)
            assert s == n * ww + o.c.end_bonus and ntl == 3 * n and aal == n
    o = Options.nasw_defaults(flag=NS_F_CIGAR)
    s, _, _, cig = oracle.port_run("gs_auto", b"TGG" * 3000, b"W" * 3000, o)
    assert s == 3000 * ww and s > 32767
    assert cig == [3000 << 4 | NS_CIGAR_STR.index("M")]


@pytest.mark.skipif("not __import__('oracle_lib').ref_lib()", reason="reference build (oracle/_ref) absent")
def test_port_matches_reference_sweep(oracle):
    rng = np.random.default_rng(7)
    opt = Options(flag=NS_F_CIGAR)
    for q in range(400):
        nt, aa = W.random_pair(rng, max_al=80)
        ss = W.random_ss(rng, len(nt)) if q % 2 else None
        for fn in ("gs16b", "gs32b"):
            assert oracle.port_run(fn, nt, aa, opt, ss) == oracle.ref_run("ns_global_" + fn, nt, aa, opt, ss)
    for q in range(300):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 160)))
        o = Options(flag=NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT, xdrop=[100, 30, 10 ** 6][q % 3])
        assert oracle.port_run("gs16b", nt, aa, o) == oracle.ref_run("ns_global_gs16b", nt, aa, o)


@pytest.mark.skipif("not __import__('oracle_lib').ref_lib()", reason="reference build (oracle/_ref) absent")
def test_tables_equal_reference(oracle):
    ref = oracle.ref_lib()
    o = Options()
    for name, mine in (("ns_tab_nt4", o.nt4), ("ns_tab_aa20", o.aa20), ("ns_tab_codon", o.codon)):
        arr = (C.c_uint8 * len(mine)).in_dll(ref, name)
        assert bytes(arr) == mine.tobytes(), name
    m = (C.c_int8 * 484).in_dll(ref, "ns_mat_blosum62")
    assert np.array(m, dtype=np.int8).tobytes() == BLOSUM62.tobytes()


def test_workload_shapes():
    nt, aa = W.single_locus(seed=0)
    assert len(aa) == 500 and len(nt) == 20000
    jobs = W.batch_pairs(8, seed=3)
    assert len(jobs) == 16
    for (a, p), (b, q) in zip(jobs[0::2], jobs[1::2]):
        assert b == W.revcomp(a) and p == q
        assert 50 <= len(p) <= 2500 and 1000 <= len(a)
