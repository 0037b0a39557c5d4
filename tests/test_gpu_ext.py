"""GPU parity of the batched extension DP (ns_global_gs16b with NS_F_EXT_LEFT /
NS_F_EXT_RIGHT: nt_len, aa_len, score, bit-exact) against the reference's
golden vectors and the oracle restatement.

The reference's own coverage is test/test_gpu.c:294-386 (a 42-request sweep
compared with ns_global_gs16b) and test/test_dp32.c:33-54; these tests add
both stripe widths, position-specific scores, splice-score tracks, long
windows that the x-drop cuts short, int16 saturation, the wide row-key
variant, and the batch object with several flushes in flight and threads.
"""
import threading

import numpy as np
import pytest

from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import NS_F_EXT_LEFT, NS_F_EXT_RIGHT, Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def _oracle(oracle, r, opt):
    o = opt.with_flag(r.get("flag", 0))
    if r.get("pssm") is not None:
        o = o.with_pssm(r["pssm"])
    s, ntl, aal, _ = oracle.port_run("gs16b", r["nt"], r["aa"], o, r.get("ss"), avx2=r.get("width", 8) == 16)
    return s, ntl, aal


def _check(engine, oracle, opt, reqs):
    got = engine.ext_host(opt, reqs)
    bad = [(q, len(r["nt"]), len(r["aa"]), g, _oracle(oracle, r, opt)) for q, (r, g) in enumerate(zip(reqs, got))
           if g != _oracle(oracle, r, opt)]
    assert not bad, f"{len(bad)} of {len(reqs)} mismatches, first: {bad[:4]}"


def test_ext_golden(engine, oracle, ext_golden):
    """Every extension golden vector of the reference (both stripe widths), one batch per option set."""
    groups = {}
    for c in ext_golden["cases"]:
        spec = dict(c["opt"])
        spec.pop("flag", None)
        groups.setdefault(repr(sorted(spec.items())), []).append(c)
    n = 0
    for cases in groups.values():
        opt = oracle.make_ext_options(cases[0]["opt"])
        reqs = []
        for c in cases:
            r = {"nt": c["nt"].encode(), "aa": c["aa"].encode(), "flag": c["opt"].get("flag", 0), "width": c["width"]}
            if c["ss"]:
                r["ss"] = bytes.fromhex(c["ss"])
            if c["opt"].get("pssm_seed") is not None:
                r["pssm"] = np.frombuffer(bytes(oracle.make_ext_options(c["opt"]).pssm_arr), dtype=np.int8)
            reqs.append(r)
        got = engine.ext_host(opt.with_pssm(None), reqs)
        for c, g in zip(cases, got):
            assert g == (c["score"], c["nt_len"], c["aa_len"]), (c["group"], c["width"], g, c)
        n += len(cases)
    assert n == len(ext_golden["cases"])


def test_ext_random_sweep(engine, oracle):
    """Seeded random requests: both orientations, both widths, ss tracks, pssm, x-drop settings."""
    rng = np.random.default_rng(11)
    for xdrop, eb, io in ((100, 5, 29), (30, 0, 20), (10 ** 6, -3, 29)):
        opt = Options(xdrop=xdrop, end_bonus=eb, io=io)
        reqs = []
        for q in range(150):
            nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 200)))
            r = {"nt": nt, "aa": aa, "flag": NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT,
                 "width": 16 if (q >> 1) & 1 else 8}
            if q % 5 == 2:
                r["ss"] = W.random_ss(rng, len(nt))
            if q % 7 == 3:
                r["pssm"] = rng.integers(-6, 10, size=(len(aa), 22)).astype(np.int8)
            reqs.append(r)
        _check(engine, oracle, opt, reqs)


def test_ext_long_windows(engine, oracle):
    """Genes with long trailing windows: many 256-row strips; the x-drop ends most DPs early."""
    reqs = []
    for q in range(24):
        al = 60 + 37 * q
        nt, aa = W.single_locus(seed=300 + q, al=al, window=3 * al + 500 + 211 * q, n_intron=q % 3)
        if q % 4 == 3:
            nt = W.revcomp(nt)
        reqs.append({"nt": nt, "aa": aa, "flag": NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT,
                     "width": 16 if q % 3 else 8})
    for xdrop in (100, 30, 10 ** 6):
        _check(engine, oracle, Options(xdrop=xdrop), reqs)


def test_ext_wide_keys(engine, oracle):
    """The int64 row-key variant: an end bonus outside the narrow key range, and al > 16384."""
    rng = np.random.default_rng(5)
    reqs = []
    for q in range(40):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 90)))
        reqs.append({"nt": nt, "aa": aa, "flag": NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT, "width": 16 if q & 2 else 8})
    _check(engine, oracle, Options(end_bonus=70000), reqs)
    _check(engine, oracle, Options(end_bonus=-40000), reqs)
    aa = bytes(rng.choice(list(b"ACDEFGHIKLMNPQRSTVWY"), size=16500))
    nt = bytes(rng.choice(list(b"ACGT"), size=70))
    _check(engine, oracle, Options(), [{"nt": nt, "aa": aa, "flag": NS_F_EXT_RIGHT, "width": 16},
                                       {"nt": nt, "aa": aa, "flag": NS_F_EXT_LEFT, "width": 8}])


def test_ext_default_width(engine, oracle):
    """width 0 takes pl_ext_stripe_width(), the host rule of nasw-sse.c:744-750."""
    rng = np.random.default_rng(8)
    opt = Options()
    reqs = []
    for q in range(30):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 60)))
        reqs.append({"nt": nt, "aa": aa, "flag": NS_F_EXT_RIGHT})
    got = engine.ext_host(opt, reqs)
    for r, g in zip(reqs, got):
        r["width"] = L.ext_stripe_width(opt.with_flag(NS_F_EXT_RIGHT), len(r["aa"]))
        assert g == _oracle(oracle, r, opt)


def _batch_reqs(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 120)))
        out.append((nt, aa, NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT, W.random_ss(rng, len(nt)) if q % 3 == 0 else None))
    return out


def _want(oracle, opt, nt, aa, flag, ss):
    r = {"nt": nt, "aa": aa, "flag": flag, "ss": ss, "width": L.ext_stripe_width(opt.with_flag(flag), len(aa))}
    return _oracle(oracle, r, opt)


def test_ext_batch_object(oracle):
    """ns_ext_batch_*: several flushes in flight, ready/wait polling, results fetched out of order."""
    opt = Options()
    launches0, reqs0 = L.load().ns_ext_gpu_launch_count(), L.load().ns_ext_gpu_request_count()
    b = L.ExtBatch()
    flushes = []
    for g in range(4):
        reqs = _batch_reqs(100 + g, 30 + 10 * g)
        ids = [b.add(nt, aa, opt.with_flag(flag), ss) for nt, aa, flag, ss in reqs]
        assert b.flush() == len(reqs)
        flushes.append((ids, reqs))
    assert b.flush() == 0
    for ids, reqs in reversed(flushes):
        while not b.ready(ids[-1]):
            b.wait()
        for rid, (nt, aa, flag, ss) in reversed(list(zip(ids, reqs))):
            assert b.get(rid) == _want(oracle, opt, nt, aa, flag, ss)
    b.close()
    assert L.load().ns_ext_gpu_request_count() - reqs0 == sum(len(nt) >= 3 for _, r in flushes for nt, _, _, _ in r)
    assert L.load().ns_ext_gpu_launch_count() > launches0


def test_ext_batch_threads(oracle):
    """One batch object per thread (as align.c's mapping threads do), sharing the executor."""
    opt = Options()
    errors = []

    def worker(t):
        try:
            b = L.ExtBatch()
            for g in range(3):
                reqs = _batch_reqs(1000 + 10 * t + g, 25)
                ids = [b.add(nt, aa, opt.with_flag(flag), ss) for nt, aa, flag, ss in reqs]
                b.flush()
                for rid, (nt, aa, flag, ss) in zip(ids, reqs):
                    got, want = b.get(rid), _want(oracle, opt, nt, aa, flag, ss)
                    if got != want:
                        errors.append((t, g, rid, got, want))
            b.close()
        except Exception as e:  # noqa: BLE001
            errors.append((t, repr(e)))

    th = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert not errors, errors[:3]
