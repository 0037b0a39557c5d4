"""GPU parity of the global spliced DP (score + CIGAR, bit-exact) against the oracle.

Cases follow the reference's own GPU tests (test/test_gpu.c:51-219) and add
seeded sweeps that the reference's tests lack: random pairs with and without
a splice-score track, planted loci on both strands, the 32-bit width,
saturation at -32768, cooperative (whole-CTA) jobs and multi-wave batches.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import AA_I2C, BLOSUM62, NS_F_CIGAR, NS_F_EXT_LEFT, NS_F_EXT_RIGHT, NsRst, Options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def queue_ready():
    assert L.gpu_init(0), L.load().ns_gpu_error()


def _check(engine, oracle, opt, pairs, ss=None, fn="gs_auto"):
    got = engine.align_host(opt, pairs, ss)
    bad = []
    for q, ((nt, aa), (score, cig, _mode)) in enumerate(zip(pairs, got)):
        want = oracle.run(fn, nt, aa, opt, ss[q] if ss else None)
        if (score, cig) != (want[0], want[3]):
            bad.append((q, len(nt), len(aa), score, want[0]))
    assert not bad, f"{len(bad)} mismatches, first: {bad[:5]}"
    return got


def test_golden_vectors(engine, oracle, golden):
    """Every global-DP golden vector produced by the reference, run through the bulk path."""
    _golden(engine, oracle, golden)


def _golden(engine, oracle, golden):
    by_opt = {}
    for c in golden["cases"]:
        if c["opt"].get("flag", NS_F_CIGAR) & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT):
            continue  # extension DPs have their own entry point
        opt = oracle.make_options(c["opt"])
        wide = oracle.port_lib().port_needs_wide(opt.ptr, len(c["aa"]))
        if c["fn"] == "ns_global_gs32b" and not wide:
            continue  # the bulk path picks the width by ns_global_gs_auto's rule
        if c["fn"] == "ns_global_gs16b" and wide:
            continue
        by_opt.setdefault(repr(sorted(c["opt"].items())), []).append(c)
    n = 0
    for cases in by_opt.values():
        opt = oracle.make_options(cases[0]["opt"])
        pairs = [(c["nt"].encode(), c["aa"].encode()) for c in cases]
        ss = [bytes.fromhex(c["ss"]) if c["ss"] else None for c in cases]
        got = engine.align_host(opt, pairs, ss if any(s is not None for s in ss) else None)
        for c, (score, cig, _m) in zip(cases, got):
            assert (score, cig) == (c["score"], c["cigar"]), (c["group"], c["fn"], len(c["nt"]), len(c["aa"]),
                                                              score, c["score"])
            n += 1
    assert n >= 250


def test_random_sweep(engine, oracle):
    rng = np.random.default_rng(11)
    pairs = [W.random_pair(rng, max_al=60) for _ in range(1500)]
    ss = [W.random_ss(rng, len(nt)) if q % 3 == 0 else None for q, (nt, _) in enumerate(pairs)]
    _check(engine, oracle, Options(flag=NS_F_CIGAR), pairs, ss)


def test_planted_both_strands(engine, oracle):
    rng = np.random.default_rng(12)
    pairs = []
    for q in range(40):
        al = int(rng.integers(40, 700))
        nt, aa = W.single_locus(seed=500 + q, al=al, window=int(rng.integers(3 * al + 100, 3 * al + 9000)),
                                n_intron=int(rng.integers(0, 5)), n_frameshift=int(rng.integers(0, 3)))
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    _check(engine, oracle, Options(flag=NS_F_CIGAR), pairs)


def test_nasw_default_options(engine, oracle):
    """ns_opt_init() scoring (fs=17, MAMMAL splice model, plain BLOSUM62)."""
    rng = np.random.default_rng(13)
    pairs = [W.random_pair(rng, max_al=50) for _ in range(400)]
    _check(engine, oracle, Options.nasw_defaults(flag=NS_F_CIGAR), pairs)


def test_saturation_at_int16_floor(engine, oracle):
    """Penalties large enough that cells saturate at -32768 (_mm_subs_epi16)."""
    rng = np.random.default_rng(14)
    opt = Options(flag=NS_F_CIGAR, go=3000, ge=200, io=9000, fs=5000, stop_pen=23)
    pairs = [W.random_pair(rng, max_al=40) for _ in range(300)]
    _check(engine, oracle, opt, pairs)


def test_upper_clamp_mode(engine, oracle):
    """al*max(sc) near +32767 with a negative end bonus: both int16 clamps are live."""
    rng = np.random.default_rng(15)
    m = BLOSUM62.copy()
    w = AA_I2C.index("W")
    m[w, w] = 110
    opt = Options(flag=NS_F_CIGAR, matrix=m, end_bonus=-6000)
    pairs = []
    for _ in range(12):
        al = int(rng.integers(296, 320))
        aa = rng.choice(list(b"WWWWWACDEFG"), size=al).astype(np.uint8).tobytes()
        nt = W.random_dna(rng, int(rng.integers(3 * al, 3 * al + 400))).encode()
        pairs.append((nt, aa))
    got = _check(engine, oracle, opt, pairs)
    widths = [w for _, _, w in got]
    assert widths == [16] * len(pairs), widths


def test_wide_width(engine, oracle):
    """ns_global_gs_auto's 32-bit route (al*max(sc)+end_bonus > 30000), test_gpu.c:91-124 shape."""
    rng = np.random.default_rng(16)
    m = BLOSUM62.copy()
    w = AA_I2C.index("W")
    m[w, w] = 127
    opt = Options.nasw_defaults(flag=NS_F_CIGAR, matrix=m)
    pairs = [(b"TGG" * 300, b"W" * 300)]
    for _ in range(40):
        al = int(rng.integers(240, 420))
        nt, aa = W.single_locus(seed=int(rng.integers(1 << 30)), al=al, window=3 * al + int(rng.integers(50, 2000)))
        pairs.append((nt, aa))
    got = _check(engine, oracle, opt, pairs)
    widths = [w for _, _, w in got]
    assert widths == [32] * len(pairs), widths


def test_cooperative_jobs_and_waves(oracle):
    """Large jobs run by a whole CTA, and a trace budget small enough to force several waves."""
    e = L.Engine(0, trace_budget_bytes=96 << 20)
    try:
        rng = np.random.default_rng(17)
        pairs = []
        for q in range(6):
            al = int(rng.integers(220, 500))
            nt, aa = W.single_locus(seed=900 + q, al=al, window=int(rng.integers(9000, 16000)), n_intron=3)
            pairs += [(nt, aa), (W.revcomp(nt), aa)]
        pairs += [W.random_pair(rng, max_al=60) for _ in range(200)]
        _check(e, oracle, Options(flag=NS_F_CIGAR), pairs)
        plan = e.last_plan()
        assert plan["coop"] > 0 and plan["waves"] > 1, plan
    finally:
        e.close()


@pytest.mark.parametrize("r4_rows,ratio", [(1 << 30, 0.7), (1 << 30, 0.05), (3000, 0.3)])
def test_four_rows_per_lane(oracle, golden, r4_rows, ratio):
    """Jobs on the 4-rows-per-lane kernels (all of them, or those up to 3000 rows beside
    8-row ones), solo and cooperative, over golden vectors, planted loci and a forced
    multi-wave plan."""
    e = L.Engine(0, trace_budget_bytes=64 << 20)
    try:
        e.set_tuning(r4_rows, ratio)
        assert e.tuning()["r4_rows"] == r4_rows
        rng = np.random.default_rng(31)
        pairs = []
        for q in range(8):
            al = int(rng.integers(200, 480))
            nt, aa = W.single_locus(seed=1300 + q, al=al, window=int(rng.integers(2500, 12000)), n_intron=3)
            pairs += [(nt, aa), (W.revcomp(nt), aa)]
        pairs += [W.random_pair(rng, max_al=60) for _ in range(150)]
        _check(e, oracle, Options(flag=NS_F_CIGAR), pairs)
        plan = e.last_plan()
        assert plan["coop"] > 0, plan
        _golden(e, oracle, golden)
    finally:
        e.close()


def test_autotune_picks_a_grid_point(oracle):
    """The autotuner runs the batch under its grid, keeps a point of it on the engine,
    and the batch still comes out bit-exact under the kept tuning."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    from protlocus_b200.abi import SpliceJob
    rng = np.random.default_rng(41)
    pairs = []
    for q in range(10):
        al = int(rng.integers(200, 420))
        nt, aa = W.single_locus(seed=1500 + q, al=al, window=int(rng.integers(1500, 9000)), n_intron=2)
        pairs.append((nt, aa))
    pairs += [W.random_pair(rng, max_al=60) for _ in range(100)]
    n = len(pairs)
    tab = (SpliceJob * n)()
    nt_off = aa_off = 0
    for q, (nt, aa) in enumerate(pairs):
        tab[q].nt_off, tab[q].aa_off, tab[q].ss_off, tab[q].nl, tab[q].al = nt_off, aa_off, -1, len(nt), len(aa)
        nt_off += len(nt)
        aa_off += len(aa)
    d_nt = torch.from_numpy(np.frombuffer(b"".join(p[0] for p in pairs), np.uint8).copy()).cuda()
    d_aa = torch.from_numpy(np.frombuffer(b"".join(p[1] for p in pairs), np.uint8).copy()).cuda()
    e = L.Engine(0)
    try:
        opt = Options(flag=NS_F_CIGAR)
        r4, ratio = C.c_int32(), C.c_double()
        assert e.lib.pl_engine_autotune(e.h, opt.ptr, tab, n, d_nt.data_ptr(), d_aa.data_ptr(), None, C.byref(r4),
                                        C.byref(ratio)), L.error()
        assert r4.value in (0, 1536, 3072, 6144, 12288) and ratio.value in (0.5, 0.7, 1.0)
        assert e.tuning() == {"r4_rows": r4.value, "coop_ratio": ratio.value}
        _check(e, oracle, opt, pairs)
    finally:
        e.close()


def test_device_entry_point(oracle):
    """pl_splice_batch_device with device-resident inputs and outputs."""
    torch = pytest.importorskip("torch")
    from protlocus_b200.abi import SpliceJob, SpliceResult
    rng = np.random.default_rng(18)
    pairs = [W.random_pair(rng, max_al=80) for _ in range(300)]
    opt = Options(flag=NS_F_CIGAR)
    n = len(pairs)
    jobs = (SpliceJob * n)()
    pos_nt = pos_aa = 0
    for q, (nt, aa) in enumerate(pairs):
        jobs[q].nt_off, jobs[q].aa_off, jobs[q].ss_off, jobs[q].nl, jobs[q].al = pos_nt, pos_aa, -1, len(nt), len(aa)
        pos_nt += len(nt)
        pos_aa += len(aa)
    d_nt = torch.tensor(np.frombuffer(b"".join(p[0] for p in pairs), dtype=np.uint8), device="cuda")
    d_aa = torch.tensor(np.frombuffer(b"".join(p[1] for p in pairs), dtype=np.uint8), device="cuda")
    cap = sum(len(a) + len(b) + 8 for a, b in pairs)
    d_res = torch.zeros(n * C.sizeof(SpliceResult), dtype=torch.uint8, device="cuda")
    d_cig = torch.zeros(cap, dtype=torch.int32, device="cuda")
    e = L.Engine(0)
    total = C.c_int64()
    ok = e.lib.pl_splice_batch_device(e.h, opt.ptr, jobs, n, d_nt.data_ptr(), d_aa.data_ptr(), None,
                                      d_res.data_ptr(), d_cig.data_ptr(), cap, C.byref(total),
                                      torch.cuda.current_stream().cuda_stream)
    assert ok, L.error()
    res = (SpliceResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
    cig = d_cig.cpu().numpy().view(np.uint32)
    assert total.value == sum(r.n_cigar for r in res)
    for q, (nt, aa) in enumerate(pairs):
        want = oracle.run("gs_auto", nt, aa, opt)
        r = res[q]
        assert r.status == 0 and r.score == want[0]
        assert cig[r.cigar_off:r.cigar_off + r.n_cigar].tolist() == want[3]
    e.close()


# ---------------------------------------------------------------- request queue API (test_gpu.c)

def test_queue_tile_boundaries(queue_ready, oracle):
    """test_gpu.c:51-89."""
    opt = Options.nasw_defaults(flag=NS_F_CIGAR)
    for nl, al in ((3, 1), (9, 3), (12, 4), (15, 5), (18, 6), (21, 7), (24, 8), (27, 9), (45, 15), (48, 16), (51, 17)):
        nt, aa = (b"TGG" * 20)[:nl], b"W" * al
        ok, score, ntl, aal, cig = L.gpu_global(nt, aa, opt)
        assert ok, L.load().ns_gpu_error()
        want = oracle.run("gs16b", nt, aa, opt)
        assert (score, ntl, aal, cig) == want


def test_queue_wide_not_dispatched(queue_ready):
    """test_gpu.c:91-124: the 32-bit route is not taken by the request queue."""
    lib = L.load()
    m = BLOSUM62.copy()
    w = AA_I2C.index("W")
    m[w, w] = 127
    opt = Options.nasw_defaults(flag=NS_F_CIGAR, matrix=m)
    before = lib.ns_gpu_dispatch_count()
    ok, *_ = L.gpu_global(b"TGG" * 300, b"W" * 300, opt)
    assert not ok
    assert lib.ns_gpu_dispatch_count() == before


def test_queue_concurrent_threads(queue_ready, oracle):
    """test_gpu.c:141-185: 32 concurrent callers are coalesced into fewer launches."""
    lib = L.load()
    opt = Options.nasw_defaults(flag=NS_F_CIGAR, go=3, ge=1, io=100, fs=100, sp_model=0)
    want = oracle.run("gs16b", b"ATGAAAACTTGG", b"MKQTW", opt)
    barrier = threading.Barrier(33)
    out = [None] * 32

    def worker(k):
        barrier.wait()
        out[k] = L.gpu_global(b"ATGAAAACTTGG", b"MKQTW", opt)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(32)]
    for t in threads:
        t.start()
    d0, l0 = lib.ns_gpu_dispatch_count(), lib.ns_gpu_launch_count()
    barrier.wait()
    for t in threads:
        t.join()
    for ok, score, ntl, aal, cig in out:
        assert ok and (score, ntl, aal, cig) == want
    assert lib.ns_gpu_dispatch_count() - d0 == 32
    assert 0 < lib.ns_gpu_launch_count() - l0 < 32


def test_queue_async_submits(queue_ready, oracle):
    """test_gpu.c:187-219: 129 submits before any wait."""
    lib = L.load()
    opt = Options.nasw_defaults(flag=NS_F_CIGAR, go=3, ge=1, io=100, fs=100, sp_model=0)
    want = oracle.run("gs16b", b"ATGAAAACTTGG", b"MKQTW", opt)
    d0, l0 = lib.ns_gpu_dispatch_count(), lib.ns_gpu_launch_count()
    reqs = [lib.ns_gpu_submit(None, b"ATGAAAACTTGG", 12, b"MKQTW", 5, opt.ptr, None) for _ in range(129)]
    assert all(reqs)
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    for rq in reqs:
        r = NsRst()
        assert lib.ns_gpu_wait(rq, C.byref(r))
        cig = [r.cigar[k] for k in range(r.n_cigar)]
        assert (r.score, r.nt_len, r.aa_len, cig) == want
        libc.free(C.cast(r.cigar, C.c_void_p))
    assert lib.ns_gpu_dispatch_count() - d0 == 129
    assert lib.ns_gpu_launch_count() - l0 >= 2


def _paired_batch(rng, n, max_al=80):
    """Random loci on both strands plus exact duplicates: every job has a partner with the same
    protein and window length, so the engine runs them as int16x2 pairs."""
    pairs = []
    for q in range(n):
        nt, aa = W.random_pair(rng, max_al=max_al)
        pairs += [(nt, aa), (W.revcomp(nt), aa)] if q % 3 else [(nt, aa), (nt, aa)]
    return pairs


@pytest.mark.parametrize("seed", [21, 22])
def test_paired_int16x2_bit_exact(engine, oracle, seed):
    """The paired kernel (two jobs per 32-bit lane) against the oracle: random pairs on both
    strands, planted loci, and the golden vectors with a duplicate strand; pairing on and off
    give identical results."""
    rng = np.random.default_rng(seed)
    opt = Options(flag=NS_F_CIGAR)
    pairs = _paired_batch(rng, 150)
    for q in range(6):
        nt, aa = W.single_locus(seed=seed * 100 + q, al=int(rng.integers(120, 600)),
                                window=int(rng.integers(2000, 9000)))
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    engine.set_pairing(2)  # every eligible job, whatever the batch's size
    try:
        got = _check(engine, oracle, opt, pairs)
        assert engine.last_pairs() == len(pairs) // 2
        engine.set_pairing(False)
        plain = engine.align_host(opt, pairs)
        assert engine.last_pairs() == 0
    finally:
        engine.set_pairing(True)
    assert [(s, c) for s, c, _ in got] == [(s, c) for s, c, _ in plain]


def test_paired_golden_vectors_with_twins(engine, oracle, golden):
    """Each golden vector the 16-bit DP answers (ns_global_gs16b, and ns_global_gs_auto where
    it dispatches to 16 bits) next to its own twin (same protein, same window)."""
    by_opt = {}
    for c in golden["cases"]:
        if c["opt"].get("flag", NS_F_CIGAR) & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT) or \
                c["fn"] not in ("ns_global_gs16b", "ns_global_gs_auto"):
            continue
        if c["ss"]:
            continue
        by_opt.setdefault(repr(sorted(c["opt"].items())), []).append(c)
    n = n_pairs = 0
    engine.set_pairing(2)
    try:
        for cases in by_opt.values():
            opt = oracle.make_options(cases[0]["opt"])
            cases = [c for c in cases if not oracle.port_lib().port_needs_wide(opt.ptr, len(c["aa"]))]
            pairs = []
            for c in cases:
                pairs += [(c["nt"].encode(), c["aa"].encode())] * 2
            got = engine.align_host(opt, pairs)
            n_pairs += engine.last_pairs()
            for k, c in enumerate(cases):
                for t in range(2):
                    score, cig, _ = got[2 * k + t]
                    assert (score, cig) == (c["score"], c["cigar"]), (c["group"], len(c["nt"]), len(c["aa"]), score)
                    n += 1
    finally:
        engine.set_pairing(True)
    assert n >= 300 and n_pairs >= 100, (n, n_pairs)


def test_paired_cooperative_and_waves(oracle):
    """Long pairs on whole-CTA wavefronts, in a batch split into several trace waves."""
    rng = np.random.default_rng(23)
    opt = Options(flag=NS_F_CIGAR)
    pairs = []
    for q in range(10):
        al = int(rng.integers(250, 700))
        nt, aa = W.single_locus(seed=2300 + q, al=al, window=int(rng.integers(12000, 30000)))
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    pairs += _paired_batch(rng, 60, max_al=50)
    eng = L.Engine(0, trace_budget_bytes=96 << 20)
    try:
        eng.set_tuning(0, 0.1)
        eng.set_pairing(2)
        got = _check(eng, oracle, opt, pairs)
        plan = eng.last_plan()
        assert plan["waves"] >= 2 and plan["coop"] >= 2 and eng.last_pairs() == len(pairs) // 2, plan
    finally:
        eng.close()


def test_pairs_only_when_they_fill_the_gpu(oracle):
    """Default pairing: 3000 small loci on both strands (more pairs than the DP launch has
    warps) all pair; a batch of a few large loci keeps its jobs single.  Results equal the
    oracle's in both."""
    rng = np.random.default_rng(26)
    opt = Options(flag=NS_F_CIGAR)
    small = []
    for q in range(3000):
        nt, aa = W.random_pair(rng, max_al=30)
        small += [(nt, aa), (W.revcomp(nt), aa)]
    big = []
    for q in range(2):
        nt, aa = W.single_locus(seed=2600 + q, al=500, window=16000)
        big += [(nt, aa), (W.revcomp(nt), aa)]
    eng = L.Engine(0)
    try:
        _check(eng, oracle, opt, small + big)
        assert eng.last_pairs() == len(small + big) // 2
        _check(eng, oracle, opt, big)
        assert eng.last_pairs() == 0
    finally:
        eng.close()


def test_pairs_not_formed_outside_the_15_bit_range(engine, oracle):
    """Penalties large enough to reach the int16 floor keep jobs unpaired (32-bit lanes)."""
    rng = np.random.default_rng(24)
    opt = Options(flag=NS_F_CIGAR, go=3000, ge=200, io=9000, fs=5000, stop_pen=23)
    pairs = _paired_batch(rng, 40, max_al=40)
    _check(engine, oracle, opt, pairs)
    assert engine.last_pairs() == 0


def test_graph_replay_bit_exact(oracle):
    """A batch fed again and again: the second call captures the launch plan into a CUDA graph,
    later calls replay it; every call's results equal the oracle's, and with graphs off too."""
    rng = np.random.default_rng(25)
    opt = Options(flag=NS_F_CIGAR)
    pairs = _paired_batch(rng, 40, max_al=60) + [W.random_pair(rng, max_al=60) for _ in range(30)]
    eng = L.Engine(0)
    try:
        r0 = int(eng.lib.pl_engine_graph_replays(eng.h))
        outs = [_check(eng, oracle, opt, pairs) for _ in range(4)]
        assert int(eng.lib.pl_engine_graph_replays(eng.h)) - r0 >= 2
        eng.lib.pl_engine_set_graphs(eng.h, 0)
        outs.append(_check(eng, oracle, opt, pairs))
        assert all(o == outs[0] for o in outs)
    finally:
        eng.close()
