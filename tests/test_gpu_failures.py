"""Failures surface as error codes, never as an abort or a CPU fallback.

Every failure here is made on the host (pl_debug_fault's injection sites, a
trace budget that is too small, corrupt spans, a km arena without kalloc); no
test faults, traps or hangs the GPU.  After each failure the same engine or
executor must serve the next call with bit-exact results.

The reference's extension executor drains failed jobs to its CPU kernel
(nasw-ext-gpu.c:835-844); this library has no CPU path, so a failed request is
reported: ns_ext_batch_get() returns NULL and ns_gpu_error() says why.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import NS_F_CIGAR, NS_F_EXT_RIGHT, NsRst, Options, SpliceJob, SpliceResult, ExtJob, ExtResult

pytestmark = pytest.mark.gpu

SITE_HOST_ALLOC, SITE_DEV_ALLOC, SITE_EXT_BATCH = 0, 1, 2


@pytest.fixture(autouse=True)
def _disarm():
    lib = L.load()
    yield
    for site in (SITE_HOST_ALLOC, SITE_DEV_ALLOC, SITE_EXT_BATCH):
        lib.pl_debug_fault(site, -1)


def _ext_requests(rng, n):
    out = []
    for _ in range(n):
        nt, aa = W.random_pair(rng, max_al=50)
        out.append((nt, aa))
    return out


def _ext_want(opt, nt, aa):
    s, ntl, aal, _ = O.port_run("gs16b", nt, aa, opt, None, avx2=L.ext_stripe_width(opt, len(aa)) == 16)
    return (s, ntl, aal)


def test_ext_executor_device_batch_failure_is_reported():
    lib = L.load()
    opt = Options(flag=NS_F_EXT_RIGHT)
    rng = np.random.default_rng(5)
    b = L.ExtBatch()
    reqs = _ext_requests(rng, 8)
    ids = [b.add(nt, aa, opt) for nt, aa in reqs]
    before = lib.pl_ext_failed_count()
    assert lib.pl_debug_fault(SITE_EXT_BATCH, 0) == 1
    assert b.flush() == len(ids)
    for rid in ids:
        assert not lib.ns_ext_batch_get(b.h, rid)          # NULL: failed, no CPU result
        assert b.ready(rid)
    assert lib.pl_ext_failed_count() - before == len(ids)
    assert "injected" in lib.ns_gpu_error().decode()
    # the executor keeps serving: the next flush is bit-exact
    reqs2 = _ext_requests(rng, 8)
    ids2 = [b.add(nt, aa, opt) for nt, aa in reqs2]
    b.flush()
    for rid, (nt, aa) in zip(ids2, reqs2):
        assert b.get(rid) == _ext_want(opt, nt, aa)
    b.close()


def test_ext_batch_host_allocation_failure_is_reported():
    lib = L.load()
    opt = Options(flag=NS_F_EXT_RIGHT)
    rng = np.random.default_rng(6)
    b = L.ExtBatch()
    assert lib.pl_debug_fault(SITE_HOST_ALLOC, 0) == 1     # the first queue growth fails
    reqs = _ext_requests(rng, 5)
    ids = [b.add(nt, aa, opt) for nt, aa in reqs]
    assert ids == list(range(ids[0], ids[0] + 5))           # ids are still handed out
    assert b.flush() == 0                                   # nothing reached the device
    for rid in ids:
        assert b.ready(rid) and not lib.ns_ext_batch_get(b.h, rid)
    assert "out of host memory" in lib.pl_last_error().decode()
    reqs2 = _ext_requests(rng, 5)
    ids2 = [b.add(nt, aa, opt) for nt, aa in reqs2]
    assert b.flush() == 5
    for rid, (nt, aa) in zip(ids2, reqs2):
        assert b.get(rid) == _ext_want(opt, nt, aa)
    b.close()


def test_engine_device_allocation_failure_then_recovery():
    lib = L.load()
    opt = Options(flag=NS_F_CIGAR)
    rng = np.random.default_rng(7)
    pairs = [W.random_pair(rng, max_al=60) for _ in range(16)]
    eng = L.Engine(0)
    assert lib.pl_debug_fault(SITE_DEV_ALLOC, 0) == 1
    with pytest.raises(RuntimeError, match="injected"):
        eng.align_host(opt, pairs)
    got = eng.align_host(opt, pairs)
    for (nt, aa), (s, c, _w) in zip(pairs, got):
        want = O.run("gs_auto", nt, aa, opt)
        assert (s, c) == (want[0], want[3])
    eng.close()


def test_trace_budget_too_small_is_an_error():
    opt = Options(flag=NS_F_CIGAR)
    nt, aa = W.single_locus(seed=0)                         # ~20 MB of trace words
    eng = L.Engine(0, trace_budget_bytes=1 << 20)
    with pytest.raises(RuntimeError, match="over the budget"):
        eng.align_host(opt, [(nt, aa)])
    rng = np.random.default_rng(8)
    small = [W.random_pair(rng, max_al=30) for _ in range(8)]
    for (n_, a_), (s, c, _w) in zip(small, eng.align_host(opt, small)):
        want = O.run("gs_auto", n_, a_, opt)
        assert (s, c) == (want[0], want[3])
    eng.close()


def test_corrupt_spans_are_refused_before_any_device_work():
    lib = L.load()
    opt = Options(flag=NS_F_CIGAR)
    eng = L.Engine(0)
    nt = np.frombuffer(b"ACGT" * 30, dtype=np.uint8)
    aa = np.frombuffer(b"MKV" * 5, dtype=np.uint8)
    cig = np.zeros(1024, dtype=np.uint32)
    for nt_off, nl, aa_off, al in [(100, 40, 0, 10), (-1, 20, 0, 10), (0, 20, 10, 10), (0, 1 << 30, 0, 10)]:
        jobs = (SpliceJob * 1)()
        jobs[0].nt_off, jobs[0].nl, jobs[0].aa_off, jobs[0].al, jobs[0].ss_off = nt_off, nl, aa_off, al, -1
        res = (SpliceResult * 1)()
        ok = lib.pl_splice_batch_host(eng.h, opt.ptr, jobs, 1, nt.ctypes.data, nt.size, aa.ctypes.data, aa.size,
                                      None, 0, res, cig.ctypes.data, cig.size)
        assert ok == 0 and "outside" in lib.pl_last_error().decode()
    ext = (ExtJob * 1)()
    ext[0].nt_off, ext[0].nl, ext[0].aa_off, ext[0].al = 0, 200, 0, 10
    ext[0].ss_off = ext[0].pssm_off = -1
    ext[0].flag = NS_F_EXT_RIGHT
    xres = (ExtResult * 1)()
    ok = lib.pl_ext_batch_host(eng.h, opt.ptr, ext, 1, nt.ctypes.data, nt.size, aa.ctypes.data, aa.size, None, 0,
                               None, 0, xres)
    assert ok == 0 and "outside" in lib.pl_last_error().decode()
    # the engine is intact
    rng = np.random.default_rng(9)
    pairs = [W.random_pair(rng, max_al=40) for _ in range(4)]
    for (n_, a_), (s, c, _w) in zip(pairs, eng.align_host(opt, pairs)):
        want = O.run("gs_auto", n_, a_, opt)
        assert (s, c) == (want[0], want[3])
    eng.close()


def test_request_queue_reports_cigar_growth_failure():
    lib = L.load()
    opt = Options(flag=NS_F_CIGAR)
    assert L.gpu_init(0)
    nt, aa = W.single_locus(seed=0)
    # a km arena handed in by a program that links no kalloc: the CIGAR cannot be grown in it
    if hasattr(C.CDLL(None), "krealloc"):
        pytest.skip("this process links a kalloc")
    r = NsRst()
    assert lib.ns_gpu_global(C.c_void_p(1), nt, len(nt), aa, len(aa), opt.ptr, None, C.byref(r)) == 0
    assert "kalloc" in lib.ns_gpu_error().decode()
    # host allocation failure while the CIGAR grows
    r = NsRst()
    assert lib.pl_debug_fault(SITE_HOST_ALLOC, 0) == 1
    assert lib.ns_gpu_global(None, nt, len(nt), aa, len(aa), opt.ptr, None, C.byref(r)) == 0
    assert "out of host memory" in lib.ns_gpu_error().decode()
    ok, score, ntl, aal, cig = L.gpu_global(nt, aa, opt)
    want = O.run("gs_auto", nt, aa, opt)
    assert ok and (score, ntl, aal, cig) == want
