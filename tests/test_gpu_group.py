"""pl_group_splice_host on the B200: one batch split over a group of engines.

This run has one GPU, so the group holds two engines on device 0 (two slots,
two host threads, each with its own streams and buffers); the split, the
per-slot packing and the gather are the code a multi-GPU group runs.  The
results must equal pl_splice_batch_host's over the whole batch, job for job.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import NS_F_CIGAR, Options, SpliceJob, SpliceResult

pytestmark = pytest.mark.gpu


def test_group_of_two_slots_matches_one_engine():
    lib = L.load()
    rng = np.random.default_rng(41)
    pairs = [W.random_pair(rng, max_al=80) for _ in range(200)]
    for q in range(4):
        nt, aa = W.single_locus(seed=900 + q, al=300, window=4000)
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    opt = Options(flag=NS_F_CIGAR)
    n = len(pairs)
    jobs = (SpliceJob * n)()
    pn = pa = 0
    for q, (nt, aa) in enumerate(pairs):
        jobs[q].nt_off, jobs[q].aa_off, jobs[q].ss_off, jobs[q].nl, jobs[q].al = pn, pa, -1, len(nt), len(aa)
        pn += len(nt)
        pa += len(aa)
    nt = np.frombuffer(b"".join(p[0] for p in pairs), np.uint8)
    aa = np.frombuffer(b"".join(p[1] for p in pairs), np.uint8)
    cap = sum(len(a) + len(b) + 8 for a, b in pairs)
    devs = (C.c_int32 * 2)(0, 0)
    g = lib.pl_group_create(devs, 2, 2 << 30)
    assert g, L.error()
    try:
        res = (SpliceResult * n)()
        cig = np.zeros(cap, np.uint32)
        total = C.c_int64()
        assert lib.pl_group_splice_host(g, opt.ptr, jobs, n, nt.ctypes.data, nt.size, aa.ctypes.data, aa.size,
                                        None, 0, res, cig.ctypes.data, cap, C.byref(total)), L.error()
        dev, _ = L.group_plan(jobs, 2)
        assert set(dev.tolist()) == {0, 1}
        eng = L.Engine(0)
        want = eng.align_host(opt, pairs)
        eng.close()
        off = 0
        for q in range(n):
            assert res[q].status == 0 and res[q].cigar_off == off
            got = (res[q].score, cig[off:off + res[q].n_cigar].tolist())
            assert got == (want[q][0], want[q][1]), q
            off += res[q].n_cigar
        assert total.value == off
        for q in range(0, n, 37):
            w = O.run("gs_auto", pairs[q][0], pairs[q][1], opt)
            assert (res[q].score, cig[res[q].cigar_off:res[q].cigar_off + res[q].n_cigar].tolist()) == (w[0], list(w[3]))
    finally:
        lib.pl_group_destroy(g)
