"""The allocation-free entry point gives the same answers as the allocating one.

pl_splice_batch_noalloc() exists for callers that cannot allocate device memory
on this path (a program that runs under a fixed device-memory budget owned by its
own pool, or a latency-sensitive loop that cannot take cudaMalloc's device-wide
synchronisation); all of its scratch lives in one fixed array inside the library.
This test runs the same batch through pl_splice_batch_device() and then twice in a
row through pl_splice_batch_noalloc() -- the second call reuses the array the first
one left behind -- and requires identical scores and CIGARs (the DP is integer
arithmetic, so the tolerance is zero).  It also checks that a batch too large for
the fixed array is refused with a message instead of running.

Three option sets cover the three DP launches inside the entry point: the
default scoring (16-bit jobs), a matrix with W:W = 127 (the 32-bit route of
ns_global_gs_auto for the longer proteins, 16-bit for the shorter ones, so one
call launches both), and W:W = 110 with a negative end bonus (16-bit with the
upper clamp live).

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from protlocus_b200 import lib as L
from protlocus_b200 import workload as W
from protlocus_b200.abi import AA_I2C, BLOSUM62, NS_F_CIGAR, Options, SpliceJob, SpliceResult

pytestmark = pytest.mark.gpu


def _batch():
    rng = np.random.default_rng(31)
    pairs = [W.random_pair(rng, max_al=90) for _ in range(300)]
    for q in range(6):
        al = int(rng.integers(150, 500))
        nt, aa = W.single_locus(seed=700 + q, al=al, window=int(rng.integers(3 * al + 200, 3 * al + 2500)))
        pairs += [(nt, aa), (W.revcomp(nt), aa)]
    return pairs


def _case(kind):
    """(options, pairs, widths the jobs must run at) of one option set."""
    if kind == "default":
        return Options(flag=NS_F_CIGAR), _batch(), {16}
    rng = np.random.default_rng(32 if kind == "wide" else 33)
    m = BLOSUM62.copy()
    w = AA_I2C.index("W")
    pairs = []
    if kind == "wide":  # 32-bit for al*127 + end_bonus > 30000 (al >= 237), 16-bit below
        m[w, w] = 127
        opt = Options.nasw_defaults(flag=NS_F_CIGAR, matrix=m)
        for q in range(24):
            al = int(rng.integers(240, 420)) if q % 2 == 0 else int(rng.integers(20, 200))
            nt, aa = W.single_locus(seed=int(rng.integers(1 << 30)), al=al, window=3 * al + int(rng.integers(50, 1500)))
            pairs.append((nt, aa))
        return opt, pairs, {16, 32}
    m[w, w] = 110  # upper clamp: al*110 within 256 of 32767, end bonus -6000 keeps the 16-bit route
    opt = Options(flag=NS_F_CIGAR, matrix=m, end_bonus=-6000)
    for _ in range(12):
        al = int(rng.integers(296, 320))
        aa = rng.choice(list(b"WWWWWACDEFG"), size=al).astype(np.uint8).tobytes()
        nt = W.random_dna(rng, int(rng.integers(3 * al, 3 * al + 400))).encode()
        pairs.append((nt, aa))
    return opt, pairs, {16}


def _upload(torch, pairs):
    n = len(pairs)
    jobs = (SpliceJob * n)()
    pos_nt = pos_aa = 0
    for q, (nt, aa) in enumerate(pairs):
        jobs[q].nt_off, jobs[q].aa_off, jobs[q].ss_off, jobs[q].nl, jobs[q].al = pos_nt, pos_aa, -1, len(nt), len(aa)
        pos_nt += len(nt)
        pos_aa += len(aa)
    d_nt = torch.tensor(np.frombuffer(b"".join(p[0] for p in pairs), dtype=np.uint8), device="cuda")
    d_aa = torch.tensor(np.frombuffer(b"".join(p[1] for p in pairs), dtype=np.uint8), device="cuda")
    return jobs, d_nt, d_aa


def _read(torch, n, d_res, d_cig):
    res = (SpliceResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
    cig = d_cig.cpu().numpy().view(np.uint32)
    out = []
    for r in res:
        assert r.status == 0
        out.append((r.score, r.mode, cig[r.cigar_off:r.cigar_off + r.n_cigar].tolist()))
    return out


@pytest.mark.parametrize("kind", ["default", "wide", "upper_clamp"])
def test_noalloc_matches_allocating_entry_point(kind):
    torch = pytest.importorskip("torch")
    lib = L.load()
    opt, pairs, widths = _case(kind)
    n = len(pairs)
    jobs, d_nt, d_aa = _upload(torch, pairs)
    cap = sum(len(a) + len(b) + 8 for a, b in pairs)
    stream = torch.cuda.current_stream().cuda_stream

    d_res = torch.zeros(n * C.sizeof(SpliceResult), dtype=torch.uint8, device="cuda")
    d_cig = torch.zeros(cap, dtype=torch.int32, device="cuda")
    total = C.c_int64()
    eng = L.Engine(0)
    assert eng.lib.pl_splice_batch_device(eng.h, opt.ptr, jobs, n, d_nt.data_ptr(), d_aa.data_ptr(), None,
                                          d_res.data_ptr(), d_cig.data_ptr(), cap, C.byref(total), stream), L.error()
    want = _read(torch, n, d_res, d_cig)
    eng.close()
    assert {w for _, w, _ in want} == widths

    for call in range(2):  # the second call starts from the array the first one left behind
        d_res2 = torch.full((n * C.sizeof(SpliceResult),), 0xA5, dtype=torch.uint8, device="cuda")
        d_cig2 = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        total2 = C.c_int64()
        ok = lib.pl_splice_batch_noalloc(opt.ptr, jobs, n, d_nt.data_ptr(), d_aa.data_ptr(), None,
                                         d_res2.data_ptr(), d_cig2.data_ptr(), cap, C.byref(total2), stream)
        assert ok, lib.pl_noalloc_error().decode()
        got = _read(torch, n, d_res2, d_cig2)
        assert total2.value == total.value
        bad = [q for q in range(n) if got[q] != want[q]]
        assert not bad, f"call {call}: {len(bad)} jobs differ, first {bad[:5]}"


def test_noalloc_refuses_oversized_batch():
    torch = pytest.importorskip("torch")
    lib = L.load()
    opt = Options(flag=NS_F_CIGAR)
    pairs = [(b"ACGT" * 12500, b"M" * 1500)]  # ~150 MB of traceback scratch: over the fixed array
    jobs, d_nt, d_aa = _upload(torch, pairs)
    d_res = torch.zeros(C.sizeof(SpliceResult), dtype=torch.uint8, device="cuda")
    d_cig = torch.zeros(64, dtype=torch.int32, device="cuda")
    ok = lib.pl_splice_batch_noalloc(opt.ptr, jobs, 1, d_nt.data_ptr(), d_aa.data_ptr(), None, d_res.data_ptr(),
                                     d_cig.data_ptr(), 64, None, torch.cuda.current_stream().cuda_stream)
    assert ok == 0
    assert "scratch" in lib.pl_noalloc_error().decode()
