"""GPU agreement of the recheck Forward score with the reference's own rc_score
(recheck.c:283-440), float.  The device Forward keeps rc_score's operation order,
evaluates rc_logsum's expf / log1pf with the host glibc's algorithms restated
(protlocus_b200/csrc/glibc_mathf.cuh) and takes the length model's logf values
from the host, so the bit score and the null2 bias are required to be EQUAL to
the reference's, bit for bit (which implies the |d bits| <= 1e-5 |bits| bound).

Profiles are HMMER3 text parsed by the reference's rc_read_prof (which also
builds the multihit-local search profile); the checker is recheck.c itself,
compiled by oracle/Makefile into oracle/_ref/librecheck_ref.so and run over the
host's cores by its own kt_for.  Peptides: background residues (many score near
0 bits), domains sampled from the profile (high scores), degenerate residues,
lengths 1 to 900, with and without null2, profiles of 20 to 2048 positions
(1 to 64 columns per lane).
"""
import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import hmm as H
from protlocus_b200 import lib as L

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.rc_lib() is None, reason="oracle/_ref/librecheck_ref.so not built")]

TOL = 1e-5  # the relative bound on the score; the tests below ask for equality, which is tighter


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def _peptides(rng, probs, n, lmax):
    out = []
    for q in range(n):
        Lq = int(rng.integers(1, lmax + 1))
        if q % 3 == 0:  # a domain sampled from the profile's match emissions
            m = probs.shape[0]
            a = int(rng.integers(0, max(1, m - 5)))
            b = min(m, a + Lq)
            cdf = np.cumsum(probs[a:b] / probs[a:b].sum(axis=1, keepdims=True), axis=1)
            idx = (rng.random(b - a)[:, None] > cdf).sum(axis=1).clip(0, 19)
        else:
            idx = rng.integers(0, 20, size=Lq)
        seq = bytearray(H.ALPHABET[int(x)].encode()[0] for x in idx)
        for j in range(len(seq)):
            if rng.random() < 0.02:
                seq[j] = ord("X")
        out.append(bytes(seq))
    return out


@pytest.mark.parametrize("null2", [True, False])
def test_forward_vs_reference(engine, null2):
    texts, probs = H.synthetic_profiles(6, seed=51, m_min=20, m_max=1500)
    handle, profs = O.rc_load("".join(texts))
    gp = [L.RcProfile(msc, tsc) for _, msc, tsc in profs]
    rng = np.random.default_rng(9)
    peps = []
    for k in range(len(profs)):
        for s in _peptides(rng, probs[k], 12, 900):
            peps.append((k, O.rc_encode(s)))
    peps.append((0, O.rc_encode(b"W")))  # length 1
    bits, bias = engine.rc_score(gp, peps, null2)
    for (k, d), b, s in zip(peps, bits, bias):
        rb, rs = O.rc_ref_score(handle, k, d, null2)
        assert abs(b - rb) <= TOL * abs(rb), (k, len(d), b, rb)
        assert (b, s) == (np.float32(rb), np.float32(rs)), (k, len(d), b, rb, s, rs)
    assert engine.lib.pl_rc_last_cells(engine.h) == sum(len(d) * profs[k][0] for k, d in peps)
    for p in gp:
        p.close()


def _sweep_set():
    """2,400 peptides over 12 profiles of 20 to 2048 positions: background residues (scores near
    0 bits), profile-sampled domains and degenerate residues, lengths 1 to 900."""
    ms = [20, 31, 57, 128, 300, 511, 700, 1024, 1300, 1500, 2047, 2048]
    texts, probs = [], []
    for q, m in enumerate(ms):
        t, p = H.synthetic_profiles(1, seed=200 + q, m_min=m, m_max=m)
        texts += t
        probs += p
    handle, profs = O.rc_load("".join(texts))
    rng = np.random.default_rng(65)
    peps = []
    for k in range(len(ms)):
        lmax = 900 if ms[k] <= 700 else 420
        for s in _peptides(rng, probs[k], 200, lmax):
            peps.append((k, O.rc_encode(s)))
    return handle, profs, peps


@pytest.mark.parametrize("null2", [True, False])
def test_forward_sweep_bit_exact(engine, null2):
    """The widened sweep: every score and bias equal to the reference's, including the hundreds of
    peptides whose score is within 1 bit of 0 (where a relative bound is hardest to meet)."""
    handle, profs, peps = _sweep_set()
    gp = [L.RcProfile(msc, tsc) for _, msc, tsc in profs]
    bits, bias = engine.rc_score(gp, peps, null2)
    rbits, rbias = O.rc_ref_batch(handle, peps, null2)
    near0 = int(np.sum(np.abs(rbits) < 1.0))
    bad = np.nonzero((bits.view(np.uint32) != rbits.view(np.uint32)) | (bias.view(np.uint32) != rbias.view(np.uint32)))[0]
    rel = np.abs(bits.astype(np.float64) - rbits) / np.maximum(np.abs(rbits.astype(np.float64)), 1e-30)
    print(f"{len(peps)} peptides, {near0} within 1 bit of 0, {len(bad)} differ, worst relative {rel.max():.2e}")
    assert len(peps) >= 2000 and near0 >= 100 and max(profs[k][0] for k, _ in peps) == 2048
    assert len(bad) == 0, [(int(i), peps[i][0], len(peps[i][1]), bits[i], rbits[i], bias[i], rbias[i]) for i in bad[:5]]
    for p in gp:
        p.close()


def test_wait_between_warps_runs_out_cleanly(engine):
    """A Forward group's warps hand values over through bounded waits.  With the limit
    cut to a few cycles a wait runs out: the call fails with the reason (no fault, no
    hang: the warps leave their loops and the kernel ends), and with the default limit
    back the same engine scores the batch bit for bit."""
    texts, probs = H.synthetic_profiles(2, seed=53, m_min=300, m_max=400)
    handle, profs = O.rc_load("".join(texts))
    gp = [L.RcProfile(msc, tsc) for _, msc, tsc in profs]
    rng = np.random.default_rng(13)
    peps = [(k, O.rc_encode(s)) for k in range(len(profs)) for s in _peptides(rng, probs[k], 8, 300)]
    lib = engine.lib
    try:
        assert lib.pl_rc_debug_wait_limit(4) == 1
        with pytest.raises(RuntimeError, match="wait between the warps"):
            engine.rc_score(gp, peps, True)
    finally:
        lib.pl_rc_debug_wait_limit(0)
    bits, bias = engine.rc_score(gp, peps, True)
    for (k, d), b, s in zip(peps, bits, bias):
        rb, rs = O.rc_ref_score(handle, k, d, True)
        assert (b, s) == (np.float32(rb), np.float32(rs)), (k, len(d), b, rb, s, rs)
    for p in gp:
        p.close()


def _bits_of(f):
    return int(np.array([f], dtype=np.float32).view(np.uint32)[0])


@pytest.mark.parametrize("fn,lo,hi", [
    (0, 0x80000000, _bits_of(-50.0) + 1),  # expf at every float in [-50, -0], the arguments rc_logsum passes
    (1, 0x00000000, _bits_of(1.0) + 1),    # log1pf at every float in [0, 1], the values expf returns there
    (2, 0x80000000, _bits_of(-50.0) + 1),  # the branch-free forms rc_logsum runs on the device, same ranges
    (3, 0x00000000, _bits_of(1.0) + 1),    # (log1pf's includes the branch-free division)
    (4, 0x80000000, _bits_of(-50.0) + 1),  # their four-wide forms (four arguments per evaluation)
    (5, 0x00000000, _bits_of(1.0) + 1),
])
def test_device_libm_equals_host(fn, lo, hi):
    """The device build of the restated expf / log1pf against the host libm at every float bit pattern
    of the range the Forward reaches (about 1.1e9 each), in chunks."""
    import ctypes as C
    import os
    so = os.path.join(os.path.dirname(__file__), "..", "oracle", "_build", "liblmcheck.so")
    if not os.path.exists(so):
        pytest.skip("oracle/_build/liblmcheck.so not built")
    host = C.CDLL(so)
    host.lm_host.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_int64, C.c_void_p]
    lib = L.load()
    chunk = 1 << 26
    dev, ref = np.empty(chunk, np.float32), np.empty(chunk, np.float32)
    total = 0
    for start in range(lo, hi, chunk):
        n = min(chunk, hi - start)
        assert lib.pl_rc_mathf_eval(0, fn, start, 1, n, dev.ctypes.data) == 1
        host.lm_host(fn, start, 1, n, ref.ctypes.data)
        a, b = dev[:n].view(np.uint32), ref[:n].view(np.uint32)
        diff = (a != b) & ~(np.isnan(dev[:n]) & np.isnan(ref[:n]))
        assert not diff.any(), f"first mismatch at bit pattern {start + int(np.argmax(diff)):#010x}"
        total += n
    assert total == hi - lo
