"""GPU agreement of the recheck Forward score with the reference's own rc_score
(recheck.c:283-440), float: the bit score within 1e-5 relative, and the null2
bias (which is subtracted from the score) within 1e-5 of the score's scale,
max(1, |bits|).  The bias alone is exp of a sum over every residue of float
log-odds, so summation-order rounding moves it by more than 1e-5 of its own
(often tiny) value; what reaches the E-value is the score.

Profiles are HMMER3 text parsed by the reference's rc_read_prof (which also
builds the multihit-local search profile); the checker is recheck.c itself,
compiled by oracle/Makefile into oracle/_ref/librecheck_ref.so.  Peptides:
background residues, domains sampled from the profile (high scores), degenerate
residues, lengths 1 to 900, with and without null2, profiles of 1 to 3 lane
blocks per lane (m up to 1500).
"""
import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import hmm as H
from protlocus_b200 import lib as L

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.rc_lib() is None, reason="oracle/_ref/librecheck_ref.so not built")]

TOL = 1e-5


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
    worst = 0.0
    for (k, d), b, s in zip(peps, bits, bias):
        rb, rs = O.rc_ref_score(handle, k, d, null2)
        e1 = abs(b - rb) / max(1.0, abs(rb))
        e2 = abs(s - rs) / max(1.0, abs(rb))
        worst = max(worst, e1, e2)
        assert e1 <= TOL and e2 <= TOL, (k, len(d), b, rb, s, rs)
    print(f"worst relative error {worst:.2e}")
    assert engine.lib.pl_rc_last_cells(engine.h) == sum(len(d) * profs[k][0] for k, d in peps)
    for p in gp:
        p.close()
