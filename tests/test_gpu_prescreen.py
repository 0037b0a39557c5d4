"""The prescreen's banded gapped alignment on the device (pscreen.cu) against the
reference's own ps_gapped (prescreen.c:346-382) compiled behind oracle/ref_prescreen.c.

Cases: HMM-like PSSMs from synthetic Plan7 profiles parsed by the restated hmm.c
reader, and random PSSMs; ORFs with a planted profile-sampled stretch or random; the
default band (32), narrow bands, the full matrix (band <= 0), and diagonals from far
left of the ORF to far right of it (bands clipped or outside the matrix).
"""
import numpy as np
import pytest

import oracle_lib as O
from protlocus_b200 import lib as L

need_ref = pytest.mark.skipif(O.ps_lib() is None, reason="oracle/_ref/libps_ref.so not built")


def _cases(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        Lq = int(rng.integers(1, 400))
        pssm = rng.integers(-9, 8, size=(Lq, 22)).astype(np.int8)
        nq = int(rng.integers(1, 600))
        orf = rng.integers(0, 22, size=nq).astype(np.uint8)
        if q % 3 == 0 and nq > 40 and Lq > 40:  # a stretch the profile likes, on one diagonal
            d0 = int(rng.integers(-Lq // 2, nq // 2))
            for i in range(Lq):
                t = i + d0
                if 0 <= t < nq and rng.random() < 0.8:
                    orf[t] = int(np.argmax(pssm[i]))
            diag = d0 + int(rng.integers(-3, 4))
        else:
            diag = int(rng.integers(-Lq - 50, nq + 50))
        band = int(rng.choice([32, 32, 32, 8, 1, 0, -5, 64]))
        out.append((pssm, orf, diag, band))
    return out


@need_ref
def test_reference_ps_gapped_hand_case():
    """One residue the profile scores 5 on, at the diagonal: the local score is 5."""
    pssm = np.full((1, 22), -3, np.int8)
    pssm[0, 7] = 5
    assert O.ref_ps_gapped(pssm, np.array([1, 7, 2], np.uint8), 1, 32) == 5
    assert O.ref_ps_gapped(pssm, np.array([1, 2, 3], np.uint8), 1, 32) == 0


@pytest.mark.gpu
@need_ref
def test_ps_gapped_matches_reference():
    cands = _cases(3, 600)
    eng = L.Engine(0)
    try:
        got = eng.ps_gapped(cands)
    finally:
        eng.close()
    want = np.array([O.ref_ps_gapped(p, o, d, b) for p, o, d, b in cands])
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, [(int(i), cands[i][0].shape[0], cands[i][1].size, cands[i][2], cands[i][3], int(got[i]),
                            int(want[i])) for i in bad[:5]]
    assert (want > 0).mean() > 0.5


@pytest.mark.gpu
def test_ps_gapped_device_entry_equals_host_entry():
    """pl_ps_gapped_device on device-resident PSSMs and ORFs gives the host entry point's scores."""
    import torch
    cands = _cases(4, 400)
    eng = L.Engine(0)
    try:
        pk = eng.ps_pack(cands)
        want = eng.ps_run(pk).copy()
        d_pssm = torch.from_numpy(pk["pssm"]).to("cuda")
        d_orf = torch.from_numpy(pk["orf"]).to("cuda")
        d_score = torch.zeros(max(pk["n"], 1), dtype=torch.int32, device="cuda")
        eng.ps_run_device(pk, d_pssm, d_orf, d_score)
        assert np.array_equal(d_score.cpu().numpy()[: pk["n"]], want)
    finally:
        eng.close()


@pytest.mark.gpu
@need_ref
@pytest.mark.parametrize("go,ge", [(11, 1), (5, 2), (3, 3), (4, 0), (2, 5)])
def test_ps_band_kernel_matches_reference(go, ge):
    """Bands of at most 80 cells go to the 16-lane band kernel when go >= ge >= 0 (the others,
    and go < ge, to the wavefront kernel): 2000 candidates of every band width up to 39 and
    beyond, diagonals from far left of the ORF to far right, against the reference."""
    rng = np.random.default_rng(40 + go * 7 + ge)
    cands = []
    for q in range(2000):
        Lq = int(rng.integers(1, 300))
        pssm = rng.integers(-9, 8, size=(Lq, 22)).astype(np.int8)
        nq = int(rng.integers(1, 500))
        orf = rng.integers(0, 22, size=nq).astype(np.uint8)
        diag = int(rng.integers(-Lq - 60, nq + 60))
        if q % 2 == 0 and nq > 40 and Lq > 40:
            d0 = int(rng.integers(-Lq // 2, nq // 2))
            t = np.arange(Lq) + d0
            ok = (t >= 0) & (t < nq) & (rng.random(Lq) < 0.8)
            orf[t[ok]] = np.argmax(pssm[np.arange(Lq)[ok]], axis=1).astype(np.uint8)
            diag = d0 + int(rng.integers(-3, 4))
        band = int(rng.choice([1, 2, 8, 16, 32, 32, 39, 40, 0]))
        cands.append((pssm, orf, diag, band))
    eng = L.Engine(0)
    try:
        got = eng.ps_gapped(cands, go, ge)
    finally:
        eng.close()
    want = np.array([O.ref_ps_gapped(p, o, d, b, go, ge) for p, o, d, b in cands])
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, [(int(i), cands[i][0].shape[0], cands[i][1].size, cands[i][2], cands[i][3], int(got[i]),
                            int(want[i])) for i in bad[:5]]
