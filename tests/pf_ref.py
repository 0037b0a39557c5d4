"""Numpy restatement of the learned prefilter's candidate features (the checker of
protlocus_b200/csrc/pffeat.cu; test infrastructure only).

For a candidate (protein, window on the strand the DP reads):
  * protein aa 3-mers -> 256 bins, window codon-end 3-mers (every position ends a
    codon, so all three frames) -> 256 bins, each scaled by 256 / (number of valid
    3-mers) in float32;
  * anchors: window codon ends whose aa 5-mer occurs in the protein, paired with the
    smallest protein end position of that 5-mer;
  * chain: anchors sorted by (window position, protein position); f[j] = 1 + the
    best f[k] over k < j with both coordinates smaller and a nucleotide gap of at
    least 3x the residue gap minus 60 (ties: the largest k); the chain ends at the
    first j with the largest f;
  * 20 scalars of the anchors and the chain, as float32, then bf16 (round to nearest
    even).
Residues and codons use the ProtLocus tables (protlocus_b200.abi.make_tables).
"""
from __future__ import annotations

import numpy as np

MAXA = 1024
FDIM = 576


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> bf16 (round to nearest even), returned as float32 values."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32)


def h3(code: int) -> int:
    return ((code * 40503) & 0xFFFFFFFF) >> 8 & 255


def features(nt: bytes, aa: bytes, nt4: np.ndarray, aa20: np.ndarray, codon: np.ndarray):
    """(feature row float32[576] after bf16 rounding, chain ints [4], anchor count)."""
    nl, al = len(nt), len(aa)
    bins = np.zeros(512, dtype=np.int64)
    r = np.array([aa20[c] for c in aa], dtype=np.int64)
    r = np.where(r < 20, r, -1)
    tot_p = 0
    kmers: dict[int, int] = {}
    for p in range(al):
        if p >= 2 and min(r[p - 2], r[p - 1], r[p]) >= 0:
            bins[h3(int(r[p - 2] * 400 + r[p - 1] * 20 + r[p]))] += 1
            tot_p += 1
        if p >= 4 and min(r[p - 4:p + 1]) >= 0:
            code = 0
            for x in r[p - 4:p + 1]:
                code = code * 20 + int(x)
            kmers.setdefault(code, p)
    # residue of the codon ending at each position
    n4 = np.array([nt4[c] for c in nt], dtype=np.int64)
    res = np.full(nl, -1, dtype=np.int64)
    for p in range(2, nl):
        a, b, c = n4[p - 2], n4[p - 1], n4[p]
        if max(a, b, c) <= 3:
            x = int(codon[a * 16 + b * 4 + c])
            res[p] = x if x < 20 else -1
    tot_w = 0
    anchors = []
    for p in range(nl):
        if p < 8 or min(res[p], res[p - 3], res[p - 6]) < 0:
            continue
        bins[256 + h3(int(res[p - 6] * 400 + res[p - 3] * 20 + res[p]))] += 1
        tot_w += 1
        if p < 14 or min(res[p - 9], res[p - 12]) < 0:
            continue
        code = 0
        for x in (res[p - 12], res[p - 9], res[p - 6], res[p - 3], res[p]):
            code = code * 20 + int(x)
        if code in kmers:
            anchors.append((p, kmers[code]))
    na_all = len(anchors)
    assert na_all <= MAXA, "the restatement covers candidates with at most 1024 anchors"
    anchors.sort()
    na = len(anchors)
    f = [0] * na
    prev = [-1] * na
    for j in range(na):
        pj, rj = anchors[j]
        best, bk = 0, -1
        for k in range(j):
            pk, rk = anchors[k]
            if pk < pj and rk < rj and (pj - pk) >= 3 * (rj - rk) - 60 and f[k] >= best:
                best, bk = f[k], k
        f[j] = best + 1 if bk >= 0 else 1
        prev[j] = bk
    jb, fb = -1, 0
    for j in range(na):
        if f[j] > fb:
            fb, jb = f[j], j
    length = fc = cov = 0
    fp = lp = fr = lr = -1
    nxt = None
    j = jb
    while j >= 0:
        pj, rj = anchors[j]
        if length == 0:
            lp, lr = pj, rj
        else:
            if nxt[0] % 3 != pj % 3:
                fc += 1
            cov += min(5, nxt[1] - rj)
        fp, fr, nxt = pj, rj, (pj, rj)
        length += 1
        j = prev[j]
    if length:
        cov += 5
    F = np.zeros(FDIM, dtype=np.float32)
    f32 = np.float32
    sp = f32(256.0) / f32(max(1, tot_p))
    sw = f32(256.0) / f32(max(1, tot_w))
    F[:256] = bins[:256].astype(np.float32) * sp
    F[256:512] = bins[256:].astype(np.float32) * sw
    fnl, fal = f32(max(nl, 1)), f32(max(al, 1))
    lg = (lambda x: np.log2(f32(1.0) + f32(x)))
    v = np.zeros(20, dtype=np.float32)
    v[0] = lg(al) / f32(12)
    v[1] = lg(nl) / f32(16)
    v[2] = lg(na_all) / f32(10)
    v[3] = f32(length) / f32(max(1, al - 4))
    v[4] = lg(length) / f32(10)
    v[5] = f32(cov) / fal
    if length:
        v[6] = f32(lp - fp) / fnl
        v[7] = f32(fp) / fnl
        v[8] = f32(lp) / fnl
        v[9] = f32(fr) / fal
        v[10] = f32(lr) / fal
        v[12] = lg(lp - fp) / f32(16)
        v[13] = min(max(f32(fp - 3 * fr - 2) / fnl, f32(-1)), f32(2))
        v[14] = min(max(f32(lp + 3 * (al - 1 - lr)) / fnl, f32(-1)), f32(2))
    v[11] = f32(fc) / f32(8)
    v[15] = f32(min(na_all, 65535)) * f32(1000) / fnl / f32(8)
    v[16] = f32(length) / f32(max(1, na))
    v[17] = 1.0
    v[18] = 1.0 if length >= 2 else 0.0
    v[19] = 1.0 if na_all > MAXA else 0.0
    F[512:532] = v
    chain = [fp, lp, fr, lr] if length else [-1, -1, -1, -1]
    return bf16_round(F), chain, na_all, length
