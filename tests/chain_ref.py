"""Restatement of mp_chain's fill loop (chain.c:160-208) in Python (test infrastructure
only): the score f, predecessor p and peak v of every anchor, in the reference's order
of operations, with float32 rounding after every float operation as the CPU build
does.  tests/test_chain_host.py feeds its f and p to the library's host backtrack
(pl_chain_finish) and compares the chains with the reference's mp_chain; the device
fill is compared with it in tests/test_gpu_chain.py.
"""
from __future__ import annotations

import numpy as np

INT32_MIN = -(1 << 31)
BLOCK_BONUS = 2  # MP_BLOCK_BONUS (protlocus.h:47)
f32 = np.float32


def log2_approx(x: float) -> np.float32:
    """mppriv.h:143-151 for x >= 2: exponent - 128 plus a quadratic in the mantissa."""
    i = int(np.array([x], dtype=np.float32).view(np.uint32)[0])
    e = f32(((i >> 23) & 255) - 128)
    i = (i & ~(255 << 23) & 0xFFFFFFFF) + (127 << 23)
    m = np.array([i], dtype=np.uint32).view(np.float32)[0]
    q = f32(f32(f32(-0.34484843) * m) + f32(2.02466578))
    q = f32(f32(q * m) - f32(0.67487759))
    return f32(e + q)


def _i32(x: int) -> int:
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x >= 1 << 31 else x


def score(ai: int, aj: int, o: dict) -> int:
    """comput_sc (chain.c:112-152)."""
    dq = _i32(_i32(ai) - _i32(aj))
    dq3 = dq * 3
    if dq <= 0 or dq3 > o["max_dist_x"] or dq > o["max_dist_y"]:
        return INT32_MIN
    bbit, kmer = o["bbit"], o["kmer"]
    if bbit > 0:
        bs = 1 << bbit
        dr3 = _i32(((ai >> 32) - (aj >> 32)) << bbit)
        if dr3 - bs <= dq3 <= dr3 + bs:
            dd = dd_signed = 0
        elif dq3 < dr3 - bs:
            dd = dr3 - bs - dq3
            dd_signed = -dd
        else:
            dd = dq3 - (dr3 + bs)
            dd_signed = dd
    else:
        dr3 = _i32((ai >> 32) - (aj >> 32))
        if dr3 == 0:
            return INT32_MIN
        dd = abs(dr3 - dq3)
        dd_signed = dq3 - dr3
    if dd > o["bw"]:
        return INT32_MIN
    if bbit > 0:
        sc = min(kmer, dq)
    elif kmer <= dq and kmer * 3 <= dr3:
        sc = kmer
    else:
        dr = dr3 // 3 if dr3 >= 0 else -(-dr3 // 3)  # C division truncates toward zero
        q = dr3 - dr * 3
        sc = min(min(dr, dq), kmer)
        if q != 0:
            sc -= 1
    if dd > 0:
        lin = f32(f32(dd) * f32(0.33334))
        lg = f32(f32(f32(o["coef"]) * f32(log2_approx(float(dd + 1)) - f32(1.0))) + f32(1.0)) if dd >= 2 else f32(dd)
        if o["is_spliced"] and dd_signed < 0:
            sc -= int(min(lin, lg))
        else:
            sc -= int(f32(lin + lg))
    if bbit > 0 and (ai >> 32) == (aj >> 32) and dd == 0:
        sc += BLOCK_BONUS
    return sc


def normalise(o: dict) -> dict:
    o = dict(o)
    if o["max_dist_x"] < o["bw"]:
        o["max_dist_x"] = o["bw"]
    if o["max_dist_y"] < o["bw"] and not o["is_spliced"]:
        o["max_dist_y"] = o["bw"]
    return o


def fill(a, o: dict):
    """f, p, v (int32 arrays) of the anchors a (uint64, sorted)."""
    o = normalise(o)
    a = [int(x) for x in a]
    n = len(a)
    f = np.zeros(n, np.int32)
    p = np.full(n, -1, np.int32)
    v = np.zeros(n, np.int32)
    t = np.zeros(n, np.int64)
    st, hi, hf = 0, -1, 0
    for i in range(n):
        max_j, max_f, n_skip = -1, o["kmer"], 0
        while st < i and ((a[i] >> 32) - (a[st] >> 32)) << o["bbit"] > o["max_dist_x"]:
            st += 1
        if hi >= 0 and hi >= st:
            s = score(a[i], a[hi], o)
            s = hf + s
            if s > max_f:
                max_f, max_j = s, hi
        else:
            hf, hi = 0, -1
        if i - st > o["max_iter"]:
            st = i - o["max_iter"]
        for j in range(i - 1, st - 1, -1):
            s = score(a[i], a[j], o)
            if s == INT32_MIN:
                continue
            s += int(f[j])
            if s > max_f:
                max_f, max_j = s, j
                if n_skip > 0:
                    n_skip -= 1
            elif t[j] == i:
                n_skip += 1
                if n_skip > o["max_skip"]:
                    break
            if p[j] >= 0:
                t[p[j]] = i
        f[i], p[i] = max_f, max_j
        v[i] = v[max_j] if max_j >= 0 and v[max_j] > max_f else max_f
        if hf < max_f:
            hf, hi = max_f, i
    return f, p, v
