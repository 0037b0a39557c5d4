"""Profile HMM tables for the integer profile DP: HMMER3 text in, the reference's
int16 tables out, plus seeded synthetic Plan7 profiles and regions.

``parse_hmmer3`` restates the numeric conversions of the reference parser
mp_hmm_read1 (hmm.c:112-195): every score is -2*x of the file's negative natural
log probability, clamped to +-32767 and rounded half-to-even (lrint, hmm.c:46-58),
"*" reads as -32768; each position's 20 match emissions are shifted so that the
best one is +4, with the int16 wrap of the reference; the 7 transitions of a
position are the second line after its match line.  ``codon_alpha`` is the
reference's ns_tab_codon remapped to the HMMER alphabet (hmm.c:229-250): the
HMMER column of the amino acid a codon encodes, 20 for a stop codon.

``synthetic_profiles`` draws Plan7 profiles for the HMM benchmark shape: match
lengths uniform in [m_min, m_max], match emissions Dirichlet-perturbed around an
amino-acid background and transitions around M->M = 0.95.  BLOSUM62's own
background frequencies are not in the reference; its HMMER p7 background
(hmm.c:28-31) is used in their place.
"""
from __future__ import annotations

import math
import re

import numpy as np

from .abi import AA_I2C, CODE1
from .workload import P7_BG, random_dna, reverse_translate

ALPHABET = "ACDEFGHIKLMNPQRSTVWY"  # HMMER match-emission column order (hmm.c:27)


def codon_alpha(code: str = CODE1) -> np.ndarray:
    """codon index (b0<<4|b1<<2|b2, ACGT = 0123) -> HMMER column, 20 = stop (no emission)."""
    out = np.full(64, 20, dtype=np.uint8)
    for i in range(64):
        aa = code[i]
        if aa in ALPHABET:
            out[i] = ALPHABET.index(aa)
    return out


def _score(tok: str) -> int:
    """parse_score (hmm.c:46-58)."""
    if tok == "*":
        return -32768
    try:
        x = float(tok)
    except ValueError:
        return -32768
    x = -2.0 * x
    x = min(max(x, -32767.0), 32767.0)
    return int(round(x))  # round half to even, as lrint in the default rounding mode


_POS = re.compile(r"[+-]?\d+\s")


def _i16(v: int) -> int:
    return ((v + 32768) & 0xFFFF) - 32768


def parse_hmmer3(text: str):
    """All profiles of a HMMER3 text: list of dicts name, m, emit (m x 20 int16), trans (m x 7 int16)."""
    out = []
    lines = text.splitlines()
    k = 0
    while k < len(lines):
        name, m, emit, trans, pos, in_hmm = None, 0, None, None, 0, False
        while k < len(lines):
            line = lines[k]
            k += 1
            data = line.lstrip()
            if line.startswith("NAME"):
                name = line[4:].split()[0]
            elif line.startswith("LENG"):
                m = int(line[4:].split()[0])
                emit = np.zeros((m, 20), dtype=np.int16)
                trans = np.zeros((m, 7), dtype=np.int16)
            elif line.startswith("HMM") and len(line) > 3 and line[3].isspace():
                in_hmm = True
            elif in_hmm and line.startswith("/"):
                break
            elif in_hmm and _POS.match(data + "\n"):  # is_position_line (hmm.c:92-97)
                if data[0] == "0":
                    k += 2
                    continue
                tok = data.split()
                row = [_score(t) for t in tok[1:21]]
                best = max(row)
                emit[pos] = [_i16(v - best + 4) for v in row]
                pos += 1
                if k + 1 >= len(lines):
                    break
                tline = lines[k + 1].split()
                k += 2
                if len(tline) >= 7:
                    trans[pos - 1] = [_score(t) for t in tline[:7]]
        if m == 0 or pos != m:
            break
        out.append({"name": name or "hmm_query", "m": m, "emit": emit, "trans": trans})
    return out


def consensus(emit) -> bytes:
    """A profile's consensus as the parser derives it (hmm.c:181-189): per match state the
    HMMER letter of its largest emission, the first column among equal ones.  An HMM-profile
    query is mapped as this sequence (map.c:1184-1196)."""
    e = np.asarray(emit, dtype=np.int16).reshape(-1, 20)
    return bytes(ord(ALPHABET[int(j)]) for j in np.argmax(e, axis=1))


def _fmt(p: float) -> str:
    return "*" if p <= 0 else f"{-math.log(p):.5f}"


def synthetic_profiles(n: int, seed: int = 3, m_min: int = 50, m_max: int = 800, concentration: float = 20.0):
    """n Plan7 profiles as HMMER3 text and their match-emission probabilities (for sampling domains)."""
    rng = np.random.default_rng(seed)
    bg = P7_BG  # AA20 order of workload (ACDEFGHIKLMNPQRSTVWY), the same as ALPHABET
    texts, probs = [], []
    for q in range(n):
        m = int(rng.integers(m_min, m_max + 1))
        mat = rng.dirichlet(bg * concentration, size=m)
        ins = bg
        mm = np.clip(rng.normal(0.95, 0.02, size=m), 0.80, 0.995)
        mi = (1 - mm) * rng.uniform(0.3, 0.7, size=m)
        md = 1 - mm - mi
        im = np.clip(rng.normal(0.6, 0.1, size=m), 0.2, 0.95)
        dm = np.clip(rng.normal(0.7, 0.1, size=m), 0.2, 0.95)
        md[-1], dm[-1] = 0.0, 1.0  # no deletion out of the last position
        lines = [f"HMMER3/f [synthetic]", f"NAME  syn{q:04d}", f"LENG  {m}", "ALPH  amino",
                 "HMM          " + "        ".join(ALPHABET),
                 "            m->m     m->i     m->d     i->m     i->i     d->m     d->d",
                 "  COMPO   " + " ".join(_fmt(x) for x in bg),
                 "          " + " ".join(_fmt(x) for x in ins),
                 "          " + " ".join(_fmt(x) for x in (0.98, 0.01, 0.01, 0.6, 0.4, 1.0, 0.0))]
        for i in range(m):
            lines.append(f"{i + 1:7d} " + " ".join(_fmt(x) for x in mat[i]) + f" {i + 1} - - -")
            lines.append("          " + " ".join(_fmt(x) for x in ins))
            lines.append("          " + " ".join(_fmt(x) for x in (mm[i], mi[i], md[i], im[i], 1 - im[i], dm[i], 1 - dm[i])))
        lines.append("//")
        texts.append("\n".join(lines) + "\n")
        probs.append(mat)
    return texts, probs


_NT4 = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate("ACGT"):
    _NT4[ord(_c)] = _i
    _NT4[ord(_c.lower())] = _i


def nt4(seq: bytes) -> np.ndarray:
    return _NT4[np.frombuffer(seq, dtype=np.uint8)]


def regions(rng: np.random.Generator, probs: np.ndarray, n: int, len_min: int = 300, len_max: int = 3000,
            planted: float = 0.5, gc: float = 0.45):
    """n regions (nt4 codes, frame 0 at the start) of 45% GC sequence; a fraction carries a domain
    sampled from the profile's match emissions, reverse-translated in frame."""
    out = []
    for q in range(n):
        L = int(rng.integers(len_min, len_max + 1))
        s = random_dna(rng, L, gc)
        if rng.random() < planted:
            m = probs.shape[0]
            a, b = sorted(int(x) for x in rng.integers(0, m + 1, size=2))
            if b - a >= 10:
                cdf = np.cumsum(probs[a:b] / probs[a:b].sum(axis=1, keepdims=True), axis=1)
                pick = (rng.random(b - a)[:, None] > cdf).sum(axis=1).clip(0, 19)
                dom = "".join(ALPHABET[int(x)] for x in pick)
                cds = reverse_translate(rng, dom)
                start = 3 * int(rng.integers(0, max(1, (L - len(cds)) // 3)))
                s = (s[:start] + cds + s[start + len(cds):])[:max(L, start + len(cds))]
        out.append(nt4(s.encode()))
    return out


assert AA_I2C[:20] != ALPHABET  # the two alphabet orders differ: emissions are indexed in HMMER order


def genome_scan(probs, seed: int, genome_mb: float = 100.0, n_domains: int = 1000, slice_mb: float = 2.0,
                region_nt: int = 30000, overlap_nt: int = 2400, gc: float = 0.45):
    """The profile-HMM configuration's genome: genome_mb of 45% GC sequence (nt4 codes) with
    n_domains domains sampled from the profiles' match emissions, reverse-translated and planted
    on random strands; and the regions of a scan of its first slice_mb in six frames -- the slice
    and its reverse complement cut into region_nt windows overlapping by overlap_nt (a domain of
    up to 800 codons is inside one window), each window in frames 0, 1, 2.  Returns (nt4 regions
    concatenated, offsets, lengths, planted domains inside the slice)."""
    rng = np.random.default_rng(seed)
    n = int(genome_mb * 1e6)
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    g = rng.choice(4, size=n, p=p).astype(np.uint8)
    comp = np.array([3, 2, 1, 0, 4], np.uint8)
    slice_nt = min(n, int(slice_mb * 1e6))
    inside = 0
    for _ in range(n_domains):
        k = int(rng.integers(0, len(probs)))
        pr = probs[k]
        m = pr.shape[0]
        a, b = sorted(int(x) for x in rng.integers(0, m + 1, size=2))
        if b - a < 10:
            a, b = 0, m
        cdf = np.cumsum(pr[a:b] / pr[a:b].sum(axis=1, keepdims=True), axis=1)
        pick = (rng.random(b - a)[:, None] > cdf).sum(axis=1).clip(0, 19)
        cds = nt4(reverse_translate(rng, "".join(ALPHABET[int(x)] for x in pick)).encode())
        pos = int(rng.integers(0, n - len(cds)))
        if rng.random() < 0.5:
            cds = comp[cds[::-1]]
        g[pos:pos + len(cds)] = cds
        inside += pos + len(cds) <= slice_nt
    fwd = g[:slice_nt]
    rev = comp[fwd[::-1]]
    parts, offs, lens = [], [], []
    pos = 0
    step = region_nt - overlap_nt
    for strand in (fwd, rev):
        for st in range(0, max(1, len(strand) - overlap_nt), step):
            w = strand[st:st + region_nt]
            for f in range(3):
                r = w[f:]
                parts.append(r)
                offs.append(pos)
                lens.append(len(r))
                pos += len(r)
    return (np.concatenate(parts), np.array(offs, np.int32), np.array(lens, np.int32), inside)
