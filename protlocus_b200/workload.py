"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is used by the reference for this path; these generators
stand in for it.

* ``single_locus`` -- one protein (default 500 aa) drawn i.i.d. from an
  amino-acid background, reverse-translated with uniform synonymous codons
  (genetic code 1), mutated to a target divergence with BLOSUM62-weighted
  substitutions (weights proportional to exp(lambda*s), lambda = ln(2)/2,
  BLOSUM62's half-bit scale), given single-nucleotide frameshifts, split by
  GT..AG introns with log-uniform lengths and embedded in a uniform random
  ACGT window.  BLOSUM62's own background frequencies are not in the
  reference; the HMMER p7 amino-acid background (the only background the
  reference ships, hmm.c:28-31) is used in their place.
* ``batch_pairs`` -- many such loci: protein lengths log-normal (median 350,
  clipped to 50-2500), intron counts Poisson(4) with log-normal lengths
  (median 150, cap 20 kb), genomic windows uniform in 1-50 kb (never shorter
  than the gene plus 100 nt of flank on each side).  Both strands are
  searched: every pair contributes its window and the reverse complement of
  that window (the reverse-strand DP of ntseq.c:92-117), so n pairs give 2n
  DP jobs.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import AA_I2C, BLOSUM62, CODE1

AA20 = "ACDEFGHIKLMNPQRSTVWY"  # HMMER column order
P7_BG = np.array([0.0787945, 0.0151600, 0.0535222, 0.0668298, 0.0397062, 0.0695071, 0.0229198,
                  0.0590092, 0.0594422, 0.0963728, 0.0237718, 0.0414386, 0.0482904, 0.0395639,
                  0.0540978, 0.0683364, 0.0540687, 0.0673417, 0.0114135, 0.0304133])
P7_BG = P7_BG / P7_BG.sum()
LAMBDA = math.log(2.0) / 2.0

_NT = "ACGT"
_CODONS: dict[str, list[str]] = {}
for _i in range(64):
    _aa = CODE1[_i]
    _c = _NT[_i >> 4] + _NT[(_i >> 2) & 3] + _NT[_i & 3]
    _CODONS.setdefault(_aa, []).append(_c)

# substitution distribution per residue: P(b | a) ~ exp(lambda * s(a, b)), b != a
_idx = [AA_I2C.index(c) for c in AA20]
_SUB = np.zeros((20, 20))
for _a in range(20):
    for _b in range(20):
        if _a != _b:
            _SUB[_a, _b] = math.exp(LAMBDA * BLOSUM62[_idx[_a], _idx[_b]])
    _SUB[_a] /= _SUB[_a].sum()

_COMP = bytes.maketrans(b"ACGTNacgtn", b"TGCANtgcan")


def revcomp(s: bytes) -> bytes:
    return s.translate(_COMP)[::-1]


_AA20_B = np.frombuffer(AA20.encode(), dtype=np.uint8)
_NT_B = np.frombuffer(b"ACGT", dtype=np.uint8)
_SUB_CDF = np.cumsum(_SUB, axis=1)
_AA_IDX = np.full(256, 0, dtype=np.int64)
for _k, _ch in enumerate(AA20):
    _AA_IDX[ord(_ch)] = _k
# codon choices per residue index: table [20, 6] of codon strings padded by repetition
_CODON_TAB = np.array([[(_CODONS[a] * 6)[j] for j in range(6)] for a in AA20])
_CODON_N = np.array([len(_CODONS[a]) for a in AA20])


def random_protein(rng: np.random.Generator, n: int) -> str:
    return _AA20_B[rng.choice(20, size=n, p=P7_BG)].tobytes().decode()


def mutate(rng: np.random.Generator, prot: str, divergence: float) -> str:
    idx = _AA_IDX[np.frombuffer(prot.encode(), dtype=np.uint8)]
    hit = rng.random(len(idx)) < divergence
    u = rng.random(len(idx))
    new = (u[:, None] > _SUB_CDF[idx]).sum(axis=1).clip(0, 19)
    out = np.where(hit, new, idx)
    return _AA20_B[out].tobytes().decode()


def reverse_translate(rng: np.random.Generator, prot: str) -> str:
    idx = _AA_IDX[np.frombuffer(prot.encode(), dtype=np.uint8)]
    pick = (rng.random(len(idx)) * _CODON_N[idx]).astype(np.int64)
    return "".join(_CODON_TAB[idx, pick].tolist())


def random_dna(rng: np.random.Generator, n: int, gc: float = 0.5) -> str:
    p = [(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2]
    return _NT_B[rng.choice(4, size=n, p=p)].tobytes().decode()


def _intron(rng: np.random.Generator, length: int) -> str:
    length = max(length, 8)
    return "GT" + random_dna(rng, length - 4) + "AG"


def build_gene(rng: np.random.Generator, prot: str, *, divergence: float, n_frameshift: int,
               intron_lengths: list[int]) -> str:
    """Coding sequence of a mutated copy of `prot` with frameshifts and introns."""
    target = mutate(rng, prot, divergence)
    cds = list(reverse_translate(rng, target))
    for _ in range(n_frameshift):
        p = int(rng.integers(3, max(4, len(cds) - 3)))
        if rng.random() < 0.5:
            del cds[p]
        else:
            cds.insert(p, _NT[rng.integers(4)])
    cds = "".join(cds)
    if intron_lengths:
        cuts = sorted(int(x) for x in rng.choice(np.arange(6, max(7, len(cds) - 6)),
                                                 size=min(len(intron_lengths), max(1, len(cds) - 12)),
                                                 replace=False))
        parts, prev = [], 0
        for c, L in zip(cuts, intron_lengths):
            parts.append(cds[prev:c])
            parts.append(_intron(rng, L))
            prev = c
        parts.append(cds[prev:])
        cds = "".join(parts)
    return cds


def single_locus(seed: int = 0, al: int = 500, window: int = 20000, divergence: float = 0.25,
                 n_frameshift: int = 2, n_intron: int = 3):
    """One protein/window pair shaped like the single-DP configuration."""
    rng = np.random.default_rng(seed)
    prot = random_protein(rng, al)
    introns = [int(round(math.exp(rng.uniform(math.log(80), math.log(2000))))) for _ in range(n_intron)]
    gene = build_gene(rng, prot, divergence=divergence, n_frameshift=n_frameshift, intron_lengths=introns)
    flank = max(0, window - len(gene))
    left = int(rng.integers(0, flank + 1))
    nt = random_dna(rng, left) + gene + random_dna(rng, flank - left)
    return nt.encode(), prot.encode()


def batch_pairs(n_pairs: int, seed: int = 1, *, al_median: float = 350.0, al_sigma: float = 0.6,
                al_min: int = 50, al_max: int = 2500, win_min: int = 1000, win_max: int = 50000,
                intron_lambda: float = 4.0, intron_median: float = 150.0, intron_sigma: float = 0.8,
                intron_cap: int = 20000, divergence: float = 0.25, both_strands: bool = True):
    """List of (nt, protein) DP jobs shaped like the batched configuration (2 per pair with both strands)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n_pairs):
        al = int(np.clip(round(math.exp(rng.normal(math.log(al_median), al_sigma))), al_min, al_max))
        prot = random_protein(rng, al)
        k = int(rng.poisson(intron_lambda))
        introns = [int(min(intron_cap, max(20, round(math.exp(rng.normal(math.log(intron_median), intron_sigma))))))
                   for _ in range(k)]
        gene = build_gene(rng, prot, divergence=divergence, n_frameshift=int(rng.integers(0, 3)),
                          intron_lengths=introns)
        w = int(rng.integers(win_min, win_max + 1))
        w = max(w, len(gene) + 200)
        flank = w - len(gene)
        left = int(rng.integers(100, flank - 99))
        nt = (random_dna(rng, left) + gene + random_dna(rng, flank - left)).encode()
        jobs.append((nt, prot.encode()))
        if both_strands:
            jobs.append((revcomp(nt), prot.encode()))
    return jobs


def random_pair(rng: np.random.Generator, max_al: int = 60, n_rate: float = 0.01):
    """Small unstructured pair (protein <= max_al, window <= 3*al+120) for exhaustive sweeps."""
    al = int(rng.integers(1, max_al + 1))
    nl = int(rng.integers(3, 3 * al + 121))
    aa = random_protein(rng, al).encode()
    nt = np.where(rng.random(nl) < n_rate, ord("N"), _NT_B[rng.integers(0, 4, size=nl)]).astype(np.uint8).tobytes()
    return nt, aa


def random_ss(rng: np.random.Generator, nl: int, rate: float = 0.2) -> bytes:
    """Splice-score track like the reference's tests: mostly unset (0xff), some donor/acceptor scores."""
    val = ((rng.integers(0, 128, size=nl) << 1) | rng.integers(0, 2, size=nl)) & 0xff
    return np.where(rng.random(nl) < rate, val, 0xff).astype(np.uint8).tobytes()


def ext_requests(n: int, seed: int = 2, *, win_min: int = 64, win_max: int = 256, divergence: float = 0.25,
                 intron_lambda: float = 0.5, intron_median: float = 150.0, intron_sigma: float = 0.8,
                 slack_min: int = 60, slack_max: int = 600):
    """Extension requests shaped like the seed-extension configuration: protein windows of
    64-256 aa (the request window the reference extends over), nucleotide windows of
    3x the protein window plus slack.  A mutated, possibly spliced and frameshifted copy
    of the protein's anchored part (30-100 % of the window, from the anchor outwards)
    starts at the anchor end of the window; random sequence follows, where the x-drop
    ends the DP.  Alternate requests extend right (anchor at the start) and left (anchor
    at the end).  Returns a list of (nt, protein, flag)."""
    from .abi import NS_F_EXT_LEFT, NS_F_EXT_RIGHT
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        L = int(rng.integers(win_min, win_max + 1))
        prot = random_protein(rng, L)
        m = int(rng.integers(max(8, int(0.3 * L)), L + 1))
        k = int(rng.poisson(intron_lambda))
        introns = [int(max(20, round(math.exp(rng.normal(math.log(intron_median), intron_sigma))))) for _ in range(k)]
        left = bool(q & 1)
        part = prot[L - m:] if left else prot[:m]
        gene = build_gene(rng, part, divergence=divergence, n_frameshift=int(rng.integers(0, 2)), intron_lengths=introns)
        tail = random_dna(rng, max(0, 3 * L + int(rng.integers(slack_min, slack_max + 1)) + sum(introns) - len(gene)))
        nt = tail + gene if left else gene + tail
        out.append((nt.encode(), prot.encode(), NS_F_EXT_LEFT if left else NS_F_EXT_RIGHT))
    return out
