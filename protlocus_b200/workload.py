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


def pack_nt4(seq: np.ndarray) -> np.ndarray:
    """4-bit packed nucleotide codes, two per byte, low nibble first (ntseq.c:66-69)."""
    s = np.asarray(seq, dtype=np.uint8)
    if s.size & 1:
        s = np.concatenate([s, np.zeros(1, np.uint8)])
    return (s[0::2] | (s[1::2] << 4)).astype(np.uint8)


GAPLESS_CAND_DTYPE = np.dtype([("target_offset", "<i8"), ("target_length", "<i8"), ("query_offset", "<i8"),
                               ("query_length", "<i4"), ("anchor_offset", "<i4"), ("anchor_count", "<i4"),
                               ("reverse", "<i4")])
GAPLESS_ANCHOR_DTYPE = np.dtype([("target_block", "<i8"), ("query_end", "<i4"), ("reserved", "<i4")])


def gapless_workload(n_genes: int, genome_len: int, n_candidates: int, seed: int = 4, *, n_contigs: int = 64,
                     al: int = 500, divergence: float = 0.25, n_intron: int = 3, frac_true: float = 0.3,
                     anchors_per_cand: int = 8, kmer: int = 6, bbit: int = 8, gc: float = 0.45,
                     fixed_anchors: bool = False):
    """Inputs of the gapless prefilter shaped like the seed-extension configuration: a genome
    of n_contigs contigs at 45% GC with n_genes planted genes (a 25%-divergent copy of an
    al-residue protein split by n_intron GT..AG introns of 80-2000 bp, on either strand),
    the n_genes source proteins as queries, and n_candidates candidates of 1 to
    anchors_per_cand anchors each (exactly anchors_per_cand with fixed_anchors, as the
    mapper's evenly spaced pick gives for chains of 8 or more anchors, map.c:474-507).  A fraction frac_true of the candidates sits on its
    protein's planted gene with anchors on the true codon positions (target_block = the
    oriented 2^bbit block holding the anchor's last codon base, give or take six bases);
    the others are decoys on a random contig and strand.  Frameshifts are left out so that
    anchor positions are exact.  Returns numpy arrays laid out as
    ns_gpu_gapless_candidate_t / ns_gpu_gapless_anchor_t (nasw.h:157-167)."""
    from .abi import make_tables
    rng = np.random.default_rng(seed)
    nt4, aa20, _ = make_tables()
    ctg_len = np.full(n_contigs, genome_len // n_contigs, dtype=np.int64)
    ctg_len[: genome_len % n_contigs] += 1
    ctg_off = np.zeros(n_contigs, dtype=np.int64)
    ctg_off[1:] = np.cumsum(ctg_len[:-1])
    p = [(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2]
    genome = rng.choice(4, size=genome_len, p=p).astype(np.uint8)
    prots, genes = [], []  # genes: (contig, reverse, codon-end per residue in oriented coordinates)
    slot = max(1, genome_len // max(1, n_genes))
    for g in range(n_genes):
        prot = random_protein(rng, al)
        cds = reverse_translate(rng, mutate(rng, prot, divergence))
        cuts = np.sort(rng.choice(np.arange(1, al), size=min(n_intron, al - 1), replace=False))
        ilen = [int(round(math.exp(rng.uniform(math.log(80), math.log(2000))))) for _ in cuts]
        parts, ends, prev, shift = [], np.zeros(al, dtype=np.int64), 0, 0
        for c, L in zip(list(cuts) + [al], ilen + [0]):
            parts.append(cds[3 * prev:3 * c])
            ends[prev:c] = np.arange(prev, c) * 3 + 2 + shift
            if L:
                parts.append(_intron(rng, L))
                shift += max(L, 8)
            prev = c
        gene = nt4[np.frombuffer("".join(parts).encode(), dtype=np.uint8)]
        G = gene.size
        start = g * slot + int(rng.integers(0, max(1, slot - G)))
        k = int(np.searchsorted(ctg_off, start, side="right") - 1)
        if start + G > ctg_off[k] + ctg_len[k]:
            start = int(ctg_off[k] + max(0, ctg_len[k] - G - 1))
        local = start - int(ctg_off[k])
        rev = bool(rng.random() < 0.5)
        if rev:  # the reverse complement is stored; read in reverse orientation it is the gene
            genome[start:start + G] = 3 - gene[::-1]
            ostart = int(ctg_len[k]) - (local + G)
        else:
            genome[start:start + G] = gene
            ostart = local
        prots.append(prot.encode())
        genes.append((k, rev, ends + ostart))
    q_off = np.zeros(n_genes, dtype=np.int64)
    q_off[1:] = np.cumsum([len(x) for x in prots[:-1]])
    queries = aa20[np.frombuffer(b"".join(prots), dtype=np.uint8)]
    cand = np.zeros(n_candidates, dtype=GAPLESS_CAND_DTYPE)
    anc = np.zeros(n_candidates * anchors_per_cand, dtype=GAPLESS_ANCHOR_DTYPE)
    na = 0
    for ci in range(n_candidates):
        gi = int(rng.integers(0, n_genes))
        k, rev, ends = genes[gi]
        true = rng.random() < frac_true
        if not true:
            k, rev = int(rng.integers(0, n_contigs)), bool(rng.random() < 0.5)
        cnt = anchors_per_cand if fixed_anchors else int(rng.integers(1, anchors_per_cand + 1))
        qe = np.sort(rng.choice(np.arange(kmer - 1, al), size=cnt, replace=False))
        pos = ends[qe] - int(rng.integers(0, 7)) if true else rng.integers(0, int(ctg_len[k]), size=cnt)
        cand[ci] = (ctg_off[k], ctg_len[k], q_off[gi], al, na, cnt, int(rev))
        anc["target_block"][na:na + cnt] = (np.maximum(pos, 0) >> bbit) << bbit
        anc["query_end"][na:na + cnt] = qe
        na += cnt
    return {"packed": pack_nt4(genome), "bases": genome_len, "queries": queries.astype(np.uint8),
            "candidates": cand, "anchors": anc[:na].copy(), "block_width": 1 << bbit, "kmer": kmer,
            "contig_offsets": ctg_off, "contig_lengths": ctg_len}


def genome_fasta(n_genes: int, seed: int = 5, *, n_contigs: int = 4, contig_len: int = 200_000,
                 al_min: int = 80, al_max: int = 600, divergence: float = 0.2, n_decoys: int = 4,
                 max_frameshift: int = 1, gc: float = 0.45,
                 proteins: list[str] | None = None) -> tuple[str, str]:
    """A genome and a protein set for running the whole mapping program: n_contigs contigs of
    contig_len bases at the given GC, with n_genes planted genes (a `divergence`-mutated copy of
    a random al_min..al_max residue protein, 0..max_frameshift frameshifts and 0-4 GT..AG
    introns of 60-1500 bp, either strand, one gene per slot so they never overlap), and a
    protein FASTA with the n_genes source proteins followed by n_decoys unrelated proteins.
    With `proteins` given, those are planted instead of random ones (n_genes = their number).
    Returns (genome FASTA text, protein FASTA text)."""
    rng = np.random.default_rng(seed)
    if proteins is not None:
        n_genes = len(proteins)
    contigs = [list(random_dna(rng, contig_len, gc)) for _ in range(n_contigs)]
    per = max(1, -(-n_genes // n_contigs))
    slot = contig_len // per
    prots = []
    for g in range(n_genes):
        prot = proteins[g] if proteins is not None else random_protein(rng, int(rng.integers(al_min, al_max + 1)))
        introns = [int(round(math.exp(rng.uniform(math.log(60), math.log(1500)))))
                   for _ in range(int(rng.integers(0, 5)))]
        gene = build_gene(rng, prot, divergence=divergence, n_frameshift=int(rng.integers(0, max_frameshift + 1)),
                          intron_lengths=introns)
        if rng.random() < 0.5:
            gene = revcomp(gene.encode()).decode()
        c, s = g % n_contigs, g // n_contigs
        room = slot - len(gene)
        if room < 2:
            continue
        start = s * slot + int(rng.integers(1, room))
        contigs[c][start:start + len(gene)] = list(gene)
        prots.append((f"gene{g}", prot))
    for d in range(n_decoys):
        prots.append((f"decoy{d}", random_protein(rng, int(rng.integers(al_min, al_max + 1)))))

    def fasta(records):
        out = []
        for name, seq in records:
            out.append(f">{name}\n")
            out.extend(seq[i:i + 80] + "\n" for i in range(0, len(seq), 80))
        return "".join(out)

    genome = fasta([(f"ctg{c}", "".join(contigs[c])) for c in range(n_contigs)])
    return genome, fasta(prots)


def chain_anchors(n_q: int, seed: int = 7, *, genome_len: int = 100_000_000, bbit: int = 8, al_median: float = 350.0,
                  hit_rate: float = 0.15, n_noise: float = 40.0, paralog: float = 0.5):
    """Per-query seed anchors for mp_chain, as the coarse mapping collects them (blockId << 32 |
    queryPos, sorted): for each query protein (length log-normal around al_median, 50-2500 aa)
    the k-mer hits of its planted gene (exons split by Poisson(4) introns of log-normal length,
    median 150 bp, at most 20 kb; a hit per residue with probability hit_rate), half the time
    a weaker paralogous copy elsewhere, and Poisson(n_noise) random hits over the genome.
    bbit = 0 gives nucleotide coordinates instead of blocks (the refinement's chaining)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_q):
        al = int(np.clip(rng.lognormal(math.log(al_median), 0.6), 50, 2500))
        anchors = []

        def gene(rate):
            n_exon = 1 + int(rng.poisson(4))
            cuts = np.sort(rng.choice(np.arange(1, al), size=min(n_exon - 1, al - 1), replace=False)) if al > 1 else []
            bounds = [0, *[int(c) for c in cuts], al]
            span = 3 * al + 20000 * n_exon
            g = int(rng.integers(0, max(1, genome_len - span)))
            for e in range(len(bounds) - 1):
                q0, q1 = bounds[e], bounds[e + 1]
                hit = rng.random(q1 - q0) < rate
                for q in np.nonzero(hit)[0]:
                    anchors.append(((g + 3 * int(q)) >> bbit) << 32 | (q0 + int(q)))
                g += 3 * (q1 - q0) + int(min(20000, rng.lognormal(math.log(150), 1.0)))

        gene(hit_rate)
        if rng.random() < paralog:
            gene(hit_rate / 3)
        for _ in range(int(rng.poisson(n_noise))):
            anchors.append((int(rng.integers(0, genome_len)) >> bbit) << 32 | int(rng.integers(0, al)))
        out.append(np.unique(np.array(anchors, dtype=np.uint64)))
    return out
