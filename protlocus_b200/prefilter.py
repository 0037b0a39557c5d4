"""Learned candidate prefilter: host side.

A chained candidate is a protein and the genomic window its chain spans, on one
strand.  The plain path runs the exact spliced DP (pl_splice_batch_device) over
every candidate window; a candidate "passes" when it survives the reference's
output test, mp_reg_will_output (map.c:442-468), applied per protein: among the
protein's aligned candidates ranked by score, within the first out_n, score > 0,
score >= out_sim x the best score and an aligned query span of at least
out_cov x the protein length (options.c:63-65: out_n 1000, out_sim 0.99,
out_cov 0.1).  A protein's locus (its planted gene) is reported when one of the
candidates on that gene -- its own window on either strand, or the partial window
cutting the gene -- passes.  The learned path computes
features on the device (pl_pf_features_device), scores them with a 4-layer BF16
MLP on the tensor cores (pl_pf_predict), drops candidates predicted to fail,
tightens the windows of the others to the predicted alignment span plus a
margin, and runs the same exact DP there; a kept candidate whose tightened DP
does not pass falls back to its full window.  Every reported alignment comes
from the exact DP; recall is measured against the plain path.

Training pairs are the plain path's own outcomes: label = pass, and for passing
candidates the first and last aligned codon of the plain alignment (CIGAR M ops)
as fractions of the window.  Recall is measured per locus: the share of the
loci the plain path reports that the learned path reports too.

Synthetic candidates (make_candidates) follow the batched configuration: per
protein (log-normal length, median 350 aa, 50-2500) one window of 1-50 kb holding
a 25%-divergent copy split by Poisson(4) introns (log-normal, median 150 bp, cap
20 kb) with 0-2 frameshifts; its candidates are that window on both strands, a
partial window cutting the gene, and five windows of other proteins' genes on a
random strand.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import lib as L
from . import workload as W
from .abi import NS_F_CIGAR, Options, SpliceJob, SpliceResult

FDIM = 576
JOB_DTYPE = np.dtype([("nt_off", "<i8"), ("aa_off", "<i8"), ("ss_off", "<i8"), ("nl", "<i4"), ("al", "<i4")])
RES_DTYPE = np.dtype([("score", "<i4"), ("n_cigar", "<i4"), ("cigar_off", "<i8"), ("mode", "<i4"), ("status", "<i4")])
KIND_OWN_PLUS, KIND_OWN_MINUS, KIND_PARTIAL, KIND_OTHER = 0, 1, 2, 3
OUT_N, OUT_SIM, OUT_COV = 1000, 0.99, 0.1  # the reference's output defaults (options.c:63-65)


def make_candidates(seed: int, n_prot: int = 4096, n_other: int = 5, *, win_min: int = 1000, win_max: int = 50000,
                    divergence: float = 0.25) -> dict:
    """Candidates of one synthetic genome seed (3 + n_other per protein)."""
    rng = np.random.default_rng(seed * 1000003 + 17)
    nt_parts, aa_parts = [], []
    off_p = np.zeros(n_prot, np.int64)
    off_m = np.zeros(n_prot, np.int64)
    wlen = np.zeros(n_prot, np.int32)
    gpos = np.zeros((n_prot, 2), np.int64)
    aoff = np.zeros(n_prot, np.int64)
    alen = np.zeros(n_prot, np.int32)
    pn = pa = 0
    for i in range(n_prot):
        al = int(np.clip(round(math.exp(rng.normal(math.log(350.0), 0.6))), 50, 2500))
        prot = W.random_protein(rng, al)
        k = int(rng.poisson(4.0))
        introns = [int(min(20000, max(20, round(math.exp(rng.normal(math.log(150.0), 0.8)))))) for _ in range(k)]
        gene = W.build_gene(rng, prot, divergence=divergence, n_frameshift=int(rng.integers(0, 3)),
                            intron_lengths=introns)
        w = max(int(rng.integers(win_min, win_max + 1)), len(gene) + 200)
        left = int(rng.integers(100, w - len(gene) - 99))
        win = (W.random_dna(rng, left) + gene + W.random_dna(rng, w - len(gene) - left)).encode()
        nt_parts += [win, W.revcomp(win)]
        off_p[i], off_m[i] = pn, pn + w
        pn += 2 * w
        wlen[i] = w
        gpos[i] = (left, left + len(gene))
        aa_parts.append(prot.encode())
        aoff[i], alen[i] = pa, al
        pa += al
    per = 3 + n_other
    n = n_prot * per
    jobs = np.zeros(n, JOB_DTYPE)
    prot_id = np.repeat(np.arange(n_prot, dtype=np.int32), per)
    kind = np.tile(np.array([KIND_OWN_PLUS, KIND_OWN_MINUS, KIND_PARTIAL] + [KIND_OTHER] * n_other, np.int8), n_prot)
    jobs["ss_off"] = -1
    jobs["aa_off"] = aoff[prot_id]
    jobs["al"] = alen[prot_id]
    base = np.arange(n_prot) * per
    jobs["nt_off"][base], jobs["nl"][base] = off_p, wlen
    jobs["nt_off"][base + 1], jobs["nl"][base + 1] = off_m, wlen
    # partial: the window cut inside the gene, keeping the part before or after the cut
    frac = rng.uniform(0.3, 0.7, n_prot)
    cut = (gpos[:, 0] + frac * (gpos[:, 1] - gpos[:, 0])).astype(np.int64)
    keep_left = rng.random(n_prot) < 0.5
    jobs["nt_off"][base + 2] = np.where(keep_left, off_p, off_p + cut)
    jobs["nl"][base + 2] = np.where(keep_left, cut, wlen - cut)
    for t in range(n_other):
        j = (np.arange(n_prot) + rng.integers(1, n_prot, n_prot)) % n_prot
        minus = rng.random(n_prot) < 0.5
        jobs["nt_off"][base + 3 + t] = np.where(minus, off_m[j], off_p[j])
        jobs["nl"][base + 3 + t] = wlen[j]
    return {"nt": np.frombuffer(b"".join(nt_parts), np.uint8), "aa": np.frombuffer(b"".join(aa_parts), np.uint8),
            "jobs": jobs, "prot": prot_id, "kind": kind, "seed": seed}


def job_ptr(jobs: np.ndarray):
    return C.cast(jobs.ctypes.data, C.POINTER(SpliceJob))


def cigar_bounds(cig: np.ndarray, res, min_run: int = 10) -> tuple[np.ndarray, np.ndarray]:
    """First nucleotide of the first and end of the last run of >= min_run codon
    matches (M) in each job's CIGAR (words as ns_push_cigar writes them; -1 without
    one).  A global alignment over a wide window typically opens with a few residues
    at the window start and a long intron, and closes the same way; the runs skip
    those."""
    n = len(res)
    offs = np.asarray(res["cigar_off"], np.int64)
    cnt = np.asarray(res["n_cigar"], np.int64)
    start = np.full(n, -1, np.int64)
    end = np.full(n, -1, np.int64)
    if n == 0 or cnt.sum() == 0:
        return start, end
    idx = np.repeat(offs, cnt) + (np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    w = cig[idx].astype(np.int64)
    op, ln = w & 15, w >> 4
    ntc = np.where((op == 0) | (op == 2), 3 * ln, np.where(op == 1, 0, ln))
    cum = np.cumsum(ntc)
    seg = np.repeat(np.arange(n), cnt)
    first = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    base = cum[first] - ntc[first]
    pos = np.arange(len(w))
    isM = (op == 0) & (ln >= min_run)
    big = len(w) + 1
    fm = np.full(n, big)
    lm = np.full(n, -1)
    np.minimum.at(fm, seg[isM], pos[isM])
    np.maximum.at(lm, seg[isM], pos[isM])
    has = lm >= 0
    start[has] = cum[fm[has]] - ntc[fm[has]] - base[has]
    end[has] = cum[lm[has]] - base[has]
    return start, end


def query_span(cig: np.ndarray, res: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Aligned query span of each job: the residue where its first codon match (M op)
    starts and the residue where its last one ends (0, 0 without one).  res is a
    RES_DTYPE array whose CIGARs lie back to back in cig (as the compaction writes them)."""
    n = len(res)
    qs, qe = np.zeros(n, np.int64), np.zeros(n, np.int64)
    cnt = res["n_cigar"].astype(np.int64)
    if n == 0 or cnt.sum() == 0:
        return qs, qe
    start = res["cigar_off"].astype(np.int64)
    total = int(cnt.sum())
    seg = np.repeat(np.arange(n), cnt)
    idx = start[seg] + (np.arange(total) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    w = cig[idx].astype(np.int64)
    op, ln = w & 15, w >> 4
    # residues consumed (align.c:173-215): M and I one per unit, G and the split codon of U/V one per op
    aac = np.where((op == 0) | (op == 1), ln, np.where((op == 11) | (op == 12) | (op == 13), 1, 0))
    cum = np.cumsum(aac)
    base = np.zeros(n, np.int64)
    has_any = cnt > 0
    first = np.cumsum(cnt) - cnt
    base[has_any] = cum[first[has_any]] - aac[first[has_any]]
    isM = op == 0
    big = total + 1
    fm, lm = np.full(n, big), np.full(n, -1)
    pos = np.arange(total)
    np.minimum.at(fm, seg[isM], pos[isM])
    np.maximum.at(lm, seg[isM], pos[isM])
    has = lm >= 0
    qs[has] = cum[fm[has]] - aac[fm[has]] - base[has]
    qe[has] = cum[lm[has]] - base[has]
    return qs, qe


def output_set(score: np.ndarray, qs: np.ndarray, qe: np.ndarray, prot: np.ndarray, qlen: np.ndarray,
               aligned: np.ndarray | None = None, out_n: int = OUT_N, out_sim: float = OUT_SIM,
               out_cov: float = OUT_COV) -> np.ndarray:
    """Candidates that mp_reg_will_output's final test (map.c:456-462) lets through, per
    protein: among the protein's aligned candidates ranked by decreasing score (ties by
    candidate order), the first out_n with score > 0, score >= out_sim x the best score
    and qe - qs >= out_cov x qlen.  aligned: candidates that have a result (all when None)."""
    n = len(score)
    ok = np.ones(n, bool) if aligned is None else aligned.astype(bool)
    sc = score.astype(np.int64)
    order = np.lexsort((np.arange(n), -sc, prot))          # by protein, then score descending
    order = order[ok[order]]
    p_sorted = prot[order]
    first = np.ones(len(order), bool)
    first[1:] = p_sorted[1:] != p_sorted[:-1]
    grp_start = np.maximum.accumulate(np.where(first, np.arange(len(order)), 0))
    rank = np.arange(len(order)) - grp_start
    best = sc[order][grp_start]
    c = order
    passes = (sc[c] > 0) & (sc[c] >= best.astype(np.float64) * out_sim) & \
             ((qe[c] - qs[c]) >= qlen[c].astype(np.float64) * out_cov) & (rank < out_n)
    out = np.zeros(n, bool)
    out[c[passes]] = True
    return out


def loci_reported(out: np.ndarray, prot: np.ndarray, kind: np.ndarray, n_prot: int) -> np.ndarray:
    """Per protein: its planted gene is reported (a candidate on the gene -- own window on
    either strand or the partial window -- is in the output set)."""
    on_gene = out & (kind != KIND_OTHER)
    rep = np.zeros(n_prot, bool)
    rep[prot[on_gene]] = True
    return rep


class PrefilterModel:
    """The MLP on the device (pl_pf_model_*)."""

    def __init__(self, device: int = 0, hidden: int = 256, seed: int = 1, params: np.ndarray | None = None):
        self.lib = L.load()
        self.device, self.hidden = device, hidden
        self.h = self.lib.pl_pf_model_create(device, FDIM, hidden, seed)
        if not self.h:
            raise RuntimeError("pl_pf_model_create: " + L.error())
        if params is not None:
            self.set_params(params)

    def size(self) -> int:
        return int(self.lib.pl_pf_model_size(self.h))

    def params(self) -> np.ndarray:
        p = np.zeros(self.size(), np.float32)
        if not self.lib.pl_pf_model_get(self.h, p.ctypes.data, p.size):
            raise RuntimeError(L.error())
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        if not self.lib.pl_pf_model_set(self.h, p.ctypes.data, p.size):
            raise RuntimeError(L.error())

    def train(self, feats, targets, perm, batch: int, steps: int, lr: float, pos_w: float, box_w: float) -> np.ndarray:
        log = np.zeros(max(steps, 1), np.float32)
        if not self.lib.pl_pf_train(self.h, feats.data_ptr(), targets.data_ptr(), perm.data_ptr(), perm.numel(), batch,
                                    steps, lr, pos_w, box_w, log.ctypes.data, None):
            raise RuntimeError("pl_pf_train: " + L.error())
        return log[:steps]

    def predict(self, feats, n: int, out=None):
        import torch
        npad = (n + 127) // 128 * 128
        if out is None:
            out = torch.zeros(npad, 16, dtype=torch.float32, device=f"cuda:{self.device}")
        stream = torch.cuda.current_stream().cuda_stream
        if not self.lib.pl_pf_predict(self.h, feats.data_ptr(), n, out.data_ptr(), stream):
            raise RuntimeError("pl_pf_predict: " + L.error())
        return out

    def close(self):
        if self.h:
            self.lib.pl_pf_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pipeline:
    """Device-resident candidate set with the plain and learned paths over it."""

    def __init__(self, eng: L.Engine, cand: dict):
        import torch
        self.eng, self.cand = eng, cand
        self.opt = Options(flag=NS_F_CIGAR)
        dev = f"cuda:{eng.device}" if hasattr(eng, "device") else "cuda"
        self.dev = dev
        self.d_nt = torch.from_numpy(cand["nt"].copy()).to(dev)
        self.d_aa = torch.from_numpy(cand["aa"].copy()).to(dev)
        self.n = len(cand["jobs"])
        self.tune_plain = self.tune_learned = None  # engine tuning per path (None: the engine's own)

    def autotune(self, jobs: np.ndarray) -> dict:
        """pl_engine_autotune over `jobs` (sequences resident on the device); returns the tuning."""
        r4, ratio = C.c_int32(), C.c_double()
        if not self.eng.lib.pl_engine_autotune(self.eng.h, self.opt.ptr, job_ptr(jobs), len(jobs), self.d_nt.data_ptr(),
                                               self.d_aa.data_ptr(), None, C.byref(r4), C.byref(ratio)):
            raise RuntimeError("pl_engine_autotune: " + L.error())
        return {"r4_rows": r4.value, "coop_ratio": ratio.value}

    def autotune_paths(self, model: "PrefilterModel", tau: float, margin: int, tau_fb: float):
        """Separate engine tunings for the plain path (full windows) and the learned path
        (tightened windows), each chosen by the autotuner on its own jobs."""
        self.tune_plain = self.autotune(self.cand["jobs"])
        feats, chain = self.features()
        out = model.predict(feats, self.n)
        o = out[: self.n, :3].cpu().numpy()
        keep = np.nonzero(o[:, 0] >= _logit(tau))[0]
        self.tune_learned = self.autotune(self.tightened(keep, o, chain[: self.n].cpu().numpy(), margin))
        return self.tune_plain, self.tune_learned

    def _use(self, tuning):
        if tuning is not None:
            self.eng.set_tuning(tuning["r4_rows"], tuning["coop_ratio"])

    def features(self):
        import torch
        npad = (self.n + 127) // 128 * 128
        feats = torch.empty(npad, FDIM, dtype=torch.bfloat16, device=self.dev)
        chain = torch.empty(max(self.n, 1), 4, dtype=torch.int32, device=self.dev)
        stream = torch.cuda.current_stream().cuda_stream
        if not self.eng.lib.pl_pf_features_device(self.eng.h, self.opt.ptr, job_ptr(self.cand["jobs"]), self.n,
                                                  self.d_nt.data_ptr(), self.d_aa.data_ptr(), feats.data_ptr(),
                                                  chain.data_ptr(), stream):
            raise RuntimeError("pl_pf_features_device: " + L.error())
        return feats, chain

    def plain(self):
        """The plain path: the exact DP over every candidate's full window, then the output
        test per protein.  Returns (output mask, scores)."""
        self._use(self.tune_plain)
        score, qs, qe = self.dp(self.cand["jobs"], spans=True)
        return self.decide(score, qs, qe), score

    def decide(self, score, qs, qe, aligned=None):
        """The output set of a path's results (mp_reg_will_output's test, per protein)."""
        c = self.cand
        return output_set(score, qs, qe, c["prot"], c["jobs"]["al"], aligned)

    def loci(self, out):
        """Per protein: its planted gene is reported."""
        c = self.cand
        return loci_reported(out, c["prot"], c["kind"], int(c["prot"].max()) + 1 if len(c["prot"]) else 0)

    def dp(self, jobs: np.ndarray, bounds: bool = False, spans: bool = False):
        """Exact spliced DP with CIGAR over `jobs` (device-resident sequences): scores, and
        from the CIGARs either the aligned window span (first/last run of codon matches,
        bounds) or the aligned query span (first/last codon match, spans)."""
        n = len(jobs)
        if n == 0:
            z = np.zeros(0, np.int64)
            return np.zeros(0, np.int32), z, z
        res, cig = self.dp_raw(jobs, bounds or spans)
        score = res["score"].copy()
        if not bounds and not spans:
            return score, None, None
        s, e = query_span(cig, res) if spans else cigar_bounds(cig, res)
        return score, s, e

    def dp_raw(self, jobs: np.ndarray, cigars: bool = True):
        """The DP results of `jobs` (RES_DTYPE) and the CIGAR words (None unless cigars)."""
        import torch
        n = len(jobs)
        cap = int(jobs["al"].astype(np.int64).sum() * 4 + 256 * n)
        d_res = torch.zeros(n * C.sizeof(SpliceResult), dtype=torch.uint8, device=self.dev)
        d_cig = torch.zeros(cap, dtype=torch.int32, device=self.dev)
        total = C.c_int64()
        stream = torch.cuda.current_stream().cuda_stream
        if not self.eng.lib.pl_splice_batch_device(self.eng.h, self.opt.ptr, job_ptr(jobs), n, self.d_nt.data_ptr(),
                                                   self.d_aa.data_ptr(), None, d_res.data_ptr(), d_cig.data_ptr(),
                                                   cap, C.byref(total), stream):
            raise RuntimeError("pl_splice_batch_device: " + L.error())
        res = np.frombuffer(d_res.cpu().numpy().tobytes(), RES_DTYPE)
        if (res["status"] != 0).any():
            raise RuntimeError(f"{int((res['status'] != 0).sum())} DP jobs failed")
        return res, (d_cig[: int(total.value)].cpu().numpy() if cigars else None)

    def targets(self, passed, s, e):
        """[label, start fraction, end fraction, box weight] rows for training: label = the
        candidate is in the plain path's output set."""
        nl = self.cand["jobs"]["nl"].astype(np.float64)
        y = passed.astype(np.float32)
        T = np.zeros((self.n, 4), np.float32)
        T[:, 0] = y
        T[:, 1] = np.where(y > 0, s / nl, 0.0)
        T[:, 2] = np.where(y > 0, e / nl, 0.0)
        T[:, 3] = y
        return T

    def tightened(self, keep: np.ndarray, out: np.ndarray, chain: np.ndarray | None, margin: int,
                  rel: float = 0.0) -> np.ndarray:
        """Jobs of the kept candidates with windows cut to the union of the predicted
        alignment span and the span the best anchor chain implies (its first anchor
        minus 3x the residues before it, its last plus 3x the residues after it), plus
        margin + rel * span on both sides (at least 3 nt, within the window)."""
        jobs = np.ascontiguousarray(self.cand["jobs"][keep])
        n = len(jobs)
        o = np.ascontiguousarray(out[keep, :3], np.float32)
        ch = np.ascontiguousarray(chain[keep], np.int32) if chain is not None else None
        k = np.zeros(max(n, 1), np.uint8)
        tight = np.zeros(n, JOB_DTYPE)
        if n and not L.load().pl_pf_decide(n, jobs.ctypes.data, o.ctypes.data, 3,
                                           ch.ctypes.data if ch is not None else None, 0.0, int(margin), float(rel),
                                           1.0, k.ctypes.data, None, tight.ctypes.data):
            raise RuntimeError("pl_pf_decide: " + L.error())
        return tight

    def learned(self, model: PrefilterModel, tau: float, margin: int, rel: float = 0.0, tau_fb: float = 0.0):
        """The learned path: (output mask over all candidates, stats).  Candidates with
        p >= tau run the exact DP on their tightened windows; those whose score there is
        not positive and have p >= tau_fb run it again on the full window; the output test
        then runs per protein over the candidates that were aligned."""
        import torch
        t0 = time.perf_counter()
        if rel == 0.0:  # features, MLP and the decision in one C call (pl_pf_select_device)
            n = self.n
            k = np.zeros(n, np.uint8)
            fbk = np.zeros(n, np.uint8)
            tight = np.zeros(n, JOB_DTYPE)
            stream = torch.cuda.current_stream().cuda_stream
            if not self.eng.lib.pl_pf_select_device(model.h, self.eng.h, self.opt.ptr, self.cand["jobs"].ctypes.data,
                                                    n, self.d_nt.data_ptr(), self.d_aa.data_ptr(), float(tau),
                                                    int(margin), float(tau_fb), k.ctypes.data, fbk.ctypes.data,
                                                    tight.ctypes.data, None, stream):
                raise RuntimeError("pl_pf_select_device: " + L.error())
            keep = np.nonzero(k)[0]
            jobs = tight[keep]
            fb_mask = fbk.astype(bool)
        else:
            feats, chain = self.features()
            out = model.predict(feats, self.n)
            o = out[: self.n, :3].cpu().numpy()
            ch = chain[: self.n].cpu().numpy()
            z = o[:, 0]
            keep = np.nonzero(z >= _logit(tau))[0]
            jobs = self.tightened(keep, o, ch, margin, rel)
            fb_mask = z >= _logit(tau_fb)
        t1 = time.perf_counter()
        self._use(self.tune_learned)
        sc, qs, qe = self.dp(jobs, spans=True)
        t2 = time.perf_counter()
        bad = sc <= 0
        fail = keep[bad]
        fail = fail[fb_mask[fail]]
        self._use(self.tune_plain)
        sc2, qs2, qe2 = self.dp(self.cand["jobs"][fail], spans=True)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        score = np.zeros(self.n, np.int32)
        qsa, qea = np.zeros(self.n, np.int64), np.zeros(self.n, np.int64)
        aligned = np.zeros(self.n, bool)
        score[keep], qsa[keep], qea[keep], aligned[keep] = sc, qs, qe, True
        score[fail], qsa[fail], qea[fail] = sc2, qs2, qe2
        passed = self.decide(score, qsa, qea, aligned)
        t4 = time.perf_counter()
        cells_tight = int(((jobs["nl"].astype(np.int64) - 2) * jobs["al"]).sum())
        stats = {"kept": int(len(keep)), "fallback": int(len(fail)), "cells_tight": cells_tight,
                 "s_score": t1 - t0, "s_dp": t2 - t1, "s_fallback": t3 - t2, "s_output": t4 - t3, "s_total": t4 - t0}
        return passed, stats


def _logit(p: float) -> float:
    if p <= 0.0:
        return -math.inf
    if p >= 1.0:
        return math.inf
    return math.log(p / (1.0 - p))


def _gen(args):
    seed, n_prot = args
    return make_candidates(seed, n_prot)


def candidate_stream(seeds, n_prot: int, workers: int = 8):
    """make_candidates over seeds, generated ahead in spawned worker processes."""
    import concurrent.futures as cf
    import multiprocessing as mp
    if workers <= 1:
        for sd in seeds:
            yield make_candidates(sd, n_prot)
        return
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        yield from ex.map(_gen, [(sd, n_prot) for sd in seeds])


def build_set(eng: L.Engine, seeds, n_prot: int, workers: int = 8, log=None):
    """Training/validation rows of the given seeds: bf16 features [N x FDIM] and f32
    targets [N x 4] on the device (N = candidates of all seeds), plus host-side
    labels, kinds and plain-path DP time."""
    import torch
    feats, targets, labels, kinds, dp_s = [], [], [], [], 0.0
    for cand in candidate_stream(seeds, n_prot, workers):
        pipe = Pipeline(eng, cand)
        f, _ = pipe.features()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, cig = pipe.dp_raw(cand["jobs"])
        dp_s += time.perf_counter() - t0
        sc = res["score"].copy()
        s, e = cigar_bounds(cig, res)
        qs, qe = query_span(cig, res)
        T = pipe.targets(pipe.decide(sc, qs, qe), s, e)
        feats.append(f[: pipe.n])
        targets.append(torch.from_numpy(T).to(pipe.dev))
        labels.append(T[:, 0] > 0.5)
        kinds.append(cand["kind"])
        if log:
            log(f"seed {cand['seed']}: {pipe.n} candidates, {int(T[:, 0].sum())} pass, DP {time.perf_counter() - t0:.2f} s")
        del pipe
    n = sum(int(x.shape[0]) for x in feats)
    npad = (n + 127) // 128 * 128
    F = torch.zeros(npad, FDIM, dtype=torch.bfloat16, device=feats[0].device)
    r = 0
    for x in feats:
        F[r: r + x.shape[0]] = x
        r += x.shape[0]
    return {"feats": F, "targets": torch.cat(targets), "n": n, "labels": np.concatenate(labels),
            "kinds": np.concatenate(kinds), "dp_s": dp_s}


def train(model: PrefilterModel, data: dict, epochs: int = 8, batch: int = 4096, lr: float = 1e-3,
          pos_w: float = 4.0, box_w: float = 2.0, seed: int = 7) -> np.ndarray:
    """Adam over `epochs` shuffled passes of the rows (one captured CUDA graph per step)."""
    import torch
    n = data["n"]
    rng = np.random.default_rng(seed)
    steps_per = n // batch
    perm = np.concatenate([rng.permutation(n)[: steps_per * batch] for _ in range(epochs)]).astype(np.int32)
    d_perm = torch.from_numpy(perm).to(data["feats"].device)
    return model.train(data["feats"], data["targets"], d_perm, batch, steps_per * epochs, lr, pos_w, box_w)


def calibrate(model: PrefilterModel, pipe: Pipeline, labels: np.ndarray, recall: float = 0.998,
              cls_recall: float = 0.999, margins=(0, 100, 200, 400, 800), max_tight_fail: float = 0.003):
    """Decision parameters from a validation set: tau keeps cls_recall of the passing
    candidates; margin is the smallest whose tightened windows fail for at most
    max_tight_fail of the kept passers; tau_fb is the highest fallback threshold that
    still leaves the path's recall of the passers at `recall`."""
    import torch
    feats, chain = pipe.features()
    out = model.predict(feats, pipe.n)
    torch.cuda.synchronize()
    o = out[: pipe.n, :3].cpu().numpy()
    ch = chain[: pipe.n].cpu().numpy()
    z = o[:, 0]
    zp = np.sort(z[labels])
    k = int(math.floor((1.0 - cls_recall) * len(zp)))
    zt = float(zp[k]) if len(zp) else 0.0
    keep = np.nonzero(z >= zt)[0]
    chosen, sc = margins[-1], None
    for m in margins:
        sc, _, _ = pipe.dp(pipe.tightened(keep, o, ch, m))
        kp = labels[keep]
        if kp.sum() == 0 or ((sc <= 0) & kp).sum() <= max_tight_fail * kp.sum():
            chosen = m
            break
    fail = keep[sc <= 0]
    missed_cls = int(labels.sum()) - int(labels[keep].sum())
    allowed = int(math.floor((1.0 - recall) * labels.sum())) - missed_cls
    zf = np.sort(z[fail[labels[fail]]])  # passers the tightened windows lose
    if allowed < 0 or len(zf) == 0:
        z_fb = zt if len(zf) else math.inf
    elif allowed >= len(zf):
        z_fb = math.inf
    else:
        z_fb = float(zf[allowed])
    tau = 1.0 / (1.0 + math.exp(-zt))
    tau_fb = 1.0 if z_fb == math.inf else 1.0 / (1.0 + math.exp(-z_fb))
    info = {"kept": int(len(keep)), "kept_pass": int(labels[keep].sum()), "n": pipe.n, "tight_fail": int(len(fail)),
            "tight_fail_pass": int(len(zf)), "fallback": int((z[fail] >= z_fb).sum())}
    return tau, chosen, tau_fb, info


def save(path: str, model: PrefilterModel, **meta):
    np.savez(path, params=model.params(), hidden=model.hidden, **meta)


def load_model(path: str, device: int = 0):
    z = np.load(path, allow_pickle=False)
    model = PrefilterModel(device, hidden=int(z["hidden"]), params=z["params"])
    meta = {k: z[k] for k in z.files if k not in ("params", "hidden")}
    return model, meta


def evaluate(eng: L.Engine, model: PrefilterModel, cand: dict, tau: float, margin: int, tau_fb: float,
             repeats: int = 3) -> dict:
    """Plain path vs learned path on one candidate set, inputs resident on the device:
    candidates per second of each (best of `repeats` after a warm-up) and the learned
    path's recall of the plain path's passing candidates."""
    import torch
    pipe = Pipeline(eng, cand)
    pipe.autotune_paths(model, tau, margin, tau_fb)
    plain, _ = pipe.plain()  # warm-up
    t_plain = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain, _ = pipe.plain()
        torch.cuda.synchronize()
        t_plain.append(time.perf_counter() - t0)
    pipe.learned(model, tau, margin, 0.0, tau_fb)  # warm-up
    runs = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        passed, st = pipe.learned(model, tau, margin, 0.0, tau_fb)
        torch.cuda.synchronize()
        st["wall"] = time.perf_counter() - t0
        runs.append((passed, st))
    passed, st = min(runs, key=lambda r: r[1]["wall"])
    m = path_metrics(pipe, plain, passed)
    jobs = cand["jobs"]
    cells_plain = int(((jobs["nl"].astype(np.int64) - 2) * jobs["al"]).sum())
    n_loci = m["loci"]
    return {"n": pipe.n, **m, "plain_s": min(t_plain), "learned_s": st["wall"],
            "plain_loci_per_s": n_loci / min(t_plain), "learned_loci_per_s": n_loci / st["wall"],
            "speedup": min(t_plain) / st["wall"], "cells_plain": cells_plain, "tune_plain": pipe.tune_plain,
            "tune_learned": pipe.tune_learned, **st}


def path_metrics(pipe: Pipeline, plain_out: np.ndarray, learned_out: np.ndarray) -> dict:
    """Locus-level and candidate-level agreement of the learned path with the plain path."""
    lp, ll = pipe.loci(plain_out), pipe.loci(learned_out)
    return {"loci": int(len(lp)), "plain_loci": int(lp.sum()), "learned_loci": int(ll.sum()),
            "locus_recall": float((lp & ll).sum() / lp.sum()) if lp.any() else 1.0,
            "extra_loci": int((ll & ~lp).sum()), "plain_out": int(plain_out.sum()),
            "out_recall": float(learned_out[plain_out].mean()) if plain_out.any() else 1.0,
            "extra_out": int((learned_out & ~plain_out).sum())}


def main(argv=None):
    import argparse
    import json
    import sys
    ap = argparse.ArgumentParser(description="train / evaluate the learned candidate prefilter")
    ap.add_argument("cmd", choices=["train", "calibrate", "eval"])
    ap.add_argument("--train-seeds", default="1-64")
    ap.add_argument("--val-seed", type=int, default=66, help="calibration seed (held out from training and evaluation)")
    ap.add_argument("--eval-seed", type=int, default=65)
    ap.add_argument("--n-prot", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--recall", type=float, default=0.998, help="validation recall of the whole learned path")
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--model", default=None, help="weights (.npz): written by train/calibrate, read by eval")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    log = (lambda s: print(s, file=sys.stderr, flush=True))
    eng = L.Engine(a.device)
    out = a.model or "prefilter.npz"
    if a.cmd == "train":
        lo, hi = (int(x) for x in a.train_seeds.split("-"))
        t0 = time.perf_counter()
        data = build_set(eng, range(lo, hi + 1), a.n_prot, a.workers, log)
        t1 = time.perf_counter()
        model = PrefilterModel(a.device, seed=1)
        losses = train(model, data, a.epochs, a.batch, a.lr)
        t2 = time.perf_counter()
        log(f"{data['n']} rows ({int(data['labels'].sum())} pass) built in {t1 - t0:.1f} s; "
            f"{len(losses)} steps in {t2 - t1:.2f} s; loss {losses[:50].mean():.4f} -> {losses[-50:].mean():.4f}")
        meta = {"train_seeds": a.train_seeds, "n_prot": a.n_prot, "epochs": a.epochs, "train_rows": data["n"],
                "train_pass": int(data["labels"].sum()), "train_steps": len(losses), "train_s": t2 - t1,
                "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean())}
        del data
    else:
        model, meta = load_model(out if a.cmd == "calibrate" else a.model, a.device)
        meta = {k: v.item() if hasattr(v, "item") else v for k, v in meta.items()}
    if a.cmd in ("train", "calibrate"):
        cand = make_candidates(a.val_seed, a.n_prot)
        pipe = Pipeline(eng, cand)
        plain, _ = pipe.plain()
        tau, margin, tau_fb, info = calibrate(model, pipe, plain, a.recall)
        log(f"calibrated on seed {a.val_seed}: tau {tau:.4g}, margin {margin}, tau_fb {tau_fb:.4g}, {info}")
        meta.update(tau=tau, margin=margin, tau_fb=tau_fb, val_seed=a.val_seed, val_recall=a.recall)
        save(out, model, **meta)
        print(json.dumps({"model": out, **{k: (v if not isinstance(v, np.generic) else v.item()) for k, v in meta.items()}}))
    else:
        cand = make_candidates(a.eval_seed, a.n_prot)
        r = evaluate(eng, model, cand, float(meta["tau"]), int(meta["margin"]), float(meta["tau_fb"]))
        print(json.dumps(r))
    eng.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
