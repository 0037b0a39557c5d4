#!/usr/bin/env python
"""Benchmark of the batched global spliced DP (the alignment hot path).

One step = one pass of the hot path over the batched workload: 4096 synthetic
protein/window pairs searched on both strands (8192 global spliced DPs with
CIGAR): input preparation, the wavefront DP, device traceback and CIGAR
compaction.  Metric: GCUPS, cells = (nl-2)*al per DP (nasw-cuda.cu:793),
bit-exact with the reference CPU path.

  value   device-resident inputs (uploaded once), pl_splice_batch_device per step,
          CUDA events on the launching stream, max over ranks
  e2e     pl_splice_batch_host per step from pinned host buffers: H2D of the
          step's inputs, all kernels, D2H of the results and CIGARs
  roofline  the DP kernel (k_splice_dp): algorithmic int16 lane-ops per cell
          (65 with traceback, counted from the reference SSE kernel) x cells,
          divided by the DP kernel's own CUDA-event time (the union of the DP
          launches' intervals: a batch over the trace budget runs its waves on two
          streams, so launches of consecutive waves overlap), against the integer
          pipe's lane-op peak measured live on this device (pl_measure_int_peak)
  cpu_baseline  the reference's ns_global_gs_auto compiled from its own sources
          (oracle/_ref), driven by the reference's kt_for over all host cores, on
          a bounded random sample of the same jobs

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank runs its own batch (seed 1+rank): weak scaling, no
collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from protlocus_b200 import lib as L  # noqa: E402
from protlocus_b200 import workload as W  # noqa: E402
from protlocus_b200.abi import NS_F_CIGAR, ExtJob, ExtResult, Options, SpliceJob, SpliceResult  # noqa: E402
from protlocus_b200.ranks import Ranks, job_rate  # noqa: E402

METRIC = "spliced-DP GCUPS (bit-exact) at 1 B200"
DP_DRAM_BYTES_PER_CELL = 2.08  # ncu: k_splice_dp dram__bytes_read+write per cell (trace words are 2.0 B/cell)
PAIR_DRAM_BYTES_PER_CELL = 2.20  # ncu: k_splice_pair<8>, uniform 4736x2000x250 (0.41 GB read + 6.54 GB written)
OPS_PER_CELL = 65  # int16 lane-ops per cell with traceback bits, counted from nasw-sse.c:465-553
WORKLOAD = ("batched global spliced DP: 4096 protein/window pairs x 2 strands = 8192 DPs with CIGAR; "
            "protein log-normal median 350 aa (50-2500), window uniform 1-50 kb, Poisson(4) introns, "
            "25% divergence, ProtLocus default scoring")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=4096)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU work of the baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-hmm", action="store_true",
                    help="headline: skip the profile-HMM genome-scan sub-object (1000 profiles, six frames)")
    ap.add_argument("--trace-budget-gb", type=float, default=110.0,
                    help="traceback arena of the headline's engine (0: the engine's default, 40%% of free memory up to "
                         "72 GB); the batch's 175 GB of trace runs in waves of half the arena on two streams: 110 GB "
                         "gives four waves on a 180 GB B200")
    ap.add_argument("--no-prefilter", action="store_true",
                    help="leave the learned-prefilter loci/s sub-object out of the headline line")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="leave the reference's own CUDA global DP (timed in a child process) out of the headline")
    ap.add_argument("--ref-jobs", type=int, default=256, help="jobs of the reference GPU queue sample (--workload refgpu)")
    ap.add_argument("--tuning-json", default=None,
                    help="per-shape-class tuning file (default: $PLGPU_TUNING_JSON or ~/.cache/protlocus_b200/tuning.json)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the engine's default tuning instead of autotuning it on the workload (global DP)")
    ap.add_argument("--workload", default="global",
                    choices=["global", "ext", "hmm", "gapless", "forward", "prefilter", "extra", "prescreen", "chain",
                             "seed", "seed_hmm", "refgpu"],
                    help="global: the batched global spliced DP (headline); ext: the batched extension DP; "
                         "hmm: the integer profile-HMM DP; gapless: the gapless X-drop prefilter; "
                         "forward: the recheck Forward score; prefilter: learned candidate prefilter vs the plain "
                         "batched DP over the held-out seed's candidates; extra: alignment statistics and exon "
                         "features from the CIGAR; prescreen: banded gapped profile-ORF alignment; chain: anchor "
                         "chaining (mp_chain) of the coarse mapping; seed: the coarse mapping's seeding of protein "
                         "queries; seed_hmm: the same for HMM-profile queries (profile-derived seeds)")
    ap.add_argument("--peptides", type=int, default=20000, help="peptides per step (--workload forward)")
    ap.add_argument("--candidates", type=int, default=131072, help="candidates of 8 anchors (--workload gapless)")
    ap.add_argument("--profiles", type=int, default=16, help="profiles per step (--workload hmm)")
    ap.add_argument("--regions", type=int, default=4096, help="regions per profile (--workload hmm)")
    ap.add_argument("--hmm-shape", default="regions", choices=["regions", "genome"],
                    help="--workload hmm: 'regions' = synthetic regions per profile; 'genome' = the profile-HMM "
                         "configuration (use --profiles 1000): every profile against a six-frame genome slice")
    ap.add_argument("--genome-slice-mb", type=float, default=2.0, help="Mb of the 100 Mb genome scanned per step")
    ap.add_argument("--genome-region-kb", type=int, default=12, help="region window of the genome scan (kb)")
    ap.add_argument("--requests", type=int, default=65536, help="extension requests per step (--workload ext)")
    ap.add_argument("--uniform", default=None, metavar="N:NL:AL",
                    help="profiling case instead of the batched workload: N jobs, N/2 planted loci of window NL "
                         "and protein AL on both strands")
    return ap.parse_args()


def make_jobs(args, seed):
    if args.uniform:  # n jobs: n/2 planted loci of window nl and protein al, each on both strands
        n, nl, al = (int(x) for x in args.uniform.split(":"))
        out = []
        for q in range((n + 1) // 2):
            nt, aa = W.single_locus(seed=seed * 100003 + q, al=al, window=nl)
            out += [(nt, aa), (W.revcomp(nt), aa)]
        return out[:n]
    return W.batch_pairs(args.pairs, seed=seed)


def pack(jobs):
    """Packed inputs and job table; a protein searched on both strands is stored once and both
    jobs point at it (the jobs of one protein and window length then run as int16x2 pairs)."""
    n = len(jobs)
    nl = np.array([len(a) for a, _ in jobs], dtype=np.int32)
    al = np.array([len(b) for _, b in jobs], dtype=np.int32)
    nt_off = np.zeros(n, dtype=np.int64)
    aa_off = np.zeros(n, dtype=np.int64)
    nt_off[1:] = np.cumsum(nl[:-1])
    prot_off, parts, pos = {}, [], 0
    for q, (_, b) in enumerate(jobs):
        if b not in prot_off:
            prot_off[b] = pos
            parts.append(b)
            pos += len(b)
        aa_off[q] = prot_off[b]
    nt = np.frombuffer(b"".join(a for a, _ in jobs), dtype=np.uint8)
    aa = np.frombuffer(b"".join(parts), dtype=np.uint8)
    tab = (SpliceJob * n)()
    for q in range(n):
        tab[q].nt_off, tab[q].aa_off, tab[q].ss_off, tab[q].nl, tab[q].al = nt_off[q], aa_off[q], -1, nl[q], al[q]
    return nt, aa, nt_off, aa_off, nl, al, tab


def hbm_peak():
    """The HBM copy bandwidth (GB/s) a memory-bound line is measured against, and its source: the
    pool's measured figure in MEASURED_PEAKS.json when that file is present, else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback HBM copy bandwidth of this pool (6.65 TB/s)"


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.send_signal(signal.SIGTERM)
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(", ") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(jobs, nt, aa, nt_off, aa_off, nl, al, opt, target_s, steps=1):
    """The reference CPU path over a bounded random sample, all host threads.
    Returns (GCUPS, threads, kind, sample description, seconds per step)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    threads = os.cpu_count() or 1
    ref = O.ref_lib()
    if ref is not None:
        fn, kind = ref.ref_bench_global, "reference"
    else:
        fn, kind = O.port_lib().port_bench_global, "port"
    fn.restype = C.c_double
    fn.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    n = len(nl)
    rng = np.random.default_rng(12345)
    perm = rng.permutation(n)
    cells = (nl.astype(np.int64) - 2) * al
    # calibrate on a small sample: ~0.5 GCUPS per thread for the SSE kernel
    budget = target_s * 0.5e9 * threads
    take, acc = [], 0
    for q in perm:
        if acc + cells[q] > budget and take:
            continue
        take.append(q)
        acc += int(cells[q])
        if acc >= budget:
            break
    take = np.array(sorted(take), dtype=np.int64)
    s_nl, s_al = nl[take].copy(), al[take].copy()
    s_nt_off, s_aa_off = nt_off[take].copy(), aa_off[take].copy()
    score = np.zeros(len(take), dtype=np.int32)
    ncig = np.zeros(len(take), dtype=np.int32)
    secs = []
    for _ in range(steps):
        t = fn(threads, len(take), nt.ctypes.data, s_nt_off.ctypes.data, s_nl.ctypes.data, aa.ctypes.data,
               s_aa_off.ctypes.data, s_al.ctypes.data, C.addressof(opt.c), score.ctypes.data, ncig.ctypes.data)
        secs.append(t)
    sample = (f"{len(take)} of {n} DP jobs (seeded random subset, {acc / 1e9:.2f} G cells), ns_global_gs_auto "
              f"with CIGAR, {threads} threads via kt_for")
    return acc / min(secs) / 1e9, threads, kind, sample, secs, acc


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    jobs = make_jobs(args, 1)
    nt, aa, nt_off, aa_off, nl, al, _ = pack(jobs)
    opt = Options(flag=NS_F_CIGAR)
    per_step = args.cpu_seconds / 2
    gcups_w, threads, kind, sample, secs_w, cells = cpu_baseline(jobs, nt, aa, nt_off, aa_off, nl, al, opt,
                                                                 per_step, steps=max(args.warmup, 0) or 1)
    gcups, threads, kind, sample, secs, cells = cpu_baseline(jobs, nt, aa, nt_off, aa_off, nl, al, opt, per_step,
                                                             steps=args.steps)
    total = sum(secs)
    value = cells * len(secs) / total / 1e9
    line = {"metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total / len(secs) * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "n_jobs": int(len(nl)), "step": "bounded sample of the workload"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


REF_CUDA_SO = os.path.join(ROOT, "oracle", "_ref", "libnscuda_ref.so")


def main_refgpu(args):
    """The reference's own CUDA global DP (nasw-cuda.cu compiled for sm_100a from its sources,
    oracle/_ref/libnscuda_ref.so) on this GPU: its request queue over a bounded seeded sample of
    the headline jobs (ns_gpu_submit from 16 host threads, then ns_gpu_wait, which includes its
    host backtrack from the full trace copied back), and the latency of ns_gpu_global on the
    single-locus job (500 aa, 20 kb).  Runs in its own process (its own CUDA context); prints
    one JSON object."""
    if not os.path.exists(REF_CUDA_SO):
        print(json.dumps({"unavailable": "oracle/_ref/libnscuda_ref.so not built"}), flush=True)
        return 0
    lib = C.CDLL(REF_CUDA_SO)
    lib.ref_gpu_queue_bench.restype = C.c_double
    lib.ref_gpu_queue_bench.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int32] + [C.c_void_p] * 8
    lib.ref_gpu_global_latency.restype = C.c_int32
    lib.ref_gpu_global_latency.argtypes = [C.c_int32, C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32,
                                           C.c_int32, C.c_void_p]
    opt = Options(flag=NS_F_CIGAR)
    jobs = make_jobs(args, 1)
    rng = np.random.default_rng(777)
    take = np.sort(rng.permutation(len(jobs))[: args.ref_jobs])
    sub = [jobs[q] for q in take]
    nt, aa, nt_off, aa_off, nl, al, _ = pack(sub)
    n = len(sub)
    score = np.zeros(n, np.int32)
    taken = np.zeros(n, np.int32)
    # warm-up: the queue's threads, the module load and the device buffers
    w = min(n, 8)
    lib.ref_gpu_queue_bench(0, 16, C.addressof(opt.c), w, nt.ctypes.data, nt_off.ctypes.data, nl.ctypes.data,
                            aa.ctypes.data, aa_off.ctypes.data, al.ctypes.data, score.ctypes.data, taken.ctypes.data)
    secs = lib.ref_gpu_queue_bench(0, 16, C.addressof(opt.c), n, nt.ctypes.data, nt_off.ctypes.data,
                                   nl.ctypes.data, aa.ctypes.data, aa_off.ctypes.data, al.ctypes.data,
                                   score.ctypes.data, taken.ctypes.data)
    if secs <= 0:
        print(json.dumps({"unavailable": "the reference's ns_gpu_init failed"}), flush=True)
        return 0
    cells = (nl.astype(np.int64) - 2) * al
    ok = taken > 0
    c_nt, c_aa = W.single_locus(seed=0)
    lat = np.zeros(20, np.float64)
    lib.ref_gpu_global_latency(0, C.addressof(opt.c), c_nt, len(c_nt), c_aa, len(c_aa), 20, lat.ctypes.data)
    print(json.dumps({"gcups": round(float(cells[ok].sum()) / secs / 1e9, 3), "jobs": int(n), "taken": int(ok.sum()),
                      "cells": int(cells[ok].sum()), "seconds": round(secs, 3),
                      "config0_ms_median": round(float(np.median(lat[2:])) * 1e3, 3),
                      "sample": f"{n} of {len(jobs)} DP jobs of the headline batch (seeded random subset), "
                                "ns_gpu_submit from 16 threads then ns_gpu_wait (kernel, D2H of the full trace, "
                                "host backtrack)"}), flush=True)
    return 0


def config0_latency(local):
    """Latency of one DP on the single-locus job (500 aa protein, 20 kb window, CIGAR): this
    library's bulk entry point with one job and its request queue (ns_gpu_global), and the
    reference's SSE kernel on one host core.  Medians of 20 calls after 3 warm-up calls."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    opt = Options(flag=NS_F_CIGAR)
    c_nt, c_aa = W.single_locus(seed=0)
    out = {"job": f"single locus: protein {len(c_aa)} aa, window {len(c_nt)} nt, "
                  f"{(len(c_nt) - 2) * len(c_aa) / 1e6:.1f} M cells, with CIGAR"}
    eng = L.Engine(local)
    t = []
    for k in range(23):
        t0 = time.perf_counter()
        eng.align_host(opt, [(c_nt, c_aa)])
        t.append(time.perf_counter() - t0)
    eng.close()
    out["ours_ms"] = round(statistics.median(t[3:]) * 1e3, 3)
    if L.gpu_init(local):
        t = []
        for k in range(23):
            t0 = time.perf_counter()
            L.gpu_global(c_nt, c_aa, opt)
            t.append(time.perf_counter() - t0)
        out["ours_queue_ms"] = round(statistics.median(t[3:]) * 1e3, 3)
    ref = O.ref_lib()
    if ref is not None:
        fn = ref.ref_bench_global
        fn.restype = C.c_double
        fn.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 9
        ntb = np.frombuffer(c_nt, np.uint8)
        aab = np.frombuffer(c_aa, np.uint8)
        z64 = np.zeros(1, np.int64)
        nl1 = np.array([len(c_nt)], np.int32)
        al1 = np.array([len(c_aa)], np.int32)
        sc = np.zeros(1, np.int32)
        nc = np.zeros(1, np.int32)
        t = [fn(1, 1, ntb.ctypes.data, z64.ctypes.data, nl1.ctypes.data, aab.ctypes.data, z64.ctypes.data,
                al1.ctypes.data, C.addressof(opt.c), sc.ctypes.data, nc.ctypes.data) for _ in range(23)]
        out["reference_sse_1core_ms"] = round(statistics.median(t[3:]) * 1e3, 3)
    return out


def main():
    args = parse()
    if args.workload == "refgpu":
        return main_refgpu(args)
    if args.workload == "ext":
        return run_reference_ext(args) if args.impl == "reference" else main_ext(args)
    if args.workload == "hmm":
        return run_reference_hmm(args) if args.impl == "reference" else main_hmm(args)
    if args.workload == "gapless":
        return run_reference_gapless(args) if args.impl == "reference" else main_gapless(args)
    if args.workload == "forward":
        return main_forward(args)
    if args.workload == "prefilter":
        return main_prefilter(args)
    if args.workload == "extra":
        return main_extra(args)
    if args.workload == "prescreen":
        return main_prescreen(args)
    if args.workload == "chain":
        return main_chain(args)
    if args.workload == "seed":
        return main_seed(args)
    if args.workload == "seed_hmm":
        return main_seed_hmm(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    R = Ranks("nccl")
    rank, world, local, barrier, max_over_ranks = R.rank, R.world, R.local, R.barrier, R.max

    jobs = make_jobs(args, R.seed(1))
    nt, aa, nt_off, aa_off, nl, al, tab = pack(jobs)
    n = len(jobs)
    cells = int(((nl.astype(np.int64) - 2) * al).sum())
    cells_all = R.sum(cells)  # units of the whole job (every rank takes this collective)
    opt = Options(flag=NS_F_CIGAR)
    eng = L.Engine(local, int(args.trace_budget_gb * (1 << 30)))
    cap = n * 4096
    d_nt = torch.from_numpy(nt.copy()).to("cuda")
    d_aa = torch.from_numpy(aa.copy()).to("cuda")
    d_res = torch.zeros(n * C.sizeof(SpliceResult), dtype=torch.uint8, device="cuda")
    d_cig = torch.zeros(cap, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    total = C.c_int64()

    def step_device():
        ok = eng.lib.pl_splice_batch_device(eng.h, opt.ptr, tab, n, d_nt.data_ptr(), d_aa.data_ptr(), None,
                                            d_res.data_ptr(), d_cig.data_ptr(), cap, C.byref(total),
                                            stream.cuda_stream)
        if not ok:
            raise RuntimeError("pl_splice_batch_device: " + L.error())

    tuning = {"r4_rows": None, "coop_ratio": None, "autotuned": False}
    if not args.no_autotune:
        from protlocus_b200 import tuning as TU
        tf = TU.TuningFile(args.tuning_json)
        klass = TU.shape_class(nl, al)
        hit = tf.get(klass)
        if hit is not None:  # this shape class was tuned before: no search
            eng.set_tuning(hit["r4_rows"], hit["coop_ratio"])
            tuning = {**hit, "autotuned": False, "shape_class": klass, "from": tf.path}
        else:
            r4, ratio = C.c_int32(), C.c_double()
            if not eng.lib.pl_engine_autotune(eng.h, opt.ptr, tab, n, d_nt.data_ptr(), d_aa.data_ptr(), None,
                                              C.byref(r4), C.byref(ratio)):
                raise RuntimeError("pl_engine_autotune: " + L.error())
            tuning = {"r4_rows": r4.value, "coop_ratio": ratio.value, "autotuned": True, "shape_class": klass}
            try:
                tf.put(klass, r4.value, ratio.value, jobs=int(n), device=torch.cuda.get_device_name(local))
                tf.save()
                tuning["saved_to"] = tf.path
            except OSError:
                pass
    else:
        tuning.update(eng.tuning())
    for _ in range(args.warmup):
        step_device()
    res = (SpliceResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
    bad = sum(1 for r in res if r.status != 0)
    if bad:
        raise RuntimeError(f"{bad} jobs failed")
    int32_peak, i16x2_peak = L.measure_int_peak(local)
    peak = max(int32_peak, i16x2_peak)

    clocks = Clocks(local)
    launches0 = L.load().pl_kernel_launch_count()
    replays0 = int(eng.lib.pl_engine_graph_replays(eng.h))
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step_device()  # a repeated batch: replayed from the engine's captured graph
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    replays = int(eng.lib.pl_engine_graph_replays(eng.h)) - replays0
    t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    value = cells_all * args.steps / t / 1e9
    # the phase times of the roofline: the same steps again with the engine's CUDA events between the launches
    eng.set_timing(True)
    for _ in range(max(1, min(args.steps, 3))):
        step_device()
    torch.cuda.synchronize()
    tm = eng.times()
    plan = eng.last_plan()
    n_pairs = eng.last_pairs()
    dp_s = tm["dp_ms"] / 1e3
    achieved = tm["cells"] * OPS_PER_CELL / dp_s if dp_s > 0 else 0.0
    dp_gcups = tm["cells"] / dp_s / 1e9 if dp_s > 0 else 0.0

    e2e = None
    if not args.no_e2e:
        h_nt = torch.from_numpy(nt.copy()).pin_memory()
        h_aa = torch.from_numpy(aa.copy()).pin_memory()
        h_cig = torch.zeros(cap, dtype=torch.int32).pin_memory()
        h_res = (SpliceResult * n)()
        est = torch.cuda.ExternalStream(eng.stream)

        def step_host():
            ok = eng.lib.pl_splice_batch_host(eng.h, opt.ptr, tab, n, h_nt.data_ptr(), h_nt.numel(), h_aa.data_ptr(),
                                              h_aa.numel(), None, 0, h_res, h_cig.data_ptr(), cap)
            if not ok:
                raise RuntimeError("pl_splice_batch_host: " + L.error())

        for _ in range(max(1, args.warmup)):
            step_host()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(est)
        for _ in range(args.steps):
            step_host()
        e1.record(est)
        torch.cuda.synchronize()
        barrier()
        te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        d2h = n * C.sizeof(SpliceResult) + 4 * sum(h_res[q].n_cigar for q in range(n))
        e2e = {"value": round(cells_all * args.steps / te / 1e9, 3), "unit": "GCUPS",
               "h2d_bytes_per_step": int(nt.nbytes + aa.nbytes + n * C.sizeof(SpliceJob)),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": round(te / args.steps * 1e3, 2),
               "api": "pl_splice_batch_host (C ABI, pinned host buffers)"}

    cpu = None
    if rank == 0:
        gcups, threads, kind, sample, _secs, _acc = cpu_baseline(jobs, nt, aa, nt_off, aa_off, nl, al, opt,
                                                                 args.cpu_seconds)
        cpu = {"value": round(gcups, 3), "unit": "GCUPS", "cores": threads, "kind": kind, "sample": sample}

    # the second half of the metric: learned-prefilter loci/s against the plain path, same run
    pf = None
    eng.close()
    del d_nt, d_aa, d_res, d_cig
    torch.cuda.empty_cache()
    lat = config0_latency(local) if rank == 0 else None
    refgpu = None
    if rank == 0 and not args.no_refgpu:  # the reference's CUDA kernel as the GPU bar, in its own process
        try:
            pr = subprocess.run([sys.executable, os.path.abspath(__file__), "--workload", "refgpu", "--ref-jobs",
                                 str(args.ref_jobs), "--pairs", str(args.pairs)], capture_output=True, text=True,
                                timeout=600)
            refgpu = json.loads(pr.stdout.strip().splitlines()[-1]) if pr.returncode == 0 and pr.stdout.strip() \
                else {"unavailable": f"child exited {pr.returncode}: {pr.stderr.strip()[-200:]}"}
        except Exception as ex:  # a timeout or a parse error: report it, keep the line
            refgpu = {"unavailable": f"{type(ex).__name__}: {str(ex)[:200]}"}
        if lat is not None and "config0_ms_median" in refgpu:
            lat["reference_gpu_queue_ms"] = refgpu.pop("config0_ms_median")
    if not args.no_prefilter:
        pf = prefilter_measure(args, R, local, min(args.steps, 5), 3, 0.0)
        if pf is not None:
            pf = {k: pf[k] for k in ("metric", "value", "unit", "ms_per_step", "plain", "speedup_vs_plain",
                                     "locus_recall", "plain_loci", "learned_loci", "extra_loci", "candidates_per_s",
                                     "output_recall", "kept", "fallback", "phase_s", "e2e", "gpu_launches", "config")}
            if cpu is not None:
                cpc = pf["plain"]["cells_per_step"] / PF_N_PROT
                pf["cpu_baseline"] = {"value": round(cpu["value"] * 1e9 / cpc, 2), "unit": "loci/s",
                                      "cores": cpu["cores"], "kind": cpu["kind"],
                                      "sample": "the headline's CPU GCUPS converted at this set's mean cells per locus "
                                                "(plain path on the CPU)"}

    hmm = None
    if rank == 0 and world == 1 and not args.no_hmm:  # the profile-HMM configuration, in its own process
        try:
            pr = subprocess.run([sys.executable, os.path.abspath(__file__), "--workload", "hmm", "--hmm-shape", "genome",
                                 "--profiles", "1000", "--steps", "2", "--warmup", "1"], capture_output=True, text=True,
                                timeout=900)
            h = json.loads(pr.stdout.strip().splitlines()[-1]) if pr.returncode == 0 and pr.stdout.strip() else None
            hmm = {k: h.get(k) for k in ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "e2e",
                                         "gpu_launches", "cpu_baseline", "clocks")} if h else \
                {"unavailable": f"child exited {pr.returncode}: {pr.stderr.strip()[-200:]}"}
            if h:
                hmm["roofline"] = {k: h["roofline"].get(k) for k in ("kernel", "achieved", "peak", "unit", "frac")}
                hmm["config"] = {"workload": h["config"].get("workload")}
        except Exception as ex:
            hmm = {"unavailable": f"{type(ex).__name__}: {str(ex)[:200]}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
            "config": {"workload": WORKLOAD if not args.uniform else "profiling case " + args.uniform, "n_jobs": n, "cells_per_step": cells, "seed": "1+rank",
                       "l2": "inputs and the per-step traceback arena (tens of GB) are far larger than L2",
                       "waves": plan["waves"], "coop_jobs": plan["coop"], "parallelism": f"{world} independent ranks",
                       "tuning": tuning, "int16x2_pairs": n_pairs,
                       "trace_budget_gb": args.trace_budget_gb or "engine default (40% of free memory, <= 72)",
                       "graph_replays_in_timed_steps": replays},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "int", "kernel": "k_splice_pair" if n_pairs else "k_splice_dp", "achieved": achieved,
                         "peak": peak, "unit": "lane-ops/s", "frac": achieved / peak if peak else None,
                         "traffic": (int((PAIR_DRAM_BYTES_PER_CELL if n_pairs else DP_DRAM_BYTES_PER_CELL)
                                         * tm["cells"] / tm["dp_launches"]) if tm["dp_launches"] else None),
                         "traffic_source": ("ncu dram bytes read+write of one k_splice_pair launch on the uniform "
                                            "4736x2000x250 case (2.20 B/cell)" if n_pairs else
                                            "ncu dram bytes read+write of one k_splice_dp launch on the uniform "
                                            "2400x2000x350 case (2.08 B/cell)") + ", scaled by this run's cells per launch",
                         "ops_per_cell": OPS_PER_CELL, "dp_kernel_gcups": round(dp_gcups, 3),
                         "peak_source": "measured live: pl_measure_int_peak (int32 %.3g, int16x2 %.3g lane-ops/s)"
                                        % (int32_peak, i16x2_peak),
                         "phase_ms_per_step": {k: round(v / max(1, min(args.steps, 3)), 2) for k, v in tm.items()
                                               if k.endswith("_ms")},
                         "phase_source": "engine CUDA events over separate steps after the timed region"},
            "cpu_baseline": cpu,
            "clocks": clk,
            "prefilter": pf,
            "reference_gpu": refgpu,
            "hmm": hmm,
            "config0_latency": lat,
        }
        print(json.dumps(line), flush=True)
    R.close()
    return 0


# ---------------------------------------------------------------------------- extension DP

EXT_METRIC = "extension-DP GCUPS (bit-exact, nominal cells (nl-2)*al per request) at 1 B200"
EXT_OPS_PER_CELL = 31  # int16 lane-ops per cell of the score-only kernel, counted from nasw-sse.c:366-419
EXT_WORKLOAD = ("batched extension DP: 65536 requests, protein window 64-256 aa, nt window 3x + 60-600 nt slack "
                "(+ introns), alternating left/right, mutated gene copy over 30-100% of the window then random "
                "sequence (x-drop ends the DP), ProtLocus default scoring")


def ext_pack(reqs, width=0):
    n = len(reqs)
    nl = np.array([len(a) for a, _, _ in reqs], dtype=np.int32)
    al = np.array([len(b) for _, b, _ in reqs], dtype=np.int32)
    flag = np.array([f for _, _, f in reqs], dtype=np.int32)
    nt_off = np.zeros(n, dtype=np.int64)
    aa_off = np.zeros(n, dtype=np.int64)
    nt_off[1:] = np.cumsum(nl[:-1])
    aa_off[1:] = np.cumsum(al[:-1])
    nt = np.frombuffer(b"".join(a for a, _, _ in reqs), dtype=np.uint8)
    aa = np.frombuffer(b"".join(b for _, b, _ in reqs), dtype=np.uint8)
    tab = (ExtJob * n)()
    for q in range(n):
        j = tab[q]
        j.nt_off, j.aa_off, j.ss_off, j.pssm_off = int(nt_off[q]), int(aa_off[q]), -1, -1
        j.nl, j.al, j.flag, j.width = int(nl[q]), int(al[q]), int(flag[q]), width
    return nt, aa, nt_off, aa_off, nl, al, flag, tab


def cpu_baseline_ext(nt, aa, nt_off, aa_off, nl, al, flag, opt, target_s, steps=1):
    """The reference's ns_global_gs16b with each request's extension flag over a bounded random
    sample, all host threads (kt_for).  Returns (nominal GCUPS, threads, kind, sample, secs, cells)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    threads = os.cpu_count() or 1
    ref = O.ref_lib()
    if ref is None:
        raise RuntimeError("the extension CPU baseline needs oracle/_ref/libnsref.so (make -C oracle ref)")
    fn = ref.ref_bench_ext
    fn.restype = C.c_double
    fn.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 11
    n = len(nl)
    perm = np.random.default_rng(12345).permutation(n)
    cells = (nl.astype(np.int64) - 2) * al
    budget = target_s * 1.0e9 * threads  # ~1 GCUPS per thread (nominal cells) for the AVX2 kernel
    k = int(np.searchsorted(np.cumsum(cells[perm]), budget)) + 1
    take = np.sort(perm[:min(k, n)])
    acc = int(cells[take].sum())
    s_nl, s_al, s_fl = nl[take].copy(), al[take].copy(), flag[take].copy()
    s_nt_off, s_aa_off = nt_off[take].copy(), aa_off[take].copy()
    out = [np.zeros(len(take), dtype=np.int32) for _ in range(3)]
    secs = []
    for _ in range(steps):
        secs.append(fn(threads, len(take), nt.ctypes.data, s_nt_off.ctypes.data, s_nl.ctypes.data, aa.ctypes.data,
                       s_aa_off.ctypes.data, s_al.ctypes.data, s_fl.ctypes.data, C.addressof(opt.c),
                       out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data))
    sample = (f"{len(take)} of {n} extension requests (seeded random subset, {acc / 1e9:.2f} G nominal cells), "
              f"ns_global_gs16b with NS_F_EXT_LEFT/RIGHT, {threads} threads via kt_for")
    return acc / min(secs) / 1e9, threads, "reference", sample, secs, acc


def run_reference_ext(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    reqs = W.ext_requests(args.requests, seed=2)
    nt, aa, nt_off, aa_off, nl, al, flag, _ = ext_pack(reqs)
    opt = Options()
    per_step = args.cpu_seconds / 2
    cpu_baseline_ext(nt, aa, nt_off, aa_off, nl, al, flag, opt, per_step, steps=max(args.warmup, 1))
    gcups, threads, kind, sample, secs, cells = cpu_baseline_ext(nt, aa, nt_off, aa_off, nl, al, flag, opt, per_step,
                                                                 steps=args.steps)
    value = cells * len(secs) / sum(secs) / 1e9
    line = {"metric": EXT_METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sum(secs) / len(secs) * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
            "impl": "reference", "config": {"workload": EXT_WORKLOAD, "n_requests": int(len(nl)),
                                            "step": "bounded sample of the workload"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main_ext(args):
    import torch
    R = Ranks("nccl")
    rank, world, local, barrier, max_over_ranks = R.rank, R.world, R.local, R.barrier, R.max

    reqs = W.ext_requests(args.requests, seed=R.seed(2))
    nt, aa, nt_off, aa_off, nl, al, flag, tab = ext_pack(reqs)
    n = len(reqs)
    nominal = int(((nl.astype(np.int64) - 2) * al).sum())
    nominal_all, n_all = R.sum(nominal), R.sum(n)  # whole job (every rank takes these collectives)
    opt = Options()
    eng = L.Engine(local)
    d_nt = torch.from_numpy(nt.copy()).to("cuda")
    d_aa = torch.from_numpy(aa.copy()).to("cuda")
    d_res = torch.zeros(n * C.sizeof(ExtResult), dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB): written between steps
    stream = torch.cuda.current_stream()

    def step_device():
        if not eng.lib.pl_ext_batch_device(eng.h, opt.ptr, tab, n, d_nt.data_ptr(), d_aa.data_ptr(), None, None,
                                           d_res.data_ptr(), stream.cuda_stream):
            raise RuntimeError("pl_ext_batch_device: " + L.error())

    for _ in range(args.warmup):
        step_device()
    res = (ExtResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
    if any(r.status != 0 for r in res):
        raise RuntimeError("extension requests failed")
    cells_run, _ = eng.ext_last_cells()
    int32_peak, i16x2_peak = L.measure_int_peak(local)
    peak = max(int32_peak, i16x2_peak)

    clocks = Clocks(local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_device()
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
    barrier()
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    t = max_over_ranks(t)
    value = nominal_all * args.steps / t / 1e9
    tm = eng.times()
    dp_s = tm["dp_ms"] / 1e3
    achieved = tm["cells"] * EXT_OPS_PER_CELL / dp_s if dp_s > 0 else 0.0

    e2e = None
    if not args.no_e2e:
        h_nt = torch.from_numpy(nt.copy()).pin_memory()
        h_aa = torch.from_numpy(aa.copy()).pin_memory()
        h_res = (ExtResult * n)()
        est = torch.cuda.ExternalStream(eng.stream)

        def step_host():
            if not eng.lib.pl_ext_batch_host(eng.h, opt.ptr, tab, n, h_nt.data_ptr(), h_nt.numel(), h_aa.data_ptr(),
                                             h_aa.numel(), None, 0, None, 0, h_res):
                raise RuntimeError("pl_ext_batch_host: " + L.error())

        for _ in range(max(1, args.warmup)):
            step_host()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(est)
        for _ in range(args.steps):
            step_host()
        e1.record(est)
        torch.cuda.synchronize()
        barrier()
        te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        e2e = {"value": round(nominal_all * args.steps / te / 1e9, 3), "unit": "GCUPS",
               "h2d_bytes_per_step": int(nt.nbytes + aa.nbytes + n * C.sizeof(ExtJob)),
               "d2h_bytes_per_step": int(n * C.sizeof(ExtResult)), "ms_per_step": round(te / args.steps * 1e3, 2),
               "requests_per_s": round(n_all * args.steps / te, 1),
               "api": "pl_ext_batch_host (C ABI, pinned host buffers)"}

    cpu = None
    if rank == 0:
        gcups, threads, kind, sample, _s, _c = cpu_baseline_ext(nt, aa, nt_off, aa_off, nl, al, flag, opt,
                                                                args.cpu_seconds)
        cpu = {"value": round(gcups, 3), "unit": "GCUPS", "cores": threads, "kind": kind, "sample": sample}
    if rank == 0:
        line = {
            "metric": EXT_METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
            "config": {"workload": EXT_WORKLOAD, "n_requests": n, "nominal_cells_per_step": nominal,
                       "algorithmic_cells_per_step": int(cells_run), "seed": "2+rank",
                       "stripe_width": "host rule (16 lanes on an AVX2 host, as the reference CPU kernel)",
                       "l2": "a 256 MB buffer is written between timed steps", "parallelism": f"{world} independent ranks"},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "int", "kernel": "k_ext_dp", "achieved": achieved, "peak": peak,
                         "unit": "lane-ops/s", "frac": achieved / peak if peak else None, "traffic": None,
                         "ops_per_cell": EXT_OPS_PER_CELL,
                         "dp_kernel_gcups_algorithmic": round(tm["cells"] / dp_s / 1e9, 3) if dp_s > 0 else None,
                         "peak_source": "measured live: pl_measure_int_peak (int32 %.3g, int16x2 %.3g lane-ops/s)"
                                        % (int32_peak, i16x2_peak),
                         "phase_ms_per_step": {"prep_ms": round(tm["prep_ms"] / args.steps, 3),
                                               "dp_ms": round(tm["dp_ms"] / args.steps, 3)}},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    R.close()
    return 0


# ---------------------------------------------------------------------------- profile-HMM DP

HMM_METRIC = "profile-HMM DP GCUPS (exact int32, cells = frame-0 codon rows x profile length) at 1 B200"
HMM_OPS_PER_CELL = 17  # int32 ops per cell of mp_hmm_dp_score's inner loop (hmm.c:274-285)


def hmm_workload(args, seed):
    from protlocus_b200 import hmm as H
    if args.hmm_shape == "genome":  # the profile-HMM configuration: profiles x six frames of a genome slice
        texts, probs = H.synthetic_profiles(args.profiles, seed=seed, m_min=50, m_max=800)
        profs = H.parse_hmmer3("".join(texts))
        nt, offs, lens, inside = H.genome_scan(probs, seed + 1000, slice_mb=args.genome_slice_mb,
                                               region_nt=args.genome_region_kb * 1000)
        batch = (nt, offs, lens)  # one region set, scored against every profile
        desc = (f"profile-HMM genome scan: {args.profiles} synthetic Plan7 profiles (m uniform 50-800, "
                "Dirichlet-perturbed background, M->M ~0.95, HMMER3 text through the parser) against the six-frame "
                f"translation of a 100 Mb 45%-GC genome with 1000 planted profile-sampled domains; each step scans "
                f"the first {args.genome_slice_mb:g} Mb ({args.genome_slice_mb:g}% of the genome, {inside} planted "
                f"domains) as {len(lens)} regions of {args.genome_region_kb} kb overlapping by 2.4 kb (a domain of "
                "up to 800 codons lies inside one), both strands, frames 0-2; cells = the regions' codons x m")
        return texts, profs, [batch] * len(profs), desc
    texts, probs = H.synthetic_profiles(args.profiles, seed=seed, m_min=50, m_max=800)
    profs = H.parse_hmmer3("".join(texts))
    rng = np.random.default_rng(seed + 1000)
    batches = []
    for pr, p in zip(profs, probs):
        regs = H.regions(rng, p, args.regions, 300, 3000)
        lens = np.array([len(r) for r in regs], dtype=np.int32)
        offs = np.zeros(len(regs), dtype=np.int32)
        offs[1:] = np.cumsum(lens[:-1])
        batches.append((np.concatenate(regs), offs, lens))
    desc = (f"profile-HMM DP: {args.profiles} synthetic Plan7 profiles (m uniform 50-800, Dirichlet-perturbed "
            f"background, M->M ~0.95, HMMER3 text through the parser), {args.regions} regions each of 300-3000 nt "
            "(45% GC, half with a planted profile-sampled domain), one batch per profile")
    return texts, profs, batches, desc


def cpu_baseline_hmm(texts, batches, target_s):
    """The reference's mp_hmm_dp_score (its own parser's tables) over kt_for on a bounded sample of regions."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    ref = O.ref_lib()
    if ref is None:
        raise RuntimeError("the HMM CPU baseline needs oracle/_ref/libnsref.so (make -C oracle ref)")
    ref.mp_hmm_open.restype, ref.mp_hmm_open.argtypes = C.c_void_p, [C.c_char_p]
    ref.mp_hmm_read1.restype, ref.mp_hmm_read1.argtypes = C.c_void_p, [C.c_void_p]
    ref.mp_hmm_length.argtypes = [C.c_void_p]
    ref.mp_hmm_close.argtypes = [C.c_void_p]
    ref.mp_hmm_destroy.argtypes = [C.c_void_p]
    ref.ref_bench_hmm.restype = C.c_double
    ref.ref_bench_hmm.argtypes = [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    threads = os.cpu_count() or 1
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write("".join(texts))
        path = f.name
    fh = ref.mp_hmm_open(path.encode())
    hs = [ref.mp_hmm_read1(fh) for _ in texts]
    budget = target_s * 0.8e9 * threads / len(texts)  # ~0.8 GCUPS per thread, spread over the profiles
    cells = secs = 0.0
    n_reg = 0
    for h, (nt, offs, lens) in zip(hs, batches):
        m = ref.mp_hmm_length(h)
        k = int(np.searchsorted(np.cumsum((lens // 3).astype(np.int64) * m), budget)) + 1
        k = min(k, len(lens))
        score = np.zeros(k, dtype=np.int32)
        secs += ref.ref_bench_hmm(threads, h, k, nt.ctypes.data, offs.ctypes.data, lens.ctypes.data, score.ctypes.data)
        cells += float((lens[:k] // 3).astype(np.int64).sum() * m)
        n_reg += k
    for h in hs:
        ref.mp_hmm_destroy(h)
    ref.mp_hmm_close(fh)
    os.unlink(path)
    sample = (f"{n_reg} regions over {len(texts)} profiles ({cells / 1e9:.2f} G cells), mp_hmm_dp_score, "
              f"{threads} threads via kt_for")
    return cells / secs / 1e9, threads, sample, secs, cells


def run_reference_hmm(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    texts, _profs, batches, desc = hmm_workload(args, 3)
    cpu_baseline_hmm(texts, batches, args.cpu_seconds / 4)
    vals, tot = [], 0.0
    for _ in range(args.steps):
        v, threads, sample, secs, _c = cpu_baseline_hmm(texts, batches, args.cpu_seconds / 2)
        vals.append(v)
        tot += secs
    value = statistics.mean(vals)
    line = {"metric": HMM_METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot / args.steps * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "impl": "reference", "config": {"workload": desc, "step": "bounded sample of the workload"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main_hmm(args):
    import torch
    from protlocus_b200 import hmm as H
    R = Ranks("nccl")
    rank, world, local, barrier, max_over_ranks = R.rank, R.world, R.local, R.barrier, R.max

    texts, profs, batches, desc = hmm_workload(args, R.seed(3))
    ca = H.codon_alpha()
    eng = L.Engine(local)
    hp = [L.HmmProfile(p["emit"], p["trans"], ca, local) for p in profs]
    cells = sum(int((ln // 3).astype(np.int64).sum()) * p["m"] for p, (_, _, ln) in zip(profs, batches))
    cells_all = R.sum(cells)  # whole job (every rank takes this collective)
    dev_nt = {}  # one device copy per distinct region set (the genome scan shares one across profiles)
    d_nt = [dev_nt.setdefault(id(nt), torch.from_numpy(nt).to("cuda")) for nt, _, _ in batches]
    d_sc = [torch.zeros(len(ln), dtype=torch.int32, device="cuda") for _, _, ln in batches]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    shared = len(dev_nt) == 1 and len(hp) > 1  # one region set for every profile: one call for all of them
    if shared:
        _, offs0, lens0 = batches[0]
        d_all = torch.zeros(len(hp) * len(lens0), dtype=torch.int32, device="cuda")
        handles = (C.c_void_p * len(hp))(*[p.h for p in hp])

    def step_device():
        if shared:  # planned and translated once, the profiles' launches side by side (pl_hmm_score_many_device)
            if not eng.lib.pl_hmm_score_many_device(eng.h, handles, len(hp), len(lens0), d_nt[0].data_ptr(),
                                                    offs0.ctypes.data, lens0.ctypes.data, d_all.data_ptr(),
                                                    stream.cuda_stream):
                raise RuntimeError("pl_hmm_score_many_device: " + L.error())
            return
        for p, (nt, offs, lens), dn, ds in zip(hp, batches, d_nt, d_sc):
            if not eng.lib.pl_hmm_score_device(eng.h, p.h, len(lens), dn.data_ptr(), offs.ctypes.data,
                                               lens.ctypes.data, ds.data_ptr(), stream.cuda_stream):
                raise RuntimeError("pl_hmm_score_device: " + L.error())

    for _ in range(args.warmup):
        step_device()
    int32_peak, i16x2_peak = L.measure_int_peak(local)
    clocks = Clocks(local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_device()
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
    barrier()
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    t = max_over_ranks(t)
    value = cells_all * args.steps / t / 1e9
    tm = eng.times()
    dp_s = tm["dp_ms"] / 1e3
    achieved = tm["cells"] * HMM_OPS_PER_CELL / dp_s if dp_s > 0 else 0.0

    e2e = None
    if not args.no_e2e:
        pin_nt = {}
        h_nt = [pin_nt.setdefault(id(nt), torch.from_numpy(nt).pin_memory()) for nt, _, _ in batches]
        h_sc = [np.zeros(len(ln), dtype=np.int32) for _, _, ln in batches]
        est = torch.cuda.ExternalStream(eng.stream)

        if shared:
            h_all = np.zeros((len(hp), len(lens0)), dtype=np.int32)

        def step_host():
            if shared:  # the region set uploaded once for every profile (pl_hmm_score_many_host)
                if not eng.lib.pl_hmm_score_many_host(eng.h, handles, len(hp), len(lens0), h_nt[0].data_ptr(),
                                                      h_nt[0].numel(), offs0.ctypes.data, lens0.ctypes.data,
                                                      h_all.ctypes.data):
                    raise RuntimeError("pl_hmm_score_many_host: " + L.error())
                for k in range(len(hp)):
                    h_sc[k][:] = h_all[k]
                return
            for p, (nt, offs, lens), hn, hs in zip(hp, batches, h_nt, h_sc):
                if not eng.lib.pl_hmm_score_host(eng.h, p.h, len(lens), hn.data_ptr(), hn.numel(), offs.ctypes.data,
                                                 lens.ctypes.data, hs.ctypes.data):
                    raise RuntimeError("pl_hmm_score_host: " + L.error())

        for _ in range(max(1, args.warmup)):
            step_host()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(est)
        for _ in range(args.steps):
            step_host()
        e1.record(est)
        torch.cuda.synchronize()
        barrier()
        te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        h2d = (batches[0][0].nbytes + 8 * len(lens0)) if shared else sum(nt.nbytes + 8 * len(ln) for nt, _, ln in batches)
        e2e = {"value": round(cells_all * args.steps / te / 1e9, 3), "unit": "GCUPS",
               "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(sum(4 * len(ln) for _, _, ln in batches)),
               "ms_per_step": round(te / args.steps * 1e3, 2),
               "api": ("pl_hmm_score_many_host" if shared else "pl_hmm_score_host") + " (C ABI, pinned host buffers)"}
        # parity of this run's scores with the device path
        ref_sc = (list(d_all.cpu().numpy().reshape(len(hp), -1)) if shared else [ds.cpu().numpy() for ds in d_sc])
        if any((a != b).any() for a, b in zip(ref_sc, h_sc)):
            raise RuntimeError("host and device HMM scores differ")

    cpu = None
    if rank == 0:
        v, threads, sample, _s, _c = cpu_baseline_hmm(texts, batches, args.cpu_seconds)
        cpu = {"value": round(v, 3), "unit": "GCUPS", "cores": threads, "kind": "reference", "sample": sample}
    if rank == 0:
        line = {
            "metric": HMM_METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": desc, "cells_per_step": cells, "seed": "3+rank",
                       "l2": "a 256 MB buffer is written between timed steps", "parallelism": f"{world} independent ranks"},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "int", "kernel": "k_hmm_dp", "achieved": achieved, "peak": int32_peak,
                         "unit": "lane-ops/s", "frac": achieved / int32_peak if int32_peak else None, "traffic": None,
                         "ops_per_cell": HMM_OPS_PER_CELL,
                         "dp_kernel_gcups": round(tm["cells"] / dp_s / 1e9, 3) if dp_s > 0 else None,
                         "peak_source": "measured live: pl_measure_int_peak, int32 add+max chains (%.3g lane-ops/s)"
                                        % int32_peak,
                         "phase_ms_per_step": {"codons_ms": round(tm["prep_ms"] / args.steps, 3),
                                               "dp_ms": round(tm["dp_ms"] / args.steps, 3)},
                         "api": "pl_hmm_score_many_device: every profile's launch side by side on the engine's HMM "
                                "streams (dp_ms spans the translation and every launch)" if shared else
                                "pl_hmm_score_device per profile"},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    for p in hp:
        p.close()
    eng.close()
    R.close()
    return 0


# ---------------------------------------------------------------------------- gapless prefilter

GL_METRIC = "gapless prefilter G seed positions/s (anchors x block_width, bit-exact scores) at 1 B200"
GL_OPS_PER_POS = 12  # int ops per seed position: kmer=6 score lookups + adds (nasw-cuda.cu:1204-1214)


def gapless_inputs(args, seed):
    from protlocus_b200.abi import BLOSUM62, make_tables, set_stop_sc
    w = W.gapless_workload(10000, 100_000_000, args.candidates, seed=seed, fixed_anchors=True)
    mat = np.ascontiguousarray(set_stop_sc(BLOSUM62, 23), dtype=np.int8)
    desc = (f"gapless prefilter: 100 Mb genome (64 contigs, 45% GC) with 10000 planted 500-aa genes (25% divergence, "
            f"3 introns, either strand), {args.candidates} candidates x 8 anchors = {len(w['anchors'])} anchors "
            "(30% on their gene, 70% decoys), block_width 256, kmer 6, xdrop 40, BLOSUM62 with stop -23")
    return w, mat, make_tables()[2], desc


def cpu_port_gapless(w, mat, codon, target_s):
    """The C restatement (the reference has no CPU twin of this kernel) on a bounded sample of
    candidates, split across all host threads (ctypes releases the GIL)."""
    import threading
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    threads = os.cpu_count() or 1
    n = len(w["candidates"])
    k = min(n, max(threads, int(target_s * 4000 * threads)))  # ~4000 candidates/s/thread
    cand = w["candidates"][:k].copy()
    out = np.zeros(k, dtype=np.int32)
    lib = O.port_lib()
    f = lib.port_gapless_score_batch
    f.argtypes = [C.c_void_p] * 3 + [C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                     C.c_int32, C.c_void_p, C.c_void_p]
    bounds = np.linspace(0, k, threads + 1).astype(int)

    def run(a, b):
        if b > a:
            f(w["packed"].ctypes.data, w["queries"].ctypes.data, cand[a:].ctypes.data, b - a, w["anchors"].ctypes.data,
              256, 6, 40, mat.ctypes.data, 22, codon.ctypes.data, out[a:].ctypes.data)

    t0 = time.perf_counter()
    th = [threading.Thread(target=run, args=(bounds[i], bounds[i + 1])) for i in range(threads)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    secs = time.perf_counter() - t0
    pos = int(cand["anchor_count"].clip(0, 32).sum()) * 256
    return pos / secs / 1e9, threads, f"{k} of {n} candidates ({pos} seed positions), oracle restatement, {threads} threads", out


def run_reference_gapless(args):
    """The reference's own implementation of this path is its CUDA kernel (no CPU twin exists): built from
    nasw-cuda.cu into oracle/_ref/libnscuda_ref.so and timed through its ns_gpu_gapless_score_batch."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    path = os.path.join(ROOT, "oracle", "_ref", "libnscuda_ref.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libnscuda_ref.so not built"}))
        return 0
    w, mat, codon, desc = gapless_inputs(args, 5)
    ref = C.CDLL(path)
    if not ref.ns_gpu_init(0):
        print(json.dumps({"impl": "reference", "unavailable": "reference ns_gpu_init failed"}))
        return 0
    args_l, keep = L.gapless_args(w, 256, 6, 40, mat, codon)
    ref.ns_gpu_gapless_score_batch.argtypes = L.load().ns_gpu_gapless_score_batch.argtypes
    sc = np.zeros(len(w["candidates"]), dtype=np.int32)
    for _ in range(max(1, args.warmup)):
        ref.ns_gpu_gapless_score_batch(*args_l, sc.ctypes.data)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        if not ref.ns_gpu_gapless_score_batch(*args_l, sc.ctypes.data):
            raise RuntimeError("reference gapless batch failed")
    secs = (time.perf_counter() - t0) / args.steps
    pos = len(w["anchors"]) * 256
    v = pos / secs / 1e9
    line = {"metric": GL_METRIC, "value": round(v, 3), "unit": "G seed positions/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(secs * 1e3, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "implementation": "the reference's CUDA kernel (nasw-cuda.cu) on this GPU, "
                                                           "ns_gpu_gapless_score_batch with its genome cache"},
            "cpu_baseline": None,
            "e2e": {"value": round(v, 3), "unit": "G seed positions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main_gapless(args):
    import torch
    R = Ranks("nccl")
    rank, world, local, barrier, max_over_ranks = R.rank, R.world, R.local, R.barrier, R.max
    w, mat, codon, desc = gapless_inputs(args, R.seed(5))
    n, na = len(w["candidates"]), len(w["anchors"])
    pos = na * 256
    pos_all, n_all = R.sum(pos), R.sum(n)  # whole job (every rank takes these collectives)
    eng = L.Engine(local)
    d = {k: torch.from_numpy(w[k].view(np.uint8).reshape(-1).copy()).to("cuda")
         for k in ("packed", "queries", "candidates", "anchors")}
    d_sc = torch.zeros(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step_device():
        if not eng.lib.pl_gapless_score_device(eng.h, d["packed"].data_ptr(), int(w["bases"]), d["queries"].data_ptr(),
                                               int(w["queries"].size), d["candidates"].data_ptr(), n,
                                               d["anchors"].data_ptr(), na, 256, 6, 40, mat.ctypes.data, 22,
                                               codon.ctypes.data, d_sc.data_ptr(), stream.cuda_stream):
            raise RuntimeError("pl_gapless_score_device: " + L.error())

    for _ in range(args.warmup):
        step_device()
    int32_peak, _ = L.measure_int_peak(local)
    clocks = Clocks(local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step_device()
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
    barrier()
    clk = clocks.stop()
    t = max_over_ranks(t)
    launches = L.load().pl_kernel_launch_count() - launches0
    tm = eng.times()
    k_s = tm["dp_ms"] / 1e3
    steps_walked = int(eng.lib.pl_gapless_last_steps(eng.h))
    value = pos_all * args.steps / t / 1e9
    achieved = pos * args.steps * GL_OPS_PER_POS / k_s if k_s > 0 else 0.0
    # end to end through the reference-facing entry point: host buffers, genome resident after the first call
    assert L.gpu_init(local)
    ref_sc = d_sc.cpu().numpy()
    e_args, keep = L.gapless_args(w, 256, 6, 40, mat, codon)
    h_sc = np.zeros(n, dtype=np.int32)
    for _ in range(max(1, args.warmup)):
        L.load().ns_gpu_gapless_score_batch(*e_args, h_sc.ctypes.data)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        if not L.load().ns_gpu_gapless_score_batch(*e_args, h_sc.ctypes.data):
            raise RuntimeError("ns_gpu_gapless_score_batch failed")
    te = max_over_ranks((time.perf_counter() - t0) / args.steps)
    if (h_sc != ref_sc).any():
        raise RuntimeError("entry points disagree")
    e2e = {"value": round(pos_all / te / 1e9, 3), "unit": "G seed positions/s",
           "h2d_bytes_per_step": int(w["queries"].nbytes + w["candidates"].nbytes + w["anchors"].nbytes + 22 * 22 + 64),
           "d2h_bytes_per_step": int(4 * n), "ms_per_step": round(te * 1e3, 2),
           "api": "ns_gpu_gapless_score_batch (the reference's C entry point; genome resident across calls as in "
                  "nasw-cuda.cu:1362-1367), wall clock per call"}
    cpu = None
    if rank == 0:
        v, threads, sample, out = cpu_port_gapless(w, mat, codon, args.cpu_seconds)
        if (out != ref_sc[:len(out)]).any():
            raise RuntimeError("device scores differ from the restatement")
        cpu = {"value": round(v, 3), "unit": "G seed positions/s", "cores": threads, "kind": "port", "sample": sample}
        line = {"metric": GL_METRIC, "value": round(value, 3), "unit": "G seed positions/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 2),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic",
                "config": {"workload": desc, "candidates": n, "anchors": na, "seed_positions_per_step": pos,
                           "extension_steps_per_step": steps_walked, "candidates_per_s": round(n_all * args.steps / t, 1),
                           "l2": "a 256 MB buffer is written between timed steps (the 50 MB genome itself fits in L2)",
                           "parallelism": f"{world} independent ranks"},
                "e2e": e2e, "gpu_launches": int(launches),
                "roofline": {"bound": "int", "kernel": "k_gapless", "achieved": achieved, "peak": int32_peak,
                             "unit": "lane-ops/s", "frac": achieved / int32_peak if int32_peak else None,
                             "traffic": None, "ops_per_seed_position": GL_OPS_PER_POS,
                             "kernel_ms_per_step": round(tm["dp_ms"] / args.steps, 3),
                             "peak_source": "measured live: pl_measure_int_peak, int32 (%.3g lane-ops/s)" % int32_peak},
                "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line), flush=True)
    eng.close()
    R.close()
    return 0


# ---------------------------------------------------------------------------- recheck Forward

FW_METRIC = "recheck Forward GCUPS (float, null2 on; cells = peptide length x profile length) at 1 B200"


def forward_workload(args, seed):
    from protlocus_b200 import hmm as H
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    if O.rc_lib() is None:
        raise RuntimeError("--workload forward builds its profiles with recheck.c's reader (oracle/_ref/librecheck_ref.so)")
    texts, probs = H.synthetic_profiles(200, seed=seed, m_min=50, m_max=800)
    handle, profs = O.rc_load("".join(texts))
    rng = np.random.default_rng(seed + 7)
    pid = rng.integers(0, len(profs), size=args.peptides).astype(np.int32)
    lens = rng.integers(50, 601, size=args.peptides).astype(np.int32)
    dsq = rng.integers(0, 20, size=int(lens.sum())).astype(np.uint8)
    off = np.zeros(args.peptides, dtype=np.int64)
    off[1:] = np.cumsum(lens[:-1])
    desc = (f"recheck Forward: {args.peptides} peptides of 50-600 residues, each against one of 200 synthetic "
            "Plan7 profiles (m 50-800) read by recheck.c's rc_read_prof, null2 bias correction on")
    return handle, profs, pid, lens, dsq, off, desc


def main_forward(args):
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    handle, profs, pid, lens, dsq, off, desc = forward_workload(args, 11)
    threads = os.cpu_count() or 1
    cells = int((lens.astype(np.int64) * np.array([profs[k][0] for k in pid])).sum())
    if args.impl == "reference":
        k = max(threads, min(len(pid), int(args.cpu_seconds * 15 * threads)))
        bits = np.zeros(k, dtype=np.float32)
        bias = np.zeros(k, dtype=np.float32)
        secs = O.rc_lib().ref_rc_bench(threads, handle, k, pid.ctypes.data, dsq.ctypes.data, off.ctypes.data,
                                       lens.ctypes.data, 1, bits.ctypes.data, bias.ctypes.data)
        c = int((lens[:k].astype(np.int64) * np.array([profs[q][0] for q in pid[:k]])).sum())
        v = c / secs / 1e9
        print(json.dumps({"metric": FW_METRIC, "value": round(v, 4), "unit": "GCUPS", "n_gpus": 1, "steps": 1,
                          "warmup": 0, "ms_per_step": round(secs * 1e3, 2), "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                          "config": {"workload": desc}, "e2e": {"value": round(v, 4), "unit": "GCUPS",
                                                                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                          "cpu_baseline": {"value": round(v, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
                                           "sample": f"{k} peptides, recheck.c rc_score via kt_for"}}), flush=True)
        return 0
    torch.cuda.set_device(local)
    eng = L.Engine(local)
    gp = [L.RcProfile(msc, tsc, local) for _, msc, tsc in profs]
    handles = (C.c_void_p * len(gp))(*[p.h for p in gp])
    bits = np.zeros(len(pid), dtype=np.float32)
    bias = np.zeros(len(pid), dtype=np.float32)

    def step():
        if not eng.lib.pl_rc_score_host(eng.h, handles, len(gp), len(pid), pid.ctypes.data, dsq.ctypes.data, dsq.size,
                                        off.ctypes.data, lens.ctypes.data, 1, bits.ctypes.data, bias.ctypes.data):
            raise RuntimeError("pl_rc_score_host: " + L.error())

    for _ in range(max(1, args.warmup)):
        step()
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    te = (time.perf_counter() - t0) / args.steps
    launches = L.load().pl_kernel_launch_count() - launches0
    tm = eng.times()
    kern_s = tm["dp_ms"] / 1e3 / args.steps
    # reference sample on the host cores
    k = max(threads, min(len(pid), int(args.cpu_seconds * 15 * threads)))
    rb = np.zeros(k, dtype=np.float32)
    rs = np.zeros(k, dtype=np.float32)
    secs = O.rc_lib().ref_rc_bench(threads, handle, k, pid.ctypes.data, dsq.ctypes.data, off.ctypes.data,
                                   lens.ctypes.data, 1, rb.ctypes.data, rs.ctypes.data)
    err = float(np.max(np.abs(bits[:k] - rb) / np.maximum(1.0, np.abs(rb))))
    c = int((lens[:k].astype(np.int64) * np.array([profs[q][0] for q in pid[:k]])).sum())
    line = {"metric": FW_METRIC, "value": round(cells / kern_s / 1e9, 3), "unit": "GCUPS", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(kern_s * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "cells_per_step": cells, "max_rel_err_vs_reference": err},
            "e2e": {"value": round(cells / te / 1e9, 3), "unit": "GCUPS", "ms_per_step": round(te * 1e3, 2),
                    "h2d_bytes_per_step": int(dsq.nbytes + 20 * len(pid)), "d2h_bytes_per_step": int(8 * len(pid)),
                    "api": "pl_rc_score_host (C ABI, host buffers), wall clock"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "latency", "kernel": "k_rc_lanes", "achieved": None, "peak": None, "frac": None,
                         "note": "one peptide per lane; the longest peptide's chains (three dependent logsums per "
                                 "Backward cell, each a restated glibc expf + log1pf) bound the step"},
            "cpu_baseline": {"value": round(c / secs / 1e9, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
                             "sample": f"{k} peptides, recheck.c rc_score via kt_for"}}
    print(json.dumps(line), flush=True)
    for p in gp:
        p.close()
    eng.close()
    return 0


# ---------------------------------------------------------------------------- learned prefilter

PF_METRIC = "loci/sec learned-prefilter vs plain at >=99.5% locus recall (1 B200)"
PF_MODEL = os.path.join(ROOT, "protlocus_b200", "data", "prefilter.npz")


PF_N_PROT = 4096


def prefilter_measure(args, R, local, steps, warmup, cpu_seconds):
    """The learned prefilter against the plain batched DP on the held-out seed, inputs
    resident on the device.  One step of each path covers every candidate of the seed:
    the plain path runs the exact DP on every full window; the learned path computes
    features, runs the MLP, runs the exact DP on the tightened windows of the kept
    candidates and the full-window fallback.  Both then apply the reference's output test
    per protein (mp_reg_will_output: score > 0, out_sim, out_cov), and a locus -- a
    protein's planted gene -- counts as reported when a candidate on the gene passes.
    Returns the measurement as a dict (rank 0; None elsewhere)."""
    import torch
    from protlocus_b200 import prefilter as P
    rank, world = R.rank, R.world
    seed = R.seed(65)
    cand = P.make_candidates(seed, PF_N_PROT)
    n = len(cand["jobs"])
    n_all = R.sum(n)
    loci_all = R.sum(PF_N_PROT)
    jobs = cand["jobs"]
    cells_plain = int(((jobs["nl"].astype(np.int64) - 2) * jobs["al"]).sum())
    eng = L.Engine(local)
    model, meta = P.load_model(PF_MODEL, local)
    tau, margin, tau_fb = float(meta["tau"]), int(meta["margin"]), float(meta["tau_fb"])
    pipe = P.Pipeline(eng, cand)
    if not args.no_autotune:
        pipe.autotune_paths(model, tau, margin, tau_fb)
    plain, _ = pipe.plain()
    for _ in range(max(3, warmup)):
        pipe.learned(model, tau, margin, 0.0, tau_fb)
    clocks = Clocks(local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(steps):
        passed, st = pipe.learned(model, tau, margin, 0.0, tau_fb)
    torch.cuda.synchronize()
    t_learned = (time.perf_counter() - t0) / steps
    R.barrier()
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    tm = eng.times()
    t_learned = R.max(t_learned)
    m = P.path_metrics(pipe, plain, passed)
    # the plain batched DP over the same candidates, with the same output test
    R.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pipe.plain()
    torch.cuda.synchronize()
    t_plain = R.max((time.perf_counter() - t0) / steps)
    # end to end: candidate sequences from pinned host memory, pass flags back
    h_nt = torch.from_numpy(cand["nt"].copy()).pin_memory()
    h_aa = torch.from_numpy(cand["aa"].copy()).pin_memory()
    R.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pipe.d_nt.copy_(h_nt, non_blocking=True)
        pipe.d_aa.copy_(h_aa, non_blocking=True)
        pipe.learned(model, tau, margin, 0.0, tau_fb)
    torch.cuda.synchronize()
    t_e2e = R.max((time.perf_counter() - t0) / steps)
    dp_s = tm["dp_ms"] / 1e3
    int32_peak, i16x2_peak = L.measure_int_peak(local)
    peak = max(int32_peak, i16x2_peak)
    achieved = tm["cells"] * OPS_PER_CELL / dp_s if dp_s > 0 else 0.0
    out = None
    if rank == 0:
        cpu = None
        if cpu_seconds > 0:
            gcups, threads, kind, sample, _secs, _acc = cpu_baseline(
                None, cand["nt"], cand["aa"], jobs["nt_off"].copy(), jobs["aa_off"].copy(), jobs["nl"].copy(),
                jobs["al"].copy(), Options(flag=NS_F_CIGAR), cpu_seconds)
            v = gcups * 1e9 / (cells_plain / PF_N_PROT)
            cpu = {"value": round(v, 2), "unit": "loci/s", "cores": threads, "kind": kind,
                   "sample": sample + ", converted at the set's mean cells per locus (plain path on the CPU)"}
        out = {"metric": PF_METRIC, "value": round(loci_all / t_learned, 1), "unit": "loci/s", "n_gpus": world,
               "steps": steps, "warmup": max(3, warmup), "ms_per_step": round(t_learned * 1e3, 2),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16+bf16",
               "data": "synthetic",
               "config": {"workload": f"{PF_N_PROT} loci of held-out seed {seed}: per protein 8 chained candidates "
                                      "(own window both strands, a partial window, 5 windows of other genes), "
                                      f"{n} candidates, windows 1-50 kb",
                          "model": f"4-layer BF16 MLP {model.hidden} wide, trained on "
                                   f"{int(meta['train_rows'])} plain-path outcomes of seeds {meta['train_seeds']}, "
                                   f"calibrated on seed {int(meta['val_seed'])}",
                          "output_test": "mp_reg_will_output per protein: score > 0, >= 0.99 x best, "
                                         "aligned query span >= 0.1 x length, first 1000",
                          "tau": tau, "margin_nt": margin, "tau_fallback": tau_fb,
                          "tuning_plain": pipe.tune_plain, "tuning_learned": pipe.tune_learned,
                          "l2": "the candidate sequences (205 MB) and the DP trace arena exceed L2"},
               "plain": {"value": round(loci_all / t_plain, 1), "unit": "loci/s",
                         "ms_per_step": round(t_plain * 1e3, 2), "cells_per_step": cells_plain},
               "speedup_vs_plain": round(t_plain / t_learned, 2),
               "locus_recall": round(m["locus_recall"], 5), "plain_loci": m["plain_loci"],
               "learned_loci": m["learned_loci"], "extra_loci": m["extra_loci"],
               "candidates_per_s": round(n_all / t_learned, 1), "output_recall": round(m["out_recall"], 5),
               "plain_outputs": m["plain_out"], "extra_outputs": m["extra_out"],
               "kept": st["kept"], "fallback": st["fallback"], "cells_tight_per_step": st["cells_tight"],
               "phase_s": {"features_mlp": round(st["s_score"], 4), "dp_tight": round(st["s_dp"], 4),
                           "dp_fallback": round(st["s_fallback"], 4), "output_test": round(st["s_output"], 4)},
               "e2e": {"value": round(loci_all / t_e2e, 1), "unit": "loci/s", "ms_per_step": round(t_e2e * 1e3, 2),
                       "h2d_bytes_per_step": int(cand["nt"].nbytes + cand["aa"].nbytes + jobs.nbytes),
                       "d2h_bytes_per_step": int(n * 16 * 4 + n * 4 * 4), "api": "prefilter.Pipeline over the C ABI "
                       "(pl_pf_features_device, pl_pf_predict, pl_splice_batch_device), wall clock"},
               "gpu_launches": int(launches),
               "roofline": {"bound": "int", "kernel": "k_splice_dp (tightened windows)", "achieved": achieved,
                            "peak": peak, "unit": "lane-ops/s", "frac": achieved / peak if peak else None,
                            "traffic": None, "ops_per_cell": OPS_PER_CELL,
                            "peak_source": "measured live: pl_measure_int_peak"},
               "cpu_baseline": cpu, "clocks": clk}
    model.close()
    eng.close()
    return out


def main_prefilter(args):
    """--workload prefilter: the learned path's loci/s line (see prefilter_measure).  The
    reference arm times the plain spliced DP on the host cores over a bounded sample of the
    same candidates, converted to loci/s at the set's mean cells per locus."""
    from protlocus_b200 import prefilter as P
    R = Ranks("nccl")
    if args.impl == "reference":
        if R.rank == 0:
            seed = R.seed(65)
            cand = P.make_candidates(seed, PF_N_PROT)
            jobs = cand["jobs"]
            n = len(jobs)
            cells_plain = int(((jobs["nl"].astype(np.int64) - 2) * jobs["al"]).sum())
            gcups, threads, kind, sample, secs, acc = cpu_baseline(
                None, cand["nt"], cand["aa"], jobs["nt_off"].copy(), jobs["aa_off"].copy(), jobs["nl"].copy(),
                jobs["al"].copy(), Options(flag=NS_F_CIGAR), args.cpu_seconds / 2, steps=max(1, args.steps))
            v = gcups * 1e9 / (cells_plain / PF_N_PROT)
            print(json.dumps({"metric": PF_METRIC, "value": round(v, 2), "unit": "loci/s", "n_gpus": args.gpus,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(PF_N_PROT / v * 1e3, 1),
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16",
                              "data": "synthetic", "impl": "reference",
                              "config": {"workload": f"plain spliced DP over the {n} candidates of the {PF_N_PROT} "
                                                     f"loci of seed {seed}",
                                         "step": "bounded sample, converted at the set's mean cells per locus"},
                              "cpu_baseline": {"value": round(v, 2), "unit": "loci/s", "cores": threads,
                                               "kind": kind, "sample": sample},
                              "e2e": {"value": round(v, 2), "unit": "loci/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        R.close()
        return 0
    line = prefilter_measure(args, R, R.local, args.steps, args.warmup, args.cpu_seconds)
    if line is not None:
        print(json.dumps(line), flush=True)
    R.close()
    return 0


# ---------------------------------------------------------------------------- alignment statistics / features

def _simple_line(metric, value, unit, args, world, ms, dtype, desc, e2e, launches, roofline, cpu, clk, extra=None):
    line = {"metric": metric, "value": round(value, 3), "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": {"workload": desc, **(extra or {})},
            "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)


def main_extra(args):
    """One step = mp_extra_cal's counts and exon features over the alignments of the batched
    global DP (4096 pairs x 2 strands).  `value` times pl_extra_cal_device on device-resident
    CIGARs, bases and residues (CUDA events, a 256 MB buffer written between steps); `e2e`
    times pl_extra_cal_host, host buffers in and out, on the wall clock."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    from protlocus_b200.abi import BLOSUM62, ExtraResult, make_tables
    R = Ranks("nccl")
    jobs = make_jobs(args, R.seed(1))
    nt, aa, nt_off, aa_off, nl, al, tab = pack(jobs)
    n = len(jobs)
    opt = Options(flag=NS_F_CIGAR)
    eng = L.Engine(R.local)
    got = eng.align_host(opt, jobs)
    nt4, aa20, codon = make_tables()
    mat = np.asarray(BLOSUM62, np.int8).reshape(-1)
    alns = []
    for q, (score, cig, _w) in enumerate(got):
        alns.append({"cigar": cig, "nt4": nt4[nt[nt_off[q]: nt_off[q] + nl[q]]], "aa": bytes(aa[aa_off[q]: aa_off[q] + al[q]]),
                     "vs": 0, "ve": int(nl[q]), "qs": 0, "qe": int(al[q]), "has_stop": q % 4 == 0})
    pk = eng.extra_pack(alns)
    for _ in range(max(3, args.warmup)):
        eng.extra_run(pk, 11, 1, 23, mat, codon, aa20)
    d = eng.extra_upload(pk)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB): written between steps
    for _ in range(max(3, args.warmup)):
        eng.extra_run_device(pk, d, 11, 1, 23, mat, codon, aa20, stream=stream.cuda_stream)
    clocks = Clocks(R.local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.extra_run_device(pk, d, 11, 1, 23, mat, codon, aa20, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
    t = R.max(t / args.steps)
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    k_s = eng.times()["dp_ms"] / 1e3 / args.steps
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.extra_run(pk, 11, 1, 23, mat, codon, aa20)
    te = R.max((time.perf_counter() - t0) / args.steps)
    res = [(pk["res"][q], None) for q in range(n)]
    bad = sum(1 for r, _ in res if not r.ok)
    same = bytes(d["res"].cpu().numpy().tobytes())[: C.sizeof(ExtraResult) * n] == bytes(pk["res"])[: C.sizeof(ExtraResult) * n]
    n_all = R.sum(n)
    ncig = sum(len(a["cigar"]) for a in alns)
    nfeat = sum(r.n_feat for r, _ in res)
    # algorithmic bytes: the aligned codons' bases and residues, the CIGAR, the records in and out
    alg = int(sum(3 * a["qe"] + a["qe"] for a in alns) + 4 * ncig + 80 * n + 56 * nfeat)
    peak, _ = hbm_peak()
    cpu = None
    if R.is_root:
        k = min(n, 2000)
        t1 = time.perf_counter()
        for a in alns[:k]:
            O.ref_extra(a["cigar"], a["nt4"], a["aa"], a["vs"], a["ve"], a["qs"], a["qe"], a["has_stop"], 11, 1, 23, mat)
        v = k / (time.perf_counter() - t1)
        cpu = {"value": round(v, 1), "unit": "alignments/s", "cores": 1, "kind": "reference",
               "sample": f"{k} alignments, align.c mp_extra_cal (compiled from the reference) called one by one"}
        _simple_line("alignment statistics + exon features (mp_extra_cal) alignments/s at 1 B200", n_all / t,
                     "alignments/s", args, R.world, t * 1e3, "int32",
                     f"{n} global spliced alignments of the batched DP (4096 pairs x 2 strands), {ncig} CIGAR ops",
                     {"value": round(n_all / te, 1), "unit": "alignments/s", "ms_per_step": round(te * 1e3, 2),
                      "h2d_bytes_per_step": int(sum(len(a["nt4"]) + a["qe"] for a in alns) + 4 * ncig + 64 * n),
                      "d2h_bytes_per_step": int(40 * n + 56 * (ncig + 2 * n)), "api": "pl_extra_cal_host, wall clock"},
                     launches, {"bound": "hbm", "kernel": "k_extra", "achieved": alg / k_s / 1e9, "peak": peak,
                                "unit": "GB/s", "frac": alg / k_s / 1e9 / peak, "traffic": None,
                                "kernel_ms": round(k_s * 1e3, 4),
                                "note": "algorithmic bytes: 4 B per aligned residue, 4 B per CIGAR op, the records"},
                     cpu, clk, {"span_mismatches": bad, "features": nfeat, "device_equals_host_records": same,
                                "api": "pl_extra_cal_device (device-resident inputs and outputs)",
                                "l2": "a 256 MB buffer is written between timed steps"})
    eng.close()
    R.close()
    return 0


PS_OPS_PER_CELL = 11  # int32 ops per banded cell (prescreen.c:368-378): add, 2 sub + max, 3 max, 2 sub + max, max


def main_prescreen(args):
    """One step = the banded gapped alignment of 20,000 (profile, ORF, diagonal) candidates:
    PSSMs of 50-800 rows, ORFs of 100-1500 residues with a planted profile-favoured stretch on
    half of them, band 32 (the default).  `value` times pl_ps_gapped_device on device-resident
    PSSMs and ORFs (CUDA events, a 256 MB buffer written between steps); `e2e` times
    pl_ps_gapped_host, host buffers in and out, on the wall clock."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    R = Ranks("nccl")
    rng = np.random.default_rng(R.seed(9))
    n = 20000
    cands = []
    for q in range(n):
        Lq = int(rng.integers(50, 801))
        pssm = rng.integers(-9, 8, size=(Lq, 22)).astype(np.int8)
        nq = int(rng.integers(100, 1501))
        orf = rng.integers(0, 22, size=nq).astype(np.uint8)
        d0 = int(rng.integers(-Lq // 2, max(1, nq - Lq // 2)))
        if q % 2 == 0:
            rows = np.arange(Lq)
            t = rows + d0
            ok = (t >= 0) & (t < nq) & (rng.random(Lq) < 0.7)
            orf[t[ok]] = np.argmax(pssm[rows[ok]], axis=1).astype(np.uint8)
        cands.append((pssm, orf, d0 + int(rng.integers(-2, 3)), 32))
    eng = L.Engine(R.local)
    pk = eng.ps_pack(cands)
    for _ in range(max(3, args.warmup)):
        eng.ps_run(pk)
    stream = torch.cuda.current_stream()
    d_pssm = torch.from_numpy(pk["pssm"]).to("cuda")
    d_orf = torch.from_numpy(pk["orf"]).to("cuda")
    d_score = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB): written between steps
    for _ in range(max(3, args.warmup)):
        eng.ps_run_device(pk, d_pssm, d_orf, d_score, stream=stream.cuda_stream)
    clocks = Clocks(R.local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.ps_run_device(pk, d_pssm, d_orf, d_score, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t += e0.elapsed_time(e1) / 1e3
    t = R.max(t / args.steps)
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    tm = eng.times()
    k_s = tm["dp_ms"] / 1e3 / args.steps
    cells = tm["cells"] // args.steps
    cells_all = R.sum(cells)
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sc = eng.ps_run(pk)
    te = R.max((time.perf_counter() - t0) / args.steps)
    same = bool(np.array_equal(d_score.cpu().numpy()[:n], sc))
    int32_peak, _ = L.measure_int_peak(R.local)
    achieved = cells * PS_OPS_PER_CELL / k_s
    cpu = None
    if R.is_root:
        k = 400
        t1 = time.perf_counter()
        for p, o, d, b in cands[:k]:
            O.ref_ps_gapped(p, o, d, b)
        secs = time.perf_counter() - t1
        c_k = sum(min(b_hi, o.size - 1) - max(b_lo, 0) + 1 for p, o, d, b in cands[:k]
                  for b_lo, b_hi in [(i + d - 32, i + d + 32) for i in range(p.shape[0])] if min(b_hi, o.size - 1) >= max(b_lo, 0))
        cpu = {"value": round(c_k / secs / 1e9, 4), "unit": "GCUPS", "cores": 1, "kind": "reference",
               "sample": f"{k} candidates, prescreen.c ps_gapped (compiled from the reference) called one by one"}
        _simple_line("prescreen banded gapped alignment GCUPS at 1 B200", cells_all / t / 1e9, "GCUPS", args, R.world,
                     t * 1e3, "int32",
                     f"{n} profile x ORF candidates: PSSM 50-800 rows, ORF 100-1500 aa, band 32, half planted",
                     {"value": round(cells_all / te / 1e9, 3), "unit": "GCUPS", "ms_per_step": round(te * 1e3, 2),
                      "h2d_bytes_per_step": int(sum(p.size + o.size for p, o, _, _ in cands) + 24 * n),
                      "d2h_bytes_per_step": 4 * n, "api": "pl_ps_gapped_host, wall clock"},
                     launches, {"bound": "int", "kernel": "k_ps_gapped", "achieved": achieved, "peak": int32_peak,
                                "unit": "lane-ops/s", "frac": achieved / int32_peak if int32_peak else None,
                                "traffic": None, "ops_per_cell": PS_OPS_PER_CELL, "kernel_ms": round(k_s * 1e3, 4),
                                "peak_source": "measured live: pl_measure_int_peak, int32"},
                     cpu, clk, {"cells_per_step": int(cells), "positive_scores": int((sc > 0).sum()),
                                "device_equals_host_scores": same,
                                "api": "pl_ps_gapped_device (device-resident PSSMs, ORFs and scores)",
                                "l2": "a 256 MB buffer is written between timed steps"})
    eng.close()
    R.close()
    return 0


# ---------------------------------------------------------------------------- anchor chaining

CHAIN_OPS_PER_PAIR = 47  # lane-ops per scored predecessor: comput_sc (chain.c:112-152) + the update (:184-199)


SEED_BYTES_PER_ANCHOR = 12  # the anchor written (8 B) and its block id read (4 B); the index's bucket starts per seed


def seed_workload(seed: int):
    """10,000 proteins (lengths log-normal, median 350, 50-2500 aa, residues uniform over the 20) and a
    synthetic index in the mapper's layout for a 100 Mb genome: kmer 6, mod_bit 1 (2^23 buckets), bucket
    sizes Poisson(12) (six frames of 100 Mb in residues, every other k-mer kept), 256 repeat buckets of
    10,000-30,000 blocks, blocks of 256 nt (bbit 8)."""
    rng = np.random.default_rng(seed)
    n_q = 10000
    lens = np.clip(np.round(np.exp(rng.normal(np.log(350), 0.7, size=n_q))), 50, 2500).astype(np.int32)
    aa = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
    seq = aa[rng.integers(0, 20, size=int(lens.sum()))]
    prots = []
    o = 0
    for L_ in lens:
        prots.append(seq[o:o + L_].tobytes())
        o += int(L_)
    ki, kb = seed_index_100mb(rng)
    return prots, ki, kb


def seed_index_100mb(rng):
    """The synthetic 100 Mb genome index of seed_workload (ki bucket starts, kb block ids)."""
    n_bucket = 1 << 23
    cnt = rng.poisson(12.0, size=n_bucket).astype(np.int64)
    cnt[rng.choice(n_bucket, size=256, replace=False)] = rng.integers(10000, 30000, size=256)
    ki = np.zeros(n_bucket, dtype=np.int64)
    ki[1:] = np.cumsum(cnt[:-1])
    kb = rng.integers(0, (100_000_000 >> 8) * 2, size=int(cnt.sum()), dtype=np.uint32)
    return ki, kb


def seed_hmm_workload(seed: int):
    """1000 synthetic Plan7 profiles (50-800 match states, protlocus_b200.hmm.synthetic_profiles) as
    HMM-profile queries (each the consensus of its profile with its match emissions) against the index of
    seed_workload; the HMMER3 texts for the reference arm."""
    from protlocus_b200.hmm import consensus, parse_hmmer3, synthetic_profiles
    texts, _ = synthetic_profiles(1000, seed=seed, m_min=50, m_max=800)
    emits = [parse_hmmer3(t)[0]["emit"] for t in texts]
    ki, kb = seed_index_100mb(np.random.default_rng(seed + 1))
    return texts, [consensus(e) for e in emits], emits, ki, kb


def main_seed(args):
    """One step = the seeding of mp_map_coarse (map.c:565-572, default mode: mp_sketch_prot, mp_cal_max_occ
    with max_occ 20000, mp_collect_anchors, the anchor sort) for 10,000 proteins against a 100 Mb genome's
    index.  value: anchors/s of the device kernels (engine CUDA events: sketch, emission and sort, the
    batch's proteins and the index resident); e2e: pl_seed_anchors_host from host buffers (the proteins up,
    the anchors back), wall clock."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    R = Ranks("nccl")
    if args.impl == "reference" and not R.is_root:
        R.close()
        return 0
    prots, ki, kb = seed_workload(R.seed(31))
    max_occ = 20000
    desc = ("mp_map_coarse seeding (sketch kmer 6 mod_bit 1, occurrence cap, anchors, sort) of 10,000 synthetic "
            "proteins (log-normal median 350 aa) against a synthetic 100 Mb genome index (2^23 buckets, "
            "Poisson(12) blocks each, 256 repeat buckets)")
    metric = "seeding anchors/s (mp_map_coarse sketch + anchors, bit-exact) at 1 B200"
    threads = os.cpu_count() or 1

    def cpu_sample(seconds):
        from concurrent.futures import ThreadPoolExecutor
        lib = O.seed_ref_lib()
        if lib is None:
            return None
        k = 0
        n_anc = 0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            while time.perf_counter() - t0 < seconds and k < len(prots):
                chunk = prots[k:k + 4 * threads]
                res = list(ex.map(lambda p: O.seed_anchors(ki, kb, 6, 1, max_occ, p, use_ref=True).size, chunk))
                n_anc += sum(res)
                k += len(chunk)
        secs = time.perf_counter() - t0
        return n_anc / secs, k, secs

    if args.impl == "reference":
        r = cpu_sample(max(2.0, args.cpu_seconds))
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libseed_ref.so not built"}), flush=True)
        else:
            v, k, secs = r
            print(json.dumps({"metric": metric, "value": round(v, 1), "unit": "anchors/s", "n_gpus": args.gpus,
                              "steps": 1, "warmup": 0, "ms_per_step": round(secs * 1e3, 2), "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
                              "impl": "reference", "config": {"workload": desc},
                              "cpu_baseline": {"value": round(v, 1), "unit": "anchors/s", "cores": threads,
                                               "kind": "reference", "sample": f"{k} of 10000 proteins, map.c's seeding "
                                               "steps per protein over a thread pool"},
                              "e2e": {"value": round(v, 1), "unit": "anchors/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        R.close()
        return 0
    eng = L.Engine(R.local)
    idx = L.SeedIndex(ki, kb, 6, 1, R.local)
    n = len(prots)
    lens = np.array([len(p) for p in prots], dtype=np.int32)
    offs = np.zeros(n, dtype=np.int64)
    offs[1:] = np.cumsum(lens[:-1])
    seq = np.frombuffer(b"".join(prots), dtype=np.uint8).copy()
    a_off = np.zeros(n + 1, dtype=np.int64)
    tot = eng.lib.pl_seed_anchors_host(eng.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data, lens.ctypes.data,
                                       max_occ, a_off.ctypes.data, None, 0)
    if tot < 0:
        raise RuntimeError("pl_seed_anchors_host: " + L.error())
    a = np.zeros(max(int(tot), 1), dtype=np.uint64)

    def step():
        r = eng.lib.pl_seed_anchors_host(eng.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                         lens.ctypes.data, max_occ, a_off.ctypes.data, a.ctypes.data, a.size)
        if r != tot:
            raise RuntimeError("pl_seed_anchors_host: " + L.error())

    for _ in range(max(3, args.warmup)):
        step()
    # parity on a sample: the reference's own steps (or the port) per protein
    for q in range(0, n, 997):
        want = O.seed_anchors(ki, kb, 6, 1, max_occ, prots[q])
        if not np.array_equal(a[a_off[q]:a_off[q + 1]], want):
            raise RuntimeError(f"seeding parity: protein {q}")
    clocks = Clocks(R.local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    te = R.max((time.perf_counter() - t0) / args.steps)
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    tm = eng.times()
    k_s = R.max(tm["dp_ms"] / 1e3 / args.steps)
    value = R.sum(int(tot)) / k_s
    r = cpu_sample(args.cpu_seconds / 2) if R.is_root else None
    hbm = hbm_peak()
    if R.is_root:
        line = {"metric": metric, "value": round(value, 1), "unit": "anchors/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(k_s * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
                "config": {"workload": desc, "anchors_per_step": int(tot), "proteins": n,
                           "l2": "the index (464 MB) and the anchors (about 200 MB) exceed L2"},
                "e2e": {"value": round(R.sum(int(tot)) / te, 1), "unit": "anchors/s", "ms_per_step": round(te * 1e3, 3),
                        "h2d_bytes_per_step": int(seq.nbytes + offs.nbytes + lens.nbytes + a_off.nbytes),
                        "d2h_bytes_per_step": int(tot) * 8 + n * 8,
                        "api": "pl_seed_anchors_host (C ABI, host buffers), wall clock"},
                "gpu_launches": int(launches),
                "roofline": {"bound": "hbm", "kernel": "k_seed_emit + segmented sort",
                             "achieved": round(int(tot) * SEED_BYTES_PER_ANCHOR / k_s / 1e9, 2), "unit": "GB/s",
                             "peak": hbm[0], "frac": round(int(tot) * SEED_BYTES_PER_ANCHOR / k_s / 1e9 / hbm[0], 4),
                             "peak_source": hbm[1], "traffic": None,
                             "note": "algorithmic bytes: the anchor written and its block id read; the sort's passes "
                                     "and the per-protein sketch are on top"},
                "clocks": clk}
        if r is not None:
            line["cpu_baseline"] = {"value": round(r[0], 1), "unit": "anchors/s", "cores": threads, "kind": "reference",
                                    "sample": f"{r[1]} of {n} proteins, map.c's seeding steps per protein over a "
                                              "thread pool"}
        print(json.dumps(line), flush=True)
    idx.close()
    eng.close()
    R.close()
    return 0


def main_seed_hmm(args):
    """One step = the seeding of 1000 HMM-profile queries (mp_map_hmm_file's query, the consensus, with
    mp_sketch_query's profile-derived seeds at the defaults hmm_seed_pos_loss 6, hmm_seed_win_loss 8,
    hmm_seed_max 16; then mp_cal_max_occ with max_occ 20000, mp_collect_anchors, the anchor sort) against a
    100 Mb genome's index.  value: anchors/s of the device kernels (engine CUDA events); e2e:
    pl_seed_anchors_hmm_host from host buffers (the consensus sequences and emission tables up, the
    anchors back), wall clock."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    R = Ranks("nccl")
    if args.impl == "reference" and not R.is_root:
        R.close()
        return 0
    texts, prots, emits, ki, kb = seed_hmm_workload(R.seed(41))
    max_occ, pos_loss, win_loss, seed_max = 20000, 6, 8, 16
    desc = ("mp_map_coarse seeding of 1000 HMM-profile queries (synthetic Plan7 profiles of 50-800 match states; "
            "the consensus's seeds and the profile-derived ones, pos_loss 6, win_loss 8, 16 per window; kmer 6 "
            "mod_bit 1, occurrence cap, anchors, sort) against a synthetic 100 Mb genome index (2^23 buckets, "
            "Poisson(12) blocks each, 256 repeat buckets)")
    metric = "HMM-profile query seeding anchors/s (mp_sketch_query with a profile + anchors, bit-exact) at 1 B200"
    threads = os.cpu_count() or 1

    def cpu_sample(seconds):
        from concurrent.futures import ThreadPoolExecutor
        lib = O.seed_ref_lib()
        if lib is None:
            return None
        lib.ref_hmm_load.argtypes, lib.ref_hmm_load.restype = [C.c_char_p], C.c_void_p
        lib.ref_hmm_free.argtypes = [C.c_void_p]
        f = lib.ref_seed_hmm_run
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                      C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
        f.restype = C.c_int64
        with tempfile.TemporaryDirectory() as tmp:  # the reference's parser reads files
            hs = []
            for q, t in enumerate(texts):
                path = os.path.join(tmp, f"p{q}.hmm")
                with open(path, "w") as fh:
                    fh.write(t)
                hs.append(lib.ref_hmm_load(path.encode()))

        def one(h):
            out = C.POINTER(C.c_uint64)()
            m = f(h, ki.ctypes.data, kb.ctypes.data, kb.size, 6, 1, max_occ, pos_loss, win_loss, seed_max,
                  C.byref(out))
            lib.ref_seed_free(out)
            return m
        k, n_anc = 0, 0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            while time.perf_counter() - t0 < seconds and k < len(hs):
                chunk = hs[k:k + 4 * threads]
                n_anc += sum(ex.map(one, chunk))
                k += len(chunk)
        secs = time.perf_counter() - t0
        for h in hs:
            lib.ref_hmm_free(h)
        return n_anc / secs, k, secs

    if args.impl == "reference":
        r = cpu_sample(max(2.0, args.cpu_seconds))
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libseed_ref.so not built"}), flush=True)
        else:
            v, k, secs = r
            print(json.dumps({"metric": metric, "value": round(v, 1), "unit": "anchors/s", "n_gpus": args.gpus,
                              "steps": 1, "warmup": 0, "ms_per_step": round(secs * 1e3, 2), "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
                              "impl": "reference", "config": {"workload": desc},
                              "cpu_baseline": {"value": round(v, 1), "unit": "anchors/s", "cores": threads,
                                               "kind": "reference", "sample": f"{k} of 1000 profiles, the reference's "
                                               "seeding steps per parsed profile over a thread pool"},
                              "e2e": {"value": round(v, 1), "unit": "anchors/s", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        R.close()
        return 0
    eng = L.Engine(R.local)
    idx = L.SeedIndex(ki, kb, 6, 1, R.local)
    n = len(prots)
    lens = np.array([len(p) for p in prots], dtype=np.int32)
    offs = np.zeros(n, dtype=np.int64)
    offs[1:] = np.cumsum(lens[:-1])
    seq = np.frombuffer(b"".join(prots), dtype=np.uint8).copy()
    e_len = np.array([e.shape[0] for e in emits], dtype=np.int32)
    e_off = np.zeros(n, dtype=np.int64)
    e_off[1:] = np.cumsum(e_len[:-1])
    emit = np.ascontiguousarray(np.concatenate(emits).astype(np.int16))
    hmm = L.SeedHmm(emit.ctypes.data, int(e_len.sum()), e_off.ctypes.data, e_len.ctypes.data, pos_loss, win_loss,
                    seed_max, 0)
    opt = L.SeedOpt(max_occ, 0, 0, None)
    a_off = np.zeros(n + 1, dtype=np.int64)
    tot = eng.lib.pl_seed_anchors_hmm_host(eng.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                           lens.ctypes.data, C.byref(opt), C.byref(hmm), a_off.ctypes.data, None, 0)
    if tot < 0:
        raise RuntimeError("pl_seed_anchors_hmm_host: " + L.error())
    a = np.zeros(max(int(tot), 1), dtype=np.uint64)

    def step():
        r = eng.lib.pl_seed_anchors_hmm_host(eng.h, idx.h, n, seq.ctypes.data, seq.size, offs.ctypes.data,
                                             lens.ctypes.data, C.byref(opt), C.byref(hmm), a_off.ctypes.data,
                                             a.ctypes.data, a.size)
        if r != tot:
            raise RuntimeError("pl_seed_anchors_hmm_host: " + L.error())

    for _ in range(max(3, args.warmup)):
        step()
    for q in range(0, n, 97):  # parity on a sample: the restatement, pinned to the reference
        want = O.anchors_hmm(ki, kb, 6, 1, max_occ, prots[q], emits[q], pos_loss, win_loss, seed_max)
        if not np.array_equal(a[a_off[q]:a_off[q + 1]], want):
            raise RuntimeError(f"HMM seeding parity: profile {q}")
    clocks = Clocks(R.local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    te = R.max((time.perf_counter() - t0) / args.steps)
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    k_s = R.max(eng.times()["dp_ms"] / 1e3 / args.steps)
    r = cpu_sample(args.cpu_seconds / 2) if R.is_root else None
    hbm = hbm_peak()
    if R.is_root:
        line = {"metric": metric, "value": round(R.sum(int(tot)) / k_s, 1), "unit": "anchors/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(k_s * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint64", "data": "synthetic",
                "config": {"workload": desc, "anchors_per_step": int(tot), "profiles": n,
                           "l2": "the index (464 MB) exceeds L2"},
                "e2e": {"value": round(R.sum(int(tot)) / te, 1), "unit": "anchors/s", "ms_per_step": round(te * 1e3, 3),
                        "h2d_bytes_per_step": int(seq.nbytes + offs.nbytes + lens.nbytes + emit.nbytes + e_off.nbytes
                                                  + e_len.nbytes + (n + 1) * 8 + a_off.nbytes),
                        "d2h_bytes_per_step": int(tot) * 8 + n * 8,
                        "api": "pl_seed_anchors_hmm_host (C ABI, host buffers), wall clock"},
                "gpu_launches": int(launches),
                "roofline": {"bound": "hbm", "kernel": "k_seed_emit + segmented sorts",
                             "achieved": round(int(tot) * SEED_BYTES_PER_ANCHOR / k_s / 1e9, 2), "unit": "GB/s",
                             "peak": hbm[0], "frac": round(int(tot) * SEED_BYTES_PER_ANCHOR / k_s / 1e9 / hbm[0], 4),
                             "peak_source": hbm[1], "traffic": None,
                             "note": "algorithmic bytes: the anchor written and its block id read; the profile "
                                     "windows' walk, the seeds' sort and deduplication are on top"},
                "clocks": clk}
        if r is not None:
            line["cpu_baseline"] = {"value": round(r[0], 1), "unit": "anchors/s", "cores": threads, "kind": "reference",
                                    "sample": f"{r[1]} of {n} profiles, the reference's seeding steps per parsed "
                                              "profile over a thread pool"}
        print(json.dumps(line), flush=True)
    idx.close()
    eng.close()
    R.close()
    return 0


def main_chain(args):
    """One step = mp_chain (main-chain arguments of mp_map_coarse, map.c:630: bw = max intron
    36000 for a 100 Mb genome, max_gap 1000, max_skip 25, kmer 6, bbit 8) over the seed anchors
    of 10,000 synthetic query proteins, about 2^20 anchors.  value: the chaining DP on the device
    with the anchors resident (pl_chain_fill_device, CUDA events); e2e: pl_chain_host with host
    buffers (upload, DP, f and p back, backtrack and compaction on the host cores), wall clock."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    from protlocus_b200.abi import chain_opt, chain_opt_struct
    R = Ranks("nccl")
    if args.impl == "reference" and not R.is_root:
        R.close()
        return 0
    n_q = 10000
    qs = W.chain_anchors(n_q, seed=R.seed(21))
    off, n, a = L.chain_pack(qs)
    n_a = len(a)
    opt = chain_opt("main")
    desc = (f"mp_chain over {n_q} synthetic query proteins' seed anchors ({n_a} anchors: planted genes with "
            "Poisson(4) introns, half with a paralog, Poisson(40) random hits; 100 Mb genome, bbit 8), main-chain "
            "arguments of the coarse mapping")
    metric = "anchor chaining (mp_chain, bit-exact) anchors/s at 1 B200"
    threads = os.cpu_count() or 1
    if args.impl == "reference":
        O.ref_chain_batch(opt, off, n, a, threads)  # warm-up
        t0 = time.perf_counter()
        reps = 0
        while reps < max(1, args.steps) or time.perf_counter() - t0 < 2.0:
            O.ref_chain_batch(opt, off, n, a, threads)
            reps += 1
        v = n_a * reps / (time.perf_counter() - t0)
        print(json.dumps({"metric": metric, "value": round(v, 1), "unit": "anchors/s", "n_gpus": args.gpus,
                          "steps": reps, "warmup": 1, "ms_per_step": round(n_a / v * 1e3, 3), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "int32+fp32", "data": "synthetic",
                          "impl": "reference", "config": {"workload": desc},
                          "cpu_baseline": {"value": round(v, 1), "unit": "anchors/s", "cores": threads,
                                           "kind": "reference", "sample": "the whole batch, chain.c mp_chain per query "
                                           "over kt_for threads"},
                          "e2e": {"value": round(v, 1), "unit": "anchors/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        R.close()
        return 0
    eng = L.Engine(R.local)
    o = chain_opt_struct(opt)
    d_a = torch.from_numpy(a.view(np.int64).copy()).cuda()
    d_f, d_p, d_v = (torch.zeros(n_a, dtype=torch.int32, device="cuda") for _ in range(3))
    stream = torch.cuda.current_stream()

    def fill():
        if not eng.lib.pl_chain_fill_device(eng.h, C.byref(o), n_q, off.ctypes.data, n.ctypes.data, d_a.data_ptr(), n_a,
                                            d_f.data_ptr(), d_p.data_ptr(), d_v.data_ptr(), stream.cuda_stream):
            raise RuntimeError("pl_chain_fill_device: " + L.error())

    for _ in range(max(3, args.warmup)):
        fill()
    clocks = Clocks(R.local)
    eng.set_timing(True)
    launches0 = L.load().pl_kernel_launch_count()
    R.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        fill()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = L.load().pl_kernel_launch_count() - launches0
    t = R.max(ev0.elapsed_time(ev1) / 1e3 / args.steps)
    tm = eng.times()
    k_s = tm["dp_ms"] / 1e3 / args.steps
    pairs = int(eng.lib.pl_chain_last_pairs(eng.h))
    int32_peak, _ = L.measure_int_peak(R.local)
    achieved = pairs * CHAIN_OPS_PER_PAIR / k_s if k_s > 0 else 0.0
    # end to end: pl_chain_host from host buffers
    u = np.zeros(n_a, np.uint64)
    a_out = np.zeros(n_a, np.uint64)
    n_u = np.zeros(n_q, np.int32)
    eng.set_timing(False)
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        if not eng.lib.pl_chain_host(eng.h, C.byref(o), n_q, off.ctypes.data, n.ctypes.data, a.ctypes.data, n_a,
                                     u.ctypes.data, n_u.ctypes.data, a_out.ctypes.data):
            raise RuntimeError("pl_chain_host: " + L.error())
    te = R.max((time.perf_counter() - t0) / args.steps)
    n_all = R.sum(n_a)
    cpu = None
    if R.is_root:
        t1 = time.perf_counter()
        tot = O.ref_chain_batch(opt, off, n, a, threads)
        secs = time.perf_counter() - t1
        ours = sum(int((u[off[q]: off[q] + n_u[q]] & np.uint64(0xFFFFFFFF)).sum()) for q in range(n_q))
        cpu = {"value": round(n_a / secs, 1), "unit": "anchors/s", "cores": threads, "kind": "reference",
               "sample": "the whole batch, chain.c mp_chain per query over kt_for threads"}
        _simple_line(metric, n_all / t, "anchors/s", args, R.world, t * 1e3, "int32+fp32", desc,
                     {"value": round(n_all / te, 1), "unit": "anchors/s", "ms_per_step": round(te * 1e3, 2),
                      "h2d_bytes_per_step": int(a.nbytes + off.nbytes + n.nbytes),
                      "d2h_bytes_per_step": int(8 * n_a), "api": "pl_chain_host (device DP, host backtrack on "
                      f"{os.cpu_count()} threads), wall clock"},
                     launches, {"bound": "int", "kernel": "k_chain_fill", "achieved": achieved, "peak": int32_peak,
                                "unit": "lane-ops/s", "frac": achieved / int32_peak if int32_peak else None,
                                "traffic": None, "ops_per_pair": CHAIN_OPS_PER_PAIR, "pairs_per_step": pairs,
                                "kernel_ms_per_step": round(k_s * 1e3, 3),
                                "peak_source": "measured live: pl_measure_int_peak, int32"},
                     cpu, clk, {"anchors_per_step": n_a, "chains": int(n_u.sum()), "chained_anchors": ours,
                                "chained_anchors_reference": tot})
    eng.close()
    R.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
