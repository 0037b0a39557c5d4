"""Regenerate the golden fixture of the gapless X-drop prefilter from the reference kernel.

The reference has no CPU twin of ns_gapless_xdrop_batch (nasw-cuda.cu:1151-1295):
its only implementation is the CUDA kernel.  This script runs that kernel, built
from the reference's own nasw-cuda.cu by `make -C oracle refcuda` into
oracle/_ref/libnscuda_ref.so, through its entry point ns_gpu_gapless_score_batch
(nasw-cuda.cu:1330) on seeded synthetic inputs, and writes the scores to
tests/golden/gapless_golden.json with a SHA-256 of each input array (the
inputs are regenerated from their seeds by case_inputs(), which the tests call
and check against those digests).  It needs a CUDA device (run it on
the GPU machine); the fixture then pins the C restatement (oracle/gapless_port.c)
and this repository's kernel everywhere.

Cases: genomes of 24 contigs with planted genes on both strands, true and decoy
candidates with 1-8 anchors; x-drop 40 (the reference default, options.c:123),
10 and 1000; kmer 6 and 4; block widths 256 and 64; plus edge cases appended to
the first case: an anchor with query_end < kmer-1, one past the query end, a
candidate with 0 anchors, one with 40 anchors (the kernel caps at 32), anchors
whose block runs past the contig end, and a contig region of N (code 4) bases.

Usage: python tests/golden/make_gapless_golden.py [out.json]
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from protlocus_b200 import workload as W  # noqa: E402
from protlocus_b200.abi import BLOSUM62, make_tables, set_stop_sc  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libnscuda_ref.so")
CASES = [  # (seed, genes, genome bases, candidates, xdrop, kmer, bbit)
    (1, 40, 240_000, 1500, 40, 6, 8),
    (2, 40, 240_000, 1500, 10, 6, 8),
    (3, 40, 240_000, 1500, 1000, 6, 8),
    (4, 30, 180_000, 1200, 40, 4, 6),
]


INPUTS = ("packed", "queries", "candidates", "anchors")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def case_inputs(k: int):
    """The workload of case k (edge cases included for k = 0)."""
    seed, genes, bases, ncand, xdrop, kmer, bbit = CASES[k]
    w = W.gapless_workload(genes, bases, ncand, seed=seed, n_contigs=24, al=300, kmer=kmer, bbit=bbit)
    if k == 0:
        edge_cases(w, kmer, bbit)
    return w


def edge_cases(w, kmer, bbit):
    """Append the edge-case candidates and the N run described above to workload w (in place)."""
    cand, anc = list(w["candidates"]), list(w["anchors"])
    lens, offs = w["contig_lengths"], w["contig_offsets"]
    packed = w["packed"].copy()
    n0 = int(offs[3]) + 1000  # a run of N inside contig 3
    for p in range(n0, n0 + 600):
        packed[p >> 1] = (packed[p >> 1] & (0xF0 if (p & 1) == 0 else 0x0F)) | (4 << (4 * (p & 1)))
    w["packed"] = packed
    qlen = int(w["candidates"][0]["query_length"])
    bw = 1 << bbit

    def add(ctg, rev, anchors):
        cand.append((int(offs[ctg]), int(lens[ctg]), 0, qlen, len(anc), len(anchors), rev))
        anc.extend(anchors)

    add(0, 0, [(0, kmer - 2, 0), (bw, kmer - 1, 0)])                           # query_end below kmer-1, then at it
    add(1, 1, [(bw, qlen, 0), (2 * bw, qlen - 1, 0)])                          # past the query end, then the last residue
    add(2, 0, [])                                                              # no anchor
    add(3, 0, [(1000 - 64 + (i % 4) * bw, 10 + i, 0) for i in range(40)])      # 40 anchors, over the N run
    add(4, 1, [(int(lens[4]) - 100, 50, 0), (int(lens[4]) + 10, 60, 0)])       # blocks past the contig end
    w["candidates"] = np.array(cand, dtype=W.GAPLESS_CAND_DTYPE)
    w["anchors"] = np.array(anc, dtype=W.GAPLESS_ANCHOR_DTYPE)


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "gapless_golden.json")
    lib = C.CDLL(LIB)
    if not lib.ns_gpu_init(0):
        lib.ns_gpu_error.restype = C.c_char_p
        sys.exit("reference ns_gpu_init failed: " + lib.ns_gpu_error().decode())
    lib.ns_gpu_gapless_score_batch.restype = C.c_int
    lib.ns_gpu_gapless_score_batch.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32,
                                               C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                               C.c_int32, C.c_void_p, C.c_void_p]
    _, _, codon = make_tables()
    mat = np.ascontiguousarray(set_stop_sc(BLOSUM62, 23), dtype=np.int8)  # ProtLocus mapping matrix, fs = 23
    cases = []
    for k, (seed, genes, bases, ncand, xdrop, kmer, bbit) in enumerate(CASES):
        w = case_inputs(k)
        cand, anc = w["candidates"], w["anchors"]
        scores = np.zeros(len(cand), dtype=np.int32)
        lib.ns_gpu_gapless_reset_target()
        ok = lib.ns_gpu_gapless_score_batch(w["packed"].ctypes.data, w["bases"], w["queries"].ctypes.data,
                                            w["queries"].size, cand.ctypes.data, len(cand), anc.ctypes.data, len(anc),
                                            1 << bbit, kmer, xdrop, mat.ctypes.data, 22, codon.ctypes.data,
                                            scores.ctypes.data)
        if not ok:
            sys.exit(f"reference ns_gpu_gapless_score_batch failed on case {k}")
        cases.append({"seed": seed, "genes": genes, "bases": int(w["bases"]), "xdrop": xdrop, "kmer": kmer,
                      "block_width": 1 << bbit, "sha256": {n: digest(w[n]) for n in INPUTS},
                      "scores": scores.tolist()})
        print(f"case {k}: {len(cand)} candidates, {len(anc)} anchors, {int((scores != -2**31).sum())} scored")
    with open(out, "w") as f:
        json.dump({"generator": "tests/golden/make_gapless_golden.py",
                   "source": "the reference's CUDA kernel ns_gapless_xdrop_batch (nasw-cuda.cu) via oracle/_ref/libnscuda_ref.so",
                   "matrix": "BLOSUM62 with stop row/column -23 (ns_set_stop_sc, fs 23)", "codon": "standard code 1",
                   "cases": cases}, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
