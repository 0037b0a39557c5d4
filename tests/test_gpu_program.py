"""The reference's whole mapping program, linked against this library, gives the
same output as its CPU build.

oracle/Makefile's `progs` target builds, from the reference's own sources where
they lie, the mapping program (main.c and every object of its default build)
three ways: protlocus_cpu (default build, the GPU entry points are
nasw-opencl.c's stubs), protlocus_plgpu (nasw-opencl.o, nasw-ext-gpu.o and
hmm-gpu.o replaced by libplgpu) and protlocus_cuda (the reference's
`make cuda=1` build, nasw-cuda.cu for sm_100a).

* `--gpu --gpu-min-cells=0` sends every spliced global DP (align.c:74-83,
  nasw-sse.c:984-986) and every terminal extension (align.c:753) through
  libplgpu: the PAF (with cs/cg tags) and GFF3 outputs must equal the CPU
  build's byte for byte, on protein and on HMM-profile queries (the profile
  path also reaches mp_hmm_dp_score_gpu_batch, hmm.c:324);
* protlocus_learned (oracle/map_learned_hook.c) runs libplgpu's learned selector at
  the mapper's candidate selection (`--gpu-prefilter` with PL_PF_MODEL set): keeping
  every candidate it must print the plain mapper's output byte for byte, and with the
  shipped model it must keep at least 99.5 % of the plain mapper's PAF lines verbatim;
* protlocus_recheck_gpu (oracle/recheck_gpu_hook.c) is the reference's recheck program
  scoring its peptides through libplgpu's Forward: its output and per-candidate table
  must equal the stock program's byte for byte;
* `--gpu-prefilter` ranks candidates with the gapless X-drop score
  (map.c:1014-1090); there is no CPU build of it, so the reference's CUDA build
  is the reference: both programs keep the DP on the CPU and must print the
  same hits, and libplgpu with `--gpu` on top must print them too.

Inputs: seeded synthetic genomes with planted spliced genes
(protlocus_b200.workload.genome_fasta).
"""
import os
import re
import subprocess

import numpy as np
import pytest

from protlocus_b200 import hmm as H
from protlocus_b200 import workload as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
CPU, PLGPU, CUDA, LEARNED = (os.path.join(REF, n) for n in ("protlocus_cpu", "protlocus_plgpu", "protlocus_cuda",
                                                            "protlocus_learned"))
RC_CPU, RC_GPU = (os.path.join(REF, n) for n in ("protlocus_recheck_cpu", "protlocus_recheck_gpu"))
need = pytest.mark.skipif(not (os.path.exists(CPU) and os.path.exists(PLGPU)),
                          reason="oracle/_ref programs not built (needs the reference tree)")
AA = "ACDEFGHIKLMNPQRSTVWY"


def run(binary, args, env=None):
    p = subprocess.run([binary, "-t8", "--profile", *args], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, **(env or {})))
    assert p.returncode == 0, p.stderr[-3000:]
    assert "GPU unavailable" not in p.stderr and "ignoring --gpu-prefilter" not in p.stderr, p.stderr[-3000:]
    prof = dict(re.findall(r"(\w+)=([0-9.]+)", p.stderr.split("[M::profile]")[-1].splitlines()[0]))
    return p.stdout, prof


@pytest.fixture(scope="module")
def protein_inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("prog")
    g, p = W.genome_fasta(96, seed=21, n_contigs=6, contig_len=400_000, al_min=60, al_max=900,
                          divergence=0.25, n_decoys=8, max_frameshift=2)
    (d / "genome.fa").write_text(g)
    (d / "prot.fa").write_text(p)
    return str(d / "genome.fa"), str(d / "prot.fa")


@pytest.fixture(scope="module")
def hmm_inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("prog_hmm")
    texts, probs = H.synthetic_profiles(16, seed=22, m_min=80, m_max=400, concentration=1.0)
    rng = np.random.default_rng(23)
    prots = ["".join(AA[rng.choice(20, p=row / row.sum())] for row in pm) for pm in probs]
    g, _ = W.genome_fasta(0, seed=24, n_contigs=4, contig_len=200_000, proteins=prots, divergence=0.08)
    (d / "genome.fa").write_text(g)
    (d / "q.hmm").write_text("".join(texts))
    return str(d / "genome.fa"), str(d / "q.hmm")


@need
@pytest.mark.parametrize("fmt", ["paf", "gff"])
def test_program_protein_queries_gpu_dp(protein_inputs, fmt):
    genome, prot = protein_inputs
    extra = ["--gff"] if fmt == "gff" else []
    want, _ = run(CPU, [*extra, genome, prot])
    got, prof = run(PLGPU, ["--gpu", "--gpu-min-cells=0", *extra, genome, prot])
    assert len(want.splitlines()) >= 80
    assert int(prof["gpu_dp"]) > 0 and int(prof["gpu_launch"]) > 0, prof
    assert got == want


@need
def test_program_hmm_queries_gpu_dp(hmm_inputs):
    genome, q = hmm_inputs
    want, _ = run(CPU, [genome, q])
    got, prof = run(PLGPU, ["--gpu", "--gpu-min-cells=0", genome, q], env={"MP_HMM_GPU": "1"})
    assert len(want.splitlines()) >= 12
    assert got == want


@need
@pytest.mark.skipif(not os.path.exists(CUDA), reason="oracle/_ref/protlocus_cuda not built")
@pytest.mark.parametrize("topk", [1, 3])
def test_program_gpu_prefilter(protein_inputs, topk):
    genome, prot = protein_inputs
    args = ["--gpu-prefilter", f"--gpu-prefilter-topk={topk}", "--gpu-prefilter-diversity=0"]
    want, prof_ref = run(CUDA, [*args, genome, prot])
    got, prof = run(PLGPU, [*args, genome, prot])
    assert int(prof["prefilter_candidate"]) > 0
    assert prof["prefilter_survivor"] == prof_ref["prefilter_survivor"]
    assert got == want
    got_dp, _ = run(PLGPU, ["--gpu", "--gpu-min-cells=0", *args, genome, prot])
    assert got_dp == want


def _model_file(path, tau=None):
    """The shipped prefilter model as the hook reads it: "hidden tau margin tau_fb n" then
    n float32 parameters."""
    z = np.load(os.path.join(ROOT, "protlocus_b200", "data", "prefilter.npz"))
    p = np.ascontiguousarray(z["params"], np.float32)
    t = float(z["tau"]) if tau is None else tau
    with open(path, "wb") as f:
        f.write(f"{int(z['hidden'])} {t!r} {int(z['margin'])} {float(z['tau_fb'])!r} {p.size}\n".encode())
        f.write(p.tobytes())


@need
@pytest.mark.skipif(not os.path.exists(LEARNED), reason="oracle/_ref/protlocus_learned not built")
def test_program_learned_selector(protein_inputs, tmp_path):
    """The reference mapper with libplgpu's learned selector in place of its candidate
    selection (map.c:1014-1089): every reported alignment is still the exact DP's, so a
    threshold that keeps every candidate prints the plain mapper's output (no prefilter,
    every coarse candidate aligned) byte for byte, and the shipped model keeps at least
    99.5 % of the plain mapper's PAF lines verbatim while dropping candidates."""
    genome, prot = protein_inputs
    want, _ = run(PLGPU, [genome, prot])
    keep_all = tmp_path / "keep_all.bin"
    _model_file(keep_all, tau=0.0)
    got_all, prof_all = run(LEARNED, ["--gpu-prefilter", genome, prot], env={"PL_PF_MODEL": str(keep_all)})
    assert int(prof_all["prefilter_candidate"]) > 0
    assert prof_all["prefilter_survivor"] == prof_all["prefilter_candidate"]
    assert got_all == want
    shipped = tmp_path / "shipped.bin"
    _model_file(shipped)
    got, prof = run(LEARNED, ["--gpu-prefilter", genome, prot], env={"PL_PF_MODEL": str(shipped)})
    lines, out = want.splitlines(), set(got.splitlines())
    kept = sum(1 for line in lines if line in out)
    print(f"learned selector: {kept} of {len(lines)} plain PAF lines kept verbatim, {len(out)} lines out; "
          f"candidates {prof['prefilter_candidate']} -> {prof['prefilter_survivor']}")
    assert len(lines) >= 80 and kept >= 0.995 * len(lines), (kept, len(lines))
    assert int(prof["prefilter_survivor"]) < int(prof["prefilter_candidate"]), prof


@pytest.fixture(scope="module")
def recheck_inputs(tmp_path_factory):
    """Candidates of an HMM-library mapping run with --trans (PAF + ##STA peptide lines) of 40
    synthetic profiles against a genome holding one planted copy of each, and the profiles
    with a STATS LOCAL FORWARD calibration on two of every three (the rest get no E-value)."""
    d = tmp_path_factory.mktemp("recheck")
    texts, probs = H.synthetic_profiles(40, seed=41, m_min=60, m_max=500, concentration=1.0)
    rng = np.random.default_rng(42)
    prots = ["".join(AA[rng.choice(20, p=row / row.sum())] for row in pm) for pm in probs]
    g, _ = W.genome_fasta(0, seed=43, n_contigs=6, contig_len=200_000, proteins=prots, divergence=0.15)
    (d / "genome.fa").write_text(g)
    (d / "q.hmm").write_text("".join(texts))
    out, k = [], 0
    for line in "".join(texts).splitlines(True):
        out.append(line)
        if line.startswith("ALPH"):
            if k % 3 != 2:
                out.append(f"STATS LOCAL FORWARD    {60 + 4 * k:.4f}  0.0{5 + k % 5}\n")
            k += 1
    (d / "q_stats.hmm").write_text("".join(out))
    p = subprocess.run([CPU, "-t8", "--trans", str(d / "genome.fa"), str(d / "q.hmm")], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    (d / "cand.paf").write_text(p.stdout)
    return str(d / "q_stats.hmm"), str(d / "cand.paf"), d


@need
@pytest.mark.skipif(not (os.path.exists(RC_CPU) and os.path.exists(RC_GPU)), reason="recheck programs not built")
@pytest.mark.parametrize("extra", [[], ["-n"], ["-e", "1e-30"]])
def test_program_recheck_gpu(recheck_inputs, extra):
    """The reference's recheck program with its Forward scoring on libplgpu prints the stock
    program's passing lines (and, with -a, the failing ones with their scores) and writes
    its per-candidate table (bits, bias, E-value, pass) byte for byte; with the null2
    correction off too, and at a threshold that fails part of the candidates."""
    hmm, cand, d = recheck_inputs
    outs = []
    for prog in (RC_CPU, RC_GPU):
        tsv = d / (os.path.basename(prog) + "".join(extra) + ".tsv")
        p = subprocess.run([prog, "-t", "8", "-a", "-T", str(tsv), *extra, hmm, cand], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        outs.append((p.stdout, tsv.read_text()))
    (want, want_tsv), (got, got_tsv) = outs
    rows = want_tsv.splitlines()[1:]
    assert len(rows) >= 30 and sum(1 for r in rows if r.split("\t")[4] != ".") >= 30, want_tsv[:500]
    assert got_tsv == want_tsv
    assert got == want
