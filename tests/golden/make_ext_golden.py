"""Regenerate the golden fixtures of the extension DP from the reference itself.

Runs ns_global_gs16b of the reference CPU code, compiled from its own sources
by `make -C oracle ref` into oracle/_ref/: libnsref.so (AVX2 dispatch: 16-lane
stripes for al >= 16 on an AVX2 host) and libnsref8.so (the reference's
no_avx2 build: 8-lane stripes).  Writes tests/golden/ext_golden.json, which
pins the oracle restatement and the GPU extension path where the reference is
absent.

Cases (each at both stripe widths):
  * test_dp32.c:33-54 W-repeat extensions, left and right;
  * random pairs, left/right, with and without a splice-score track, with
    x-drop 100 / 30 / off, intron open 29 / 20, end bonus 5 / 0 / -3;
  * position-specific scores (ns_opt_t.pssm, nasw-sse.c:217-221);
  * planted loci extended past the gene (long windows: several 256-row strips,
    x-drop stops early);
  * saturating scores (W:W = 127 matrix, al = 300): int16 upper clamp;
  * requests without an extension flag (plain global score, no CIGAR);
  * nl < 3 (no DP row).

Usage: python tests/golden/make_ext_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from protlocus_b200 import workload as W  # noqa: E402
from protlocus_b200.abi import NS_F_EXT_LEFT, NS_F_EXT_RIGHT  # noqa: E402
import oracle_lib as O  # noqa: E402


def main():
    if O.ref_lib() is None or O.ref8_lib() is None:
        sys.exit("oracle/_ref/libnsref.so or libnsref8.so is missing: run `make -C oracle ref` where the reference tree exists")
    cases = []

    def add(group, spec, nt, aa, ss=None):
        for w8 in (False, True):
            opt = O.make_ext_options(spec)
            score, nt_len, aa_len, _ = O.ref_run("ns_global_gs16b", nt, aa, opt, ss, width8=w8)
            width = 8 if w8 else (16 if (O.host_avx2() and len(aa) >= 16 and spec.get("flag", 0) & 6) else 8)
            cases.append({"group": group, "opt": spec, "width": width, "nt": nt.decode(), "aa": aa.decode(),
                          "ss": ss.hex() if ss is not None else None,
                          "score": score, "nt_len": nt_len, "aa_len": aa_len})

    for flag in (NS_F_EXT_LEFT, NS_F_EXT_RIGHT):  # test_dp32.c:33-54
        for n in (7, 19, 40):
            add("known", {"name": "nasw_init", "flag": flag}, b"TGG" * n, b"W" * n)

    rng = np.random.default_rng(20241203)
    for q in range(160):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 140)))
        flag = NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT
        spec = {"name": "protlocus", "flag": flag, "io": 20 if q % 3 == 0 else 29,
                "end_bonus": [5, 0, -3][q % 3], "xdrop": [100, 30, 1000000][(q // 2) % 3]}
        ss = W.random_ss(rng, len(nt)) if q % 4 == 1 else None
        add("random", spec, nt, aa, ss)
    for q in range(40):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 120)))
        spec = {"name": "protlocus", "flag": NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT,
                "xdrop": [100, 1000000][q % 2], "pssm_seed": 500 + q, "al": len(aa)}
        ss = W.random_ss(rng, len(nt)) if q % 3 == 0 else None
        add("pssm", spec, nt, aa, ss)
    for q in range(16):  # gene at the start of a long window: the x-drop ends the DP after a few strips
        al = int(rng.integers(40, 300))
        nt, aa = W.single_locus(seed=7000 + q, al=al, window=int(rng.integers(3 * al + 200, 3 * al + 3000)),
                                n_intron=int(rng.integers(0, 3)))
        spec = {"name": "protlocus", "flag": NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT,
                "xdrop": [100, 30, 1000000][q % 3]}
        add("planted", spec, nt, aa)
    for flag in (NS_F_EXT_LEFT, NS_F_EXT_RIGHT):  # saturation at +32767
        add("saturate", {"name": "ww127", "flag": flag}, b"TGG" * 300, b"W" * 300)
    for q in range(12):  # no extension flag: plain global score
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 100)))
        add("global", {"name": "protlocus", "flag": 0}, nt, aa)
    for nl in (0, 1, 2):
        for al, eb in ((1, 5), (7, 5), (7, 0)):
            add("norow", {"name": "protlocus", "flag": NS_F_EXT_RIGHT, "end_bonus": eb}, b"ACG"[:nl], b"MKVLAWQ"[:al])

    out = {"generator": "tests/golden/make_ext_golden.py",
           "source": "reference CPU path (nasw-sse.c ns_global_gs16b) via oracle/_ref/libnsref.so and libnsref8.so",
           "host_avx2": O.host_avx2(), "cases": cases}
    with open(os.path.join(HERE, "ext_golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
