"""Regenerate the golden fixtures of the spliced DP from the reference itself.

Runs the reference CPU code compiled from its own sources (oracle/_ref/
libnsref.so, built by `make -C oracle ref` where the reference tree exists)
on seeded inputs and writes tests/golden/splice_golden.json.  The fixture
pins the oracle restatement and the GPU path on machines where the
reference is absent.

Cases:
  * the reference's own known answers (test/test_dp32.c:7-87,
    test/test_gpu.c:51-124): MKQTW, W-repeat extensions, tile-boundary TGG/W
    repeats, the W:W=127 32-bit route;
  * random pairs (protein <= 60 aa, window <= 3*al+120, 1% N) with and
    without a splice-score track;
  * planted loci (mutated, frameshifted, spliced copies) up to 400 aa;
  * extension (left/right) cases with the 8-lane and 16-lane stripe widths.

Usage: python tests/golden/make_golden.py
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


def opt_spec(name: str, **kw):
    return {"name": name, **kw}


make_options = O.make_options


def main():
    if O.ref_lib() is None:
        sys.exit("oracle/_ref/libnsref.so is missing: run `make -C oracle ref` where the reference tree exists")
    avx2 = O.host_avx2()
    cases = []

    def add(group, spec, nt, aa, ss=None, fn="ns_global_gs_auto"):
        opt = make_options(spec)
        score, nt_len, aa_len, cig = O.ref_run(fn, nt, aa, opt, ss)
        cases.append({"group": group, "opt": spec, "fn": fn, "nt": nt.decode(), "aa": aa.decode(),
                      "ss": ss.hex() if ss is not None else None,
                      "score": score, "nt_len": nt_len, "aa_len": aa_len, "cigar": cig})

    # test_dp32.c:7-31 -- MKQTW, 16- and 32-bit
    add("known", opt_spec("mkqtw"), b"ATGAAAACTTGG", b"MKQTW", fn="ns_global_gs16b")
    add("known", opt_spec("mkqtw"), b"ATGAAAACTTGG", b"MKQTW", fn="ns_global_gs32b")
    # test_dp32.c:33-54 -- W-repeat extensions
    for flag in (NS_F_EXT_LEFT, NS_F_EXT_RIGHT):
        for n in (7, 19):
            add("known", opt_spec("nasw_init", flag=flag), b"TGG" * n, b"W" * n, fn="ns_global_gs16b")
    # test_dp32.c:72-87 -- 3000 W: 32-bit route
    add("known", opt_spec("nasw_init"), b"TGG" * 3000, b"W" * 3000)
    # test_gpu.c:51-89 -- tile boundaries
    for nl, al in ((3, 1), (9, 3), (12, 4), (15, 5), (18, 6), (21, 7), (24, 8), (27, 9), (45, 15), (48, 16), (51, 17)):
        add("tile", opt_spec("nasw_init"), (b"TGG" * 20)[:nl], b"W" * al, fn="ns_global_gs16b")
    # test_gpu.c:91-124 -- W:W=127, 32-bit
    add("known", opt_spec("ww127"), b"TGG" * 300, b"W" * 300, fn="ns_global_gs32b")

    rng = np.random.default_rng(20240611)
    for q in range(240):
        nt, aa = W.random_pair(rng, max_al=60)
        ss = W.random_ss(rng, len(nt)) if q % 3 == 0 else None
        add("random", opt_spec("protlocus"), nt, aa, ss)
        if q % 4 == 0:
            add("random32", opt_spec("protlocus"), nt, aa, ss, fn="ns_global_gs32b")
    for q in range(16):
        al = int(rng.integers(30, 400))
        nt, aa = W.single_locus(seed=1000 + q, al=al, window=int(rng.integers(3 * al + 60, 3 * al + 2500)),
                                n_intron=int(rng.integers(0, 4)))
        ss = W.random_ss(rng, len(nt)) if q % 2 else None
        add("planted", opt_spec("protlocus"), nt, aa, ss)
    for q in range(120):
        nt, aa = W.random_pair(rng, max_al=int(rng.integers(1, 120)))
        flag = NS_F_EXT_LEFT if q & 1 else NS_F_EXT_RIGHT
        spec = opt_spec("protlocus", flag=flag, io=20 if q % 3 == 0 else 29, end_bonus=5 if q % 4 else 0,
                        xdrop=[100, 30, 1000000][q % 3])
        ss = W.random_ss(rng, len(nt)) if q % 3 == 1 else None
        add("ext", spec, nt, aa, ss, fn="ns_global_gs16b")

    out = {"generator": "tests/golden/make_golden.py", "source": "reference CPU path (nasw-sse.c) via oracle/_ref",
           "host_avx2": avx2, "cases": cases}
    with open(os.path.join(HERE, "splice_golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {len(cases)} cases (host_avx2={avx2})")


if __name__ == "__main__":
    main()
