"""Regenerate the golden fixtures of the integer profile-HMM DP from the reference.

Profiles are written as HMMER3 text and parsed by the reference's own parser
(mp_hmm_open / mp_hmm_read1, hmm.c:112-195, compiled into oracle/_ref/
libnsref.so by `make -C oracle ref`); regions are scored by the reference's
mp_hmm_dp_score (hmm.c:252-291).  Writes tests/golden/hmm_golden.json with the
parsed int16 tables, the regions (nt4 codes) and the scores, so that the oracle
restatement, the Python parser and the GPU path are pinned where the reference
is absent.

Profiles:
  * the two LCG profiles of the reference's GPU test (test/test_gpu.c:222-243:
    lengths 37 and 300, seeds 1 and 2), scored on its LCG nucleotide buffer and
    its five-region batch with an empty region (test_gpu.c:246-285);
  * synthetic Plan7 profiles (protlocus_b200.hmm.synthetic_profiles, seed 11,
    m in 20-700: one to three 256-column tiles) on random regions, half with a
    planted domain, plus regions with ambiguous codes and stop codons and the
    short lengths 0, 1, 2, 3, 4, 5.

Usage: python tests/golden/make_hmm_golden.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from protlocus_b200 import hmm as H  # noqa: E402
import oracle_lib as O  # noqa: E402


def lcg_profile(name: str, length: int, seed: int) -> str:
    """The HMMER3 text of test_gpu.c:222-243 (an LCG fills the match emissions)."""
    out = [f"HMMER3/f [test]\nNAME  {name}\nLENG  {length}\nALPH  amino\nHMM          A        C        D        E        F        G        H        I        K        L        M        N        P        Q        R        S        T        V        W        Y\n",
           "            m->m     m->i     m->d     i->m     i->i     d->m     d->d\n",
           "  COMPO   " + " ".join(["2.5"] * 20) + "\n", "          " + " ".join(["2.5"] * 20) + "\n",
           "          0.02 4.5 5.0 0.6 0.8 0.0 *\n"]
    for i in range(1, length + 1):
        row = []
        for _ in range(20):
            seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
            row.append(f" {0.5 + ((seed >> 16) % 4000) / 1000.0:.3f}")
        out.append(f"{i:7d}" + "".join(row) + f" {i} - - -\n")
        out.append("          " + " ".join(["2.5"] * 20) + "\n")
        out.append("          0.02 4.5 5.0 0.6 0.8 0.5 1.0\n")
    out.append("//\n")
    return "".join(out)


def lcg_nt(n: int, seed: int = 7) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint8)
    for i in range(n):
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = (seed >> 16) & 3
    return out


def main():
    ref = O.ref_lib()
    if ref is None:
        sys.exit("oracle/_ref/libnsref.so is missing: run `make -C oracle ref` where the reference tree exists")
    ref.mp_hmm_open.restype, ref.mp_hmm_open.argtypes = C.c_void_p, [C.c_char_p]
    ref.mp_hmm_read1.restype, ref.mp_hmm_read1.argtypes = C.c_void_p, [C.c_void_p]
    ref.mp_hmm_length.argtypes = [C.c_void_p]
    ref.mp_hmm_emissions.restype, ref.mp_hmm_emissions.argtypes = C.POINTER(C.c_int16), [C.c_void_p]
    ref.mp_hmm_transitions.restype, ref.mp_hmm_transitions.argtypes = C.POINTER(C.c_int16), [C.c_void_p]
    ref.mp_hmm_dp_score.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    ref.mp_hmm_destroy.argtypes = [C.c_void_p]
    ref.mp_hmm_close.argtypes = [C.c_void_p]

    texts = [lcg_profile("tiny_a", 37, 1), lcg_profile("tiny_b", 300, 2)]
    syn, probs = H.synthetic_profiles(8, seed=11, m_min=20, m_max=700)
    texts += syn
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write("".join(texts))
        path = f.name
    fh = ref.mp_hmm_open(path.encode())
    rng = np.random.default_rng(20241204)
    profiles = []
    for q in range(len(texts)):
        h = ref.mp_hmm_read1(fh)
        m = ref.mp_hmm_length(h)
        emit = np.ctypeslib.as_array(ref.mp_hmm_emissions(h), shape=(m * 20,)).copy()
        trans = np.ctypeslib.as_array(ref.mp_hmm_transitions(h), shape=(m * 7,)).copy()
        regs = []
        if q < 2:  # test_gpu.c:246-285: the 3000-nt LCG buffer, then five regions incl. an empty one
            nt = lcg_nt(3000)
            regs.append(nt)
            off = 0
            for k in range(5):
                ln = 0 if k == 3 else 3 * (61 * (k + 1) + (2 if k == 4 else 0))
                if k == 4:
                    ln += 2
                regs.append(nt[off:off + ln])
                off += ln
        else:
            regs += H.regions(rng, probs[q - 2], 14, 30, 2400)
            for ln in (0, 1, 2, 3, 4, 5):
                regs.append(rng.integers(0, 4, size=ln).astype(np.uint8))
            amb = rng.integers(0, 4, size=900).astype(np.uint8)
            amb[rng.random(900) < 0.05] = 4
            regs.append(amb)
            stops = np.tile(np.array([3, 0, 0, 3, 0, 2, 3, 2, 0], dtype=np.uint8), 60)  # TAA TAG TGA
            regs.append(stops)
        scores = [int(ref.mp_hmm_dp_score(h, r.ctypes.data if len(r) else None, len(r))) for r in regs]
        profiles.append({"source": "test_gpu.c LCG" if q < 2 else "synthetic seed 11", "m": int(m),
                         "emit": emit.tolist(), "trans": trans.tolist(),
                         "regions": [r.tobytes().hex() for r in regs], "scores": scores})
        ref.mp_hmm_destroy(h)
    ref.mp_hmm_close(fh)
    os.unlink(path)
    out = {"generator": "tests/golden/make_hmm_golden.py",
           "source": "reference hmm.c (mp_hmm_read1, mp_hmm_dp_score) via oracle/_ref/libnsref.so",
           "synthetic": {"n": 8, "seed": 11, "m_min": 20, "m_max": 700}, "profiles": profiles}
    with open(os.path.join(HERE, "hmm_golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {len(profiles)} profiles, {sum(len(p['regions']) for p in profiles)} regions")


if __name__ == "__main__":
    main()
