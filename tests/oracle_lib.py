"""Test-side access to the oracle (test infrastructure only).

Two CPU implementations of the reference algorithm are loaded through ctypes:
  * ``ref``  -- the reference's own CPU code (nasw-sse.c, nasw-tab.c, kalloc.c,
    hmm.c) compiled from its sources by oracle/Makefile into oracle/_ref/;
  * ``port`` -- this repository's C restatement (oracle/ns_port.c etc.) built
    into oracle/_build/.
Both are checkers only; the product path never loads them.
"""
from __future__ import annotations

import ctypes as C
import os
import platform
import subprocess

import numpy as np

from protlocus_b200.abi import AA_I2C, BLOSUM62, NS_F_CIGAR, NS_S_NONE, NsOpt, NsRst, Options

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
REF_SO = os.path.join(ORACLE, "_ref", "libnsref.so")
REF8_SO = os.path.join(ORACLE, "_ref", "libnsref8.so")  # built with the reference's no-AVX2 switch
PORT_SO = os.path.join(ORACLE, "_build", "libnsport.so")

_ref = None
_port = None
_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def build_port():
    if not os.path.exists(PORT_SO):
        subprocess.run(["make", "-C", ORACLE, "port"], check=True, capture_output=True)


def _load_ref(path):
    lib = C.CDLL(path)
    if lib.ns_make_tables(1) != 0:
        raise RuntimeError("reference ns_make_tables(1) failed")
    for fn in ("ns_global_gs16b", "ns_global_gs32b", "ns_global_gs_auto"):
        f = getattr(lib, fn)
        f.argtypes = [C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt),
                      C.c_void_p, C.POINTER(NsRst)]
        f.restype = None
    lib.ns_ext_stripe_width.argtypes = [C.POINTER(NsOpt), C.c_int32]
    lib.ns_ext_stripe_width.restype = C.c_int32
    return lib


def ref_lib():
    """The compiled reference, or None when oracle/_ref was not built on this machine."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = _load_ref(REF_SO)
    return _ref


_ref8 = None


def ref8_lib():
    """The reference compiled without AVX2 dispatch (8-lane ext stripes), or None."""
    global _ref8
    if _ref8 is None and os.path.exists(REF8_SO):
        _ref8 = _load_ref(REF8_SO)
    return _ref8


def port_lib():
    global _port
    if _port is None:
        build_port()
        lib = C.CDLL(PORT_SO)
        lib.port_global_gs16b.argtypes = [C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt),
                                          C.c_void_p, C.POINTER(NsRst), C.c_int32]
        lib.port_global_gs32b.argtypes = [C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt),
                                          C.c_void_p, C.POINTER(NsRst)]
        lib.port_global_gs_auto.argtypes = lib.port_global_gs16b.argtypes
        lib.port_needs_wide.argtypes = [C.POINTER(NsOpt), C.c_int32]
        lib.port_needs_wide.restype = C.c_int32
        _port = lib
    return _port


def host_avx2() -> bool:
    """Whether the reference CPU kernel dispatches ext DPs to AVX2 on this host."""
    if platform.machine() not in ("x86_64", "AMD64"):
        return False
    try:
        with open("/proc/cpuinfo") as f:
            return " avx2" in f.read()
    except OSError:
        return False


def _take(r: NsRst):
    cig = [r.cigar[k] for k in range(r.n_cigar)] if r.n_cigar else []
    if r.cigar:
        _libc.free(C.cast(r.cigar, C.c_void_p))
    return (r.score, r.nt_len, r.aa_len, cig)


def _buf(x):
    if x is None:
        return None
    if isinstance(x, (bytes, bytearray)):
        return C.c_char_p(bytes(x))
    return C.c_char_p(bytes(x))


def ref_run(fn: str, ns: bytes, aa: bytes, opt, ss: bytes | None = None, width8: bool = False):
    """Run reference `fn` (ns_global_gs16b / gs32b / gs_auto); returns (score, nt_len, aa_len, cigar).
    width8 selects the build without AVX2 dispatch (8-lane ext stripes)."""
    lib = ref8_lib() if width8 else ref_lib()
    r = NsRst()
    ssb = C.create_string_buffer(bytes(ss), len(ss)) if ss is not None else None
    getattr(lib, fn)(None, ns, len(ns), aa, len(aa), opt.ptr, ssb, C.byref(r))
    return _take(r)


def port_run(fn: str, ns: bytes, aa: bytes, opt, ss: bytes | None = None, avx2: bool | None = None):
    lib = port_lib()
    r = NsRst()
    ssb = C.create_string_buffer(bytes(ss), len(ss)) if ss is not None else None
    if avx2 is None:
        avx2 = host_avx2()
    if fn == "gs32b":
        lib.port_global_gs32b(ns, len(ns), aa, len(aa), opt.ptr, ssb, C.byref(r))
    else:
        getattr(lib, "port_global_" + fn)(ns, len(ns), aa, len(aa), opt.ptr, ssb, C.byref(r), int(avx2))
    return _take(r)


def run(fn: str, ns: bytes, aa: bytes, opt, ss: bytes | None = None):
    """The checker's answer for `fn` in {"gs16b", "gs32b", "gs_auto"}: the reference build when it
    is present on this machine, else the restatement (pinned to the same golden vectors)."""
    if ref_lib() is not None:
        return ref_run("ns_global_" + fn, ns, aa, opt, ss)
    return port_run(fn, ns, aa, opt, ss)


def make_options(spec: dict) -> Options:
    """Option sets used by the golden fixtures (tests/golden/make_golden.py)."""
    kind = spec["name"]
    flag = spec.get("flag", NS_F_CIGAR)
    if kind == "protlocus":  # ProtLocus defaults, options.c:125-138 via align.c:59-71
        return Options(flag=flag, io=spec.get("io", 29), end_bonus=spec.get("end_bonus", 5),
                       xdrop=spec.get("xdrop", 100))
    if kind == "nasw_init":  # ns_opt_init(), nasw-tab.c:131-147
        return Options.nasw_defaults(flag=flag)
    if kind == "mkqtw":      # test/test_dp32.c:15-18
        return Options.nasw_defaults(flag=flag, go=3, ge=1, io=100, fs=100, sp_model=NS_S_NONE)
    if kind == "ww127":      # test/test_gpu.c:107-112
        m = BLOSUM62.copy()
        w = AA_I2C.index("W")
        m[w, w] = 127
        return Options.nasw_defaults(flag=flag, matrix=m)
    raise ValueError(kind)


def make_ext_options(spec: dict) -> Options:
    """Option sets of the extension fixtures (tests/golden/make_ext_golden.py): make_options plus
    seeded position-specific scores (al x 22, uniform in [-6, 9]) when spec has pssm_seed."""
    import numpy as np
    o = make_options(spec)
    if spec.get("pssm_seed") is not None:
        rng = np.random.default_rng(spec["pssm_seed"])
        o = o.with_pssm(rng.integers(-6, 10, size=(spec["al"], 22)).astype(np.int8))
    return o


def port_hmm(m: int, emit, trans, codon_alpha, nt) -> int:
    """The restatement of mp_hmm_dp_score (oracle/hmm_port.c) on one region of nt4 codes."""
    import numpy as np
    lib = port_lib()
    lib.port_hmm_dp_score.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    lib.port_hmm_dp_score.restype = C.c_int32
    e = np.ascontiguousarray(emit, dtype=np.int16)
    t = np.ascontiguousarray(trans, dtype=np.int16)
    c = np.ascontiguousarray(codon_alpha, dtype=np.uint8)
    b = np.ascontiguousarray(nt, dtype=np.uint8)
    return int(lib.port_hmm_dp_score(m, e.ctypes.data, t.ctypes.data, c.ctypes.data,
                                     b.ctypes.data if b.size else None, b.size))


def port_gapless(w: dict, block_width: int, kmer: int, xdrop: int, mat, codon):
    """The restatement of the gapless prefilter (oracle/gapless_port.c) on workload dict w
    (packed, queries, candidates, anchors as from protlocus_b200.workload.gapless_workload)."""
    import numpy as np
    lib = port_lib()
    f = lib.port_gapless_score_batch
    f.argtypes = [C.c_void_p] * 3 + [C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                                     C.c_void_p, C.c_void_p]
    m = np.ascontiguousarray(mat, dtype=np.int8)
    cd = np.ascontiguousarray(codon, dtype=np.uint8)
    sc = np.zeros(len(w["candidates"]), dtype=np.int32)
    f(w["packed"].ctypes.data, w["queries"].ctypes.data, w["candidates"].ctypes.data, len(w["candidates"]),
      w["anchors"].ctypes.data, block_width, kmer, xdrop, m.ctypes.data, int(round(len(m.reshape(-1)) ** 0.5)),
      cd.ctypes.data, sc.ctypes.data)
    return sc


RECHECK_SO = os.path.join(ORACLE, "_ref", "librecheck_ref.so")
_rc = None


def rc_lib():
    """The reference's recheck.c (rc_score and its profile reader) built by oracle/Makefile, or None."""
    global _rc
    if _rc is None and os.path.exists(RECHECK_SO):
        lib = C.CDLL(RECHECK_SO)
        lib.ref_rc_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        lib.ref_rc_M.argtypes = [C.c_void_p, C.c_int]
        lib.ref_rc_msc.argtypes = lib.ref_rc_tsc.argtypes = [C.c_void_p, C.c_int]
        lib.ref_rc_msc.restype = lib.ref_rc_tsc.restype = C.POINTER(C.c_float)
        lib.ref_rc_encode.argtypes = [C.c_char_p, C.c_int32, C.c_void_p]
        lib.ref_rc_score.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int32, C.c_int, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]
        lib.ref_rc_bench.restype = C.c_double
        lib.ref_rc_bench.argtypes = [C.c_int, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int, C.c_void_p, C.c_void_p]
        _rc = lib
    return _rc


def rc_load(text: str):
    """Parse HMMER3 text with the reference's rc_read_prof: (handle, [(M, msc, tsc), ...])."""
    import tempfile
    import numpy as np
    lib = rc_lib()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(text)
        path = f.name
    h = C.c_void_p()
    n = lib.ref_rc_load(path.encode(), C.byref(h))
    os.unlink(path)
    if n < 0:
        raise RuntimeError("rc_read_prof failed")
    out = []
    for k in range(n):
        M = lib.ref_rc_M(h, k)
        msc = np.ctypeslib.as_array(lib.ref_rc_msc(h, k), shape=(M * 21,)).copy()
        tsc = np.ctypeslib.as_array(lib.ref_rc_tsc(h, k), shape=(M * 8,)).copy()
        out.append((M, msc, tsc))
    return h, out


def rc_encode(seq: bytes):
    import numpy as np
    d = np.zeros(len(seq), dtype=np.uint8)
    rc_lib().ref_rc_encode(seq, len(seq), d.ctypes.data)
    return d


def rc_ref_batch(handle, peptides, null2: bool = True, threads: int = 0):
    """rc_score of every (profile index, residue codes) pair, run by the reference's kt_for over the host's
    cores: (bits, bias) float32 arrays."""
    import numpy as np
    n = len(peptides)
    pid = np.array([p for p, _ in peptides], dtype=np.int32)
    lens = np.array([len(d) for _, d in peptides], dtype=np.int32)
    offs = np.zeros(n, dtype=np.int64)
    if n > 1:
        offs[1:] = np.cumsum(lens[:-1])
    dsq = np.ascontiguousarray(np.concatenate([np.asarray(d, dtype=np.uint8) for _, d in peptides]))
    bits, bias = np.zeros(n, dtype=np.float32), np.zeros(n, dtype=np.float32)
    rc_lib().ref_rc_bench(threads or (os.cpu_count() or 1), handle, n, pid.ctypes.data, dsq.ctypes.data,
                          offs.ctypes.data, lens.ctypes.data, int(null2), bits.ctypes.data, bias.ctypes.data)
    return bits, bias


def rc_ref_score(handle, k: int, dsq, null2: bool = True):
    import numpy as np
    b, s = C.c_float(), C.c_float()
    d = np.ascontiguousarray(dsq, dtype=np.uint8)
    rc_lib().ref_rc_score(handle, k, d.ctypes.data, d.size, int(null2), C.byref(b), C.byref(s))
    return b.value, s.value


class RefFeat(C.Structure):
    """mp_feat_t (protlocus.h:230-237)"""
    _fields_ = [("vs", C.c_int64), ("ve", C.c_int64), ("qs", C.c_int32), ("qe", C.c_int32), ("type", C.c_int16),
                ("phase", C.c_int16), ("n_fs", C.c_int32), ("n_stop", C.c_int32), ("score", C.c_int32),
                ("n_iden", C.c_int32), ("blen", C.c_int32), ("donor", C.c_char * 2), ("acceptor", C.c_char * 2)]


_extra = None


def extra_lib():
    """oracle/_ref/libextra_ref.so: the reference's own mp_extra_cal, or None where it was not built."""
    global _extra
    if _extra is None:
        path = os.path.join(ROOT, "oracle", "_ref", "libextra_ref.so")
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path)
        lib.ref_extra_cal.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_char_p, C.c_int64, C.c_int64,
                                      C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
        lib.ref_extra_cal.restype = C.c_int
        _extra = lib
    return _extra


def ref_extra(cigar, nt4, aa: bytes, vs: int, ve: int, qs: int, qe: int, has_stop: bool, go: int, ge: int, fs: int,
              mat, pssm=None):
    """(stats [blen, n_iden, n_plus, n_fs, n_stop, dp_max, n_exon, n_feat, ok], [RefFeat]) of the reference."""
    lib = extra_lib()
    cig = np.ascontiguousarray(np.asarray(cigar, dtype=np.uint32))
    nt = np.ascontiguousarray(np.asarray(nt4, dtype=np.uint8))
    m = np.ascontiguousarray(np.asarray(mat, dtype=np.int8))
    ps = None if pssm is None else np.ascontiguousarray(np.asarray(pssm, dtype=np.int8))
    stats = np.zeros(9, dtype=np.int32)
    cap = len(cig) + 4
    feats = (RefFeat * cap)()
    lib.ref_extra_cal(cig.ctypes.data, len(cig), nt.ctypes.data, len(nt), aa, vs, ve, qs, qe, int(has_stop),
                      None if ps is None else ps.ctypes.data, go, ge, fs, m.ctypes.data, stats.ctypes.data, feats, cap)
    n = int(stats[7]) if stats[8] else 0
    return stats.tolist(), [feats[k] for k in range(n)]


_ps = None


def ps_lib():
    """oracle/_ref/libps_ref.so: the reference's own ps_gapped, or None where it was not built."""
    global _ps
    if _ps is None:
        path = os.path.join(ROOT, "oracle", "_ref", "libps_ref.so")
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path)
        lib.ref_ps_gapped.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32]
        lib.ref_ps_gapped.restype = C.c_int32
        _ps = lib
    return _ps


def ref_ps_gapped(pssm, orf, diag: int, band: int, go: int = 11, ge: int = 1) -> int:
    p = np.ascontiguousarray(np.asarray(pssm, np.int8).reshape(-1, 22))
    o = np.ascontiguousarray(np.asarray(orf, np.uint8))
    return int(ps_lib().ref_ps_gapped(p.ctypes.data, p.shape[0], o.ctypes.data, o.size, diag, band, go, ge))


_chain = None


def chain_lib():
    """oracle/_ref/libchain_ref.so: the reference's own mp_chain, or None where it was not built."""
    global _chain
    if _chain is None:
        path = os.path.join(ROOT, "oracle", "_ref", "libchain_ref.so")
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path)
        lib.ref_chain.argtypes = [C.c_int32] * 7 + [C.c_float] + [C.c_int32] * 3 + [C.c_int64, C.c_void_p, C.c_void_p,
                                                                                     C.c_void_p, C.c_void_p]
        lib.ref_chain.restype = C.c_int64
        _chain = lib
    return _chain


def ref_chain(opt: dict, a):
    """(u words, chained anchors) of the reference's mp_chain over one query's sorted anchors."""
    a = np.ascontiguousarray(a, np.uint64)
    n = len(a)
    u = np.zeros(max(n, 1), np.uint64)
    out = np.zeros(max(n, 1), np.uint64)
    n_u = C.c_int32()
    tot = chain_lib().ref_chain(opt["max_dist_x"], opt["max_dist_y"], opt["bw"], opt["max_skip"], opt["max_iter"],
                                opt["min_cnt"], opt["min_sc"], opt["coef"], opt["is_spliced"], opt["kmer"], opt["bbit"],
                                n, a.ctypes.data, u.ctypes.data, C.byref(n_u), out.ctypes.data)
    return u[:n_u.value].copy(), out[:tot].copy()


def ref_chain_batch(opt: dict, off, n, a, threads: int) -> int:
    """The reference's mp_chain over a packed batch on `threads` host threads (kt_for); the
    total number of chained anchors."""
    lib = chain_lib()
    lib.ref_chain_batch.argtypes = [C.c_int32] * 7 + [C.c_float] + [C.c_int32] * 4 + [C.c_void_p] * 3 + [C.c_int32]
    lib.ref_chain_batch.restype = C.c_int64
    return int(lib.ref_chain_batch(opt["max_dist_x"], opt["max_dist_y"], opt["bw"], opt["max_skip"], opt["max_iter"],
                                   opt["min_cnt"], opt["min_sc"], opt["coef"], opt["is_spliced"], opt["kmer"],
                                   opt["bbit"], len(n), off.ctypes.data, n.ctypes.data, a.ctypes.data, threads))


# ---------------------------------------------------------------- seeding (map.c:304-397, sketch.c:18-37)

SEED_REF_SO = os.path.join(ORACLE, "_ref", "libseed_ref.so")
_seed_ref = None


def seed_ref_lib():
    """The reference's own seeding steps (map.c with oracle/seed_ref_hook.c), or None."""
    global _seed_ref
    if _seed_ref is None and os.path.exists(SEED_REF_SO):
        lib = C.CDLL(SEED_REF_SO)
        lib.ns_make_tables(1)
        lib.ref_seed_anchors.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                         C.c_char_p, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
        lib.ref_seed_anchors.restype = C.c_int64
        lib.ref_seed_free.argtypes = [C.c_void_p]
        _seed_ref = lib
    return _seed_ref


def _seed_port():
    lib = port_lib()
    if not hasattr(lib, "_seed_ready"):
        lib.sp_anchors.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_char_p, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
        lib.sp_anchors.restype = C.c_int64
        lib.sp_free.argtypes = [C.c_void_p]
        lib._seed_ready = True
    return lib


def seed_index(rng, kmer: int = 6, mod_bit: int = 1, mean_occ: float = 3.0, n_block: int = 400_000,
               hot: int = 64, hot_occ: int = 30_000):
    """A synthetic index in the reference's layout (index.c:74-98): ki[b] = first entry of bucket
    b in kb (int64), kb = block ids (uint32).  Bucket sizes are Poisson(mean_occ) with `hot`
    buckets of about hot_occ entries (repeats, which the occurrence cap drops)."""
    n_bucket = 1 << (kmer * 4 - mod_bit)
    cnt = rng.poisson(mean_occ, size=n_bucket).astype(np.int64)
    cnt[rng.choice(n_bucket, size=hot, replace=False)] = rng.integers(hot_occ // 2, hot_occ, size=hot)
    ki = np.zeros(n_bucket, dtype=np.int64)
    ki[1:] = np.cumsum(cnt[:-1])
    kb = rng.integers(0, n_block, size=int(cnt.sum()), dtype=np.uint32)
    return ki, kb


def _seed_take(fn, free, *args):
    out = C.POINTER(C.c_uint64)()
    n = fn(*args, C.byref(out))
    if n < 0:
        raise MemoryError("seeding checker out of host memory")
    a = np.ctypeslib.as_array(out, shape=(max(n, 1),))[:n].copy() if n > 0 else np.zeros(0, np.uint64)
    free(out)
    return a


def seed_anchors(ki, kb, kmer: int, mod_bit: int, max_occ: int, seq: bytes, use_ref: bool | None = None):
    """Sorted anchors (block << 32 | position, uint64) of one protein: the reference's own
    steps when oracle/_ref/libseed_ref.so is built (or use_ref), else the port."""
    lib = seed_ref_lib() if use_ref is not False else None
    if use_ref and lib is None:
        raise RuntimeError("oracle/_ref/libseed_ref.so not built")
    if lib is not None:
        return _seed_take(lib.ref_seed_anchors, lib.ref_seed_free, ki.ctypes.data, kb.ctypes.data, kb.size, kmer,
                          mod_bit, max_occ, seq, len(seq))
    p = _seed_port()
    return _seed_take(p.sp_anchors, p.sp_free, ki.ctypes.data, ki.size, kb.ctypes.data, kb.size, kmer, mod_bit,
                      max_occ, seq, len(seq))


def seed_anchors_acc(ki, kb, kmer: int, mod_bit: int, max_occ: int, repeat_cap: int, budget: int, qname: bytes,
                     seq: bytes, use_ref: bool | None = None):
    """seed_anchors with the accuracy mode's repeat rescue (map.c:360-384) for a query named qname."""
    lib = seed_ref_lib() if use_ref is not False else None
    if use_ref and lib is None:
        raise RuntimeError("oracle/_ref/libseed_ref.so not built")
    if lib is not None:
        f = lib.ref_seed_anchors_acc
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                      C.c_char_p, C.c_char_p, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
        f.restype = C.c_int64
        return _seed_take(f, lib.ref_seed_free, ki.ctypes.data, kb.ctypes.data, kb.size, kmer, mod_bit, max_occ,
                          repeat_cap, budget, qname, seq, len(seq))
    p = _seed_port()
    p.sp_qname_hash.argtypes = [C.c_char_p]
    p.sp_qname_hash.restype = C.c_uint32
    p.sp_anchors_acc.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_int32, C.c_int64, C.c_uint32, C.c_char_p, C.c_int32,
                                 C.POINTER(C.POINTER(C.c_uint64))]
    p.sp_anchors_acc.restype = C.c_int64
    return _seed_take(p.sp_anchors_acc, p.sp_free, ki.ctypes.data, ki.size, kb.ctypes.data, kb.size, kmer, mod_bit,
                      max_occ, repeat_cap, budget, p.sp_qname_hash(qname), seq, len(seq))


def seed_qname_hash(qname: bytes) -> int:
    """mp_hash_qname (map.c:322-329), from the restatement."""
    p = _seed_port()
    p.sp_qname_hash.argtypes = [C.c_char_p]
    p.sp_qname_hash.restype = C.c_uint32
    return int(p.sp_qname_hash(qname))


# ---------------------------------------------------------------- HMM-profile seeds (sketch.c:40-118, map.c:332-343)

def _i16p(a):
    return np.ascontiguousarray(a, dtype=np.int16)


def sketch_hmm(emit, kmer: int, mod_bit: int, pos_loss: int, win_loss: int, max_per_win: int,
               use_ref: bool | None = None):
    """mp_sketch_hmm's seeds of an emission table (len x 20 int16, HMMER column order) in the
    order the reference appends them (window by window); the reference's own function when
    oracle/_ref/libseed_ref.so is built (or use_ref), else the restatement."""
    e = _i16p(emit).reshape(-1, 20)
    n = e.shape[0]
    lib = seed_ref_lib() if use_ref is not False else None
    if use_ref and lib is None:
        raise RuntimeError("oracle/_ref/libseed_ref.so not built")
    if lib is not None:
        f = lib.ref_sketch_hmm
        f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                      C.POINTER(C.POINTER(C.c_uint64))]
        f.restype = C.c_int64
        return _seed_take(f, lib.ref_seed_free, e.ctypes.data, n, kmer, mod_bit, pos_loss, win_loss, max_per_win)
    p = _seed_port()
    p.sp_sketch_hmm.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                C.c_void_p]
    p.sp_sketch_hmm.restype = C.c_int64
    cap = max(n - kmer + 1, 0) * max(max_per_win, 0)
    out = np.zeros(max(cap, 1), np.uint64)
    m = p.sp_sketch_hmm(e.ctypes.data, n, kmer, mod_bit, pos_loss, win_loss, max_per_win, out.ctypes.data)
    if m < 0:
        raise MemoryError("seeding checker out of host memory")
    return out[:m].copy()


def hmm_consensus(emit) -> bytes:
    """The parser's consensus (hmm.c:181-189): per match state the first column of the
    largest emission, as its HMMER letter."""
    e = _i16p(emit).reshape(-1, 20)
    return bytes(b"ACDEFGHIKLMNPQRSTVWY"[int(j)] for j in np.argmax(e, axis=1))


def seeds_hmm_query(seq: bytes, emit, kmer: int, mod_bit: int, pos_loss: int, win_loss: int, seed_max: int):
    """mp_sketch_query with a profile (map.c:332-343), from the restatement: the sequence's
    seeds and the profile-derived ones, sorted, duplicates removed."""
    e = _i16p(emit).reshape(-1, 20)
    p = _seed_port()
    p.sp_seeds_hmm_query.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
    p.sp_seeds_hmm_query.restype = C.c_int64
    return _seed_take(p.sp_seeds_hmm_query, p.sp_free, seq, len(seq), e.ctypes.data, e.shape[0], kmer, mod_bit,
                      pos_loss, win_loss, seed_max)


def anchors_hmm(ki, kb, kmer: int, mod_bit: int, max_occ: int, seq: bytes, emit, pos_loss: int, win_loss: int,
                seed_max: int, repeat_cap: int = 0, budget: int = 0, qname: bytes = b""):
    """The anchors of an HMM-profile query (seeds_hmm_query, then the cap and the collection,
    with the repeat rescue for a query named qname when repeat_cap > 0), from the restatement."""
    e = _i16p(emit).reshape(-1, 20)
    p = _seed_port()
    p.sp_anchors_hmm.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                 C.c_int32, C.c_int64, C.c_uint32, C.c_char_p, C.c_int32, C.c_void_p, C.c_int32,
                                 C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
    p.sp_anchors_hmm.restype = C.c_int64
    return _seed_take(p.sp_anchors_hmm, p.sp_free, ki.ctypes.data, ki.size, kb.ctypes.data, kb.size, kmer, mod_bit,
                      max_occ, repeat_cap, budget, seed_qname_hash(qname), seq, len(seq), e.ctypes.data, e.shape[0],
                      pos_loss, win_loss, seed_max)


def ref_hmm_query(path: str, kmer: int, mod_bit: int, pos_loss: int, win_loss: int, seed_max: int,
                  ki=None, kb=None, max_occ: int = 20000, repeat_cap: int = 0, budget: int = 0):
    """The reference on an HMMER3 file: its parser, the consensus as the query (the profile's
    name its name), and mp_sketch_query's seeds (ki None) or mp_map_coarse's anchors (with the
    repeat rescue when repeat_cap > 0); None when oracle/_ref/libseed_ref.so is not built."""
    lib = seed_ref_lib()
    if lib is None:
        return None
    f = lib.ref_seed_hmm_query
    f.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                  C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_uint64))]
    f.restype = C.c_int64
    return _seed_take(f, lib.ref_seed_free, path.encode(), None if ki is None else ki.ctypes.data,
                      None if kb is None else kb.ctypes.data, 0 if kb is None else kb.size, kmer, mod_bit, max_occ,
                      repeat_cap, budget, pos_loss, win_loss, seed_max)


def ref_hmm_tables(path: str):
    """The reference parser's consensus and emission table of an HMMER3 file, or None."""
    lib = seed_ref_lib()
    if lib is None:
        return None
    lib.ref_hmm_consensus.argtypes = [C.c_char_p, C.c_char_p, C.c_int32]
    lib.ref_hmm_consensus.restype = C.c_int32
    lib.ref_hmm_emissions.argtypes = [C.c_char_p, C.c_void_p, C.c_int32]
    lib.ref_hmm_emissions.restype = C.c_int32
    n = lib.ref_hmm_consensus(path.encode(), None, 0)
    if n < 0:
        raise ValueError(f"{path}: the reference parser refused it")
    buf = C.create_string_buffer(n + 1)
    lib.ref_hmm_consensus(path.encode(), buf, n + 1)
    e = np.zeros((n, 20), np.int16)
    lib.ref_hmm_emissions(path.encode(), e.ctypes.data, n * 20)
    return buf.raw[:n], e


def device_seed_fns_host(emit, kmer: int, mod_bit: int, pos_loss: int, win_loss: int, max_per_win: int):
    """The device's profile-derived seeding functions (protlocus_b200/csrc/seed_hmm.cuh) built
    for the host (oracle/_build/libseedhmmcheck.so), window by window as the kernel runs them."""
    so = os.path.join(ORACLE, "_build", "libseedhmmcheck.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", ORACLE, "port"], check=True, capture_output=True)
    lib = C.CDLL(so)
    lib.shc_sketch_hmm.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_void_p]
    lib.shc_sketch_hmm.restype = C.c_int64
    e = _i16p(emit).reshape(-1, 20)
    n = e.shape[0]
    out = np.zeros(max(max(n - kmer + 1, 0) * max(max_per_win, 0), 1), np.uint64)
    m = lib.shc_sketch_hmm(e.ctypes.data, n, kmer, mod_bit, pos_loss, win_loss, max_per_win, out.ctypes.data)
    if m < 0:
        raise MemoryError("out of host memory")
    return out[:m].copy()
