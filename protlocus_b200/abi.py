"""ctypes mirror of the C ABI in include/plgpu.h and the scoring tables it consumes.

The structs are layout-identical to the reference's nasw.h:62-82 (ns_opt_t,
ns_rst_t) and the gapless records of nasw.h:157-171.  The tables restate
nasw-tab.c: the alphabet orders (nasw-tab.c:6-12), genetic code 1
(nasw-tab.c:22), BLOSUM62 in that order (nasw-tab.c:59-83), ns_make_tables
(nasw-tab.c:85-107), the splice models (nasw-tab.c:124-129) and
ns_set_stop_sc (nasw-tab.c:149-156).  ProtLocus's option defaults come from
options.c:125-138 mapped by align.c:59-71.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

NS_CIGAR_STR = "MIDNSHP=XBFGUVE"
NS_F_CIGAR, NS_F_EXT_LEFT, NS_F_EXT_RIGHT, NS_F_GPU = 0x1, 0x2, 0x4, 0x8
NS_S_NONE, NS_S_GENERIC, NS_S_MAMMAL = 0, 1, 2

NT_I2C = "ACGTN"
AA_I2C = "ARNDCQEGHILKMFPSTWYV*X"

# NCBI translation table 1 in AAA, AAC, AAG, AAT, ACA, ... order (64 codons + 'X')
CODE1 = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLFX"

# BLOSUM62 over ARNDCQEGHILKMFPSTWYV*X
_B62 = """
 4 -1 -2 -2  0 -1 -1  0 -2 -1 -1 -1 -1 -2 -1  1  0 -3 -2  0 -4  0
-1  5  0 -2 -3  1  0 -2  0 -3 -2  2 -1 -3 -2 -1 -1 -3 -2 -3 -4 -1
-2  0  6  1 -3  0  0  0  1 -3 -3  0 -2 -3 -2  1  0 -4 -2 -3 -4 -1
-2 -2  1  6 -3  0  2 -1 -1 -3 -4 -1 -3 -3 -1  0 -1 -4 -3 -3 -4 -1
 0 -3 -3 -3  9 -3 -4 -3 -3 -1 -1 -3 -1 -2 -3 -1 -1 -2 -2 -1 -4 -2
-1  1  0  0 -3  5  2 -2  0 -3 -2  1  0 -3 -1  0 -1 -2 -1 -2 -4 -1
-1  0  0  2 -4  2  5 -2  0 -3 -3  1 -2 -3 -1  0 -1 -3 -2 -2 -4 -1
 0 -2  0 -1 -3 -2 -2  6 -2 -4 -4 -2 -3 -3 -2  0 -2 -2 -3 -3 -4 -1
-2  0  1 -1 -3  0  0 -2  8 -3 -3 -1 -2 -1 -2 -1 -2 -2  2 -3 -4 -1
-1 -3 -3 -3 -1 -3 -3 -4 -3  4  2 -3  1  0 -3 -2 -1 -3 -1  3 -4 -1
-1 -2 -3 -4 -1 -2 -3 -4 -3  2  4 -2  2  0 -3 -2 -1 -2 -1  1 -4 -1
-1  2  0 -1 -3  1  1 -2 -1 -3 -2  5 -1 -3 -1  0 -1 -3 -2 -2 -4 -1
-1 -1 -2 -3 -1  0 -2 -3 -2  1  2 -1  5  0 -2 -1 -1 -1 -1  1 -4 -1
-2 -3 -3 -3 -2 -3 -3 -3 -1  0  0 -3  0  6 -4 -2 -2  1  3 -1 -4 -1
-1 -2 -2 -1 -3 -1 -1 -2 -2 -3 -3 -1 -2 -4  7 -1 -1 -4 -3 -2 -4 -2
 1 -1  1  0 -1  0  0  0 -1 -2 -2  0 -1 -2 -1  4  1 -3 -2 -2 -4  0
 0 -1  0 -1 -1 -1 -1 -2 -2 -1 -1 -1 -1 -2 -1  1  5 -2 -2  0 -4  0
-3 -3 -4 -4 -2 -2 -3 -2 -2 -3 -2 -3 -1  1 -4 -3 -2 11  2 -3 -4 -2
-2 -2 -2 -3 -2 -1 -2 -3  2 -1 -1 -2 -1  3 -3 -2 -2  2  7 -1 -4 -1
 0 -3 -3 -3 -1 -2 -2 -3 -3  3  1 -2  1 -1 -2 -2  0 -3 -1  4 -4 -1
-4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4 -4  1 -4
 0 -1 -1 -1 -2 -1 -1 -1 -1 -1 -1 -1 -1 -1 -2  0  0 -2 -1 -1 -4 -1
"""
BLOSUM62 = np.array(_B62.split(), dtype=np.int8).reshape(22, 22)


def make_tables(code: str = CODE1):
    """nt4 / aa20 / codon lookup tables (the ns_make_tables algorithm)."""
    nt4 = np.full(256, 4, dtype=np.uint8)
    for i, ch in enumerate(NT_I2C):
        nt4[i] = i
        nt4[ord(ch.upper())] = i
        nt4[ord(ch.lower())] = i
    aa20 = np.full(256, 21, dtype=np.uint8)
    for i, ch in enumerate(AA_I2C):
        aa20[i] = i
        aa20[ord(ch.upper())] = i
        aa20[ord(ch.lower())] = i
    codon = np.array([aa20[ord(code[i])] for i in range(64)], dtype=np.uint8)
    return nt4, aa20, codon


def set_stop_sc(mat: np.ndarray, pen: int) -> np.ndarray:
    """stop row/column = -pen, except stop:stop kept (ns_set_stop_sc)."""
    m = mat.copy()
    s = AA_I2C.index("*")
    keep = m[s, s]
    m[s, :] = -pen
    m[:, s] = -pen
    m[s, s] = keep
    return m


def splice_model(model: int):
    if model == NS_S_MAMMAL:
        return [8, 15, 21, 30, 4, 4]
    if model == NS_S_GENERIC:
        return [8, 15, 21, 30, 0, 0]
    return [0] * 6


class NsOpt(C.Structure):
    _fields_ = [
        ("flag", C.c_int32), ("go", C.c_int32), ("ge", C.c_int32), ("io", C.c_int32), ("fs", C.c_int32),
        ("xdrop", C.c_int32), ("end_bonus", C.c_int32), ("asize", C.c_int32), ("gpu_device", C.c_int32),
        ("gpu_min_cells", C.c_int64), ("sp", C.c_int32 * 6), ("sp_null_bonus", C.c_int32),
        ("ie_coef", C.c_float), ("sc", C.POINTER(C.c_int8)), ("pssm", C.POINTER(C.c_int8)),
        ("nt4", C.POINTER(C.c_uint8)), ("aa20", C.POINTER(C.c_uint8)), ("codon", C.POINTER(C.c_uint8)),
    ]


class NsRst(C.Structure):
    _fields_ = [
        ("n_cigar", C.c_int32), ("m_cigar", C.c_int32), ("nt_len", C.c_int32), ("aa_len", C.c_int32),
        ("score", C.c_int32), ("cigar", C.POINTER(C.c_uint32)),
    ]


class GaplessCandidate(C.Structure):
    _fields_ = [("target_offset", C.c_int64), ("target_length", C.c_int64), ("query_offset", C.c_int64),
                ("query_length", C.c_int32), ("anchor_offset", C.c_int32), ("anchor_count", C.c_int32),
                ("reverse", C.c_int32)]


class GaplessAnchor(C.Structure):
    _fields_ = [("target_block", C.c_int64), ("query_end", C.c_int32), ("reserved", C.c_int32)]


class SpliceJob(C.Structure):
    _fields_ = [("nt_off", C.c_int64), ("aa_off", C.c_int64), ("ss_off", C.c_int64),
                ("nl", C.c_int32), ("al", C.c_int32)]


class SpliceResult(C.Structure):
    _fields_ = [("score", C.c_int32), ("n_cigar", C.c_int32), ("cigar_off", C.c_int64),
                ("mode", C.c_int32), ("status", C.c_int32)]


class ExtJob(C.Structure):
    """pl_ext_job_t"""
    _fields_ = [("nt_off", C.c_int64), ("aa_off", C.c_int64), ("ss_off", C.c_int64), ("pssm_off", C.c_int64),
                ("nl", C.c_int32), ("al", C.c_int32), ("flag", C.c_int32), ("width", C.c_int32)]


class ExtResult(C.Structure):
    """pl_ext_result_t"""
    _fields_ = [("nt_len", C.c_int32), ("aa_len", C.c_int32), ("score", C.c_int32), ("status", C.c_int32)]


assert C.sizeof(NsOpt) == 120, C.sizeof(NsOpt)
assert C.sizeof(ExtJob) == 48
assert C.sizeof(ExtResult) == 16
assert C.sizeof(SpliceJob) == 32
assert C.sizeof(SpliceResult) == 24


class Options:
    """Owns the table arrays an NsOpt points into (keeps them alive)."""

    def __init__(self, *, go=11, ge=1, io=29, fs=23, xdrop=100, end_bonus=5, sp_model=NS_S_GENERIC,
                 sp_null_bonus=-7, ie_coef=0.5, flag=0, matrix: np.ndarray | None = None,
                 stop_pen: int | None = None, sp: list[int] | None = None, code: str = CODE1):
        self.nt4, self.aa20, self.codon = make_tables(code)
        if matrix is None:
            matrix = set_stop_sc(BLOSUM62, fs if stop_pen is None else stop_pen)
        self.mat = np.ascontiguousarray(matrix, dtype=np.int8).reshape(-1)
        o = NsOpt()
        o.flag, o.go, o.ge, o.io, o.fs = flag, go, ge, io, fs
        o.xdrop, o.end_bonus, o.asize = xdrop, end_bonus, 22
        o.gpu_device, o.gpu_min_cells = 0, 0
        for i, v in enumerate(sp if sp is not None else splice_model(sp_model)):
            o.sp[i] = v
        o.sp_null_bonus = sp_null_bonus
        o.ie_coef = ie_coef
        o.sc = self.mat.ctypes.data_as(C.POINTER(C.c_int8))
        o.pssm = None
        o.nt4 = self.nt4.ctypes.data_as(C.POINTER(C.c_uint8))
        o.aa20 = self.aa20.ctypes.data_as(C.POINTER(C.c_uint8))
        o.codon = self.codon.ctypes.data_as(C.POINTER(C.c_uint8))
        self.c = o

    @property
    def ptr(self):
        return C.byref(self.c)

    def with_flag(self, flag: int) -> "Options":
        n = Options.__new__(Options)
        n.nt4, n.aa20, n.codon, n.mat = self.nt4, self.aa20, self.codon, self.mat
        n.pssm_arr = getattr(self, "pssm_arr", None)
        n.c = NsOpt.from_buffer_copy(self.c)
        n.c.flag = flag
        return n

    def with_pssm(self, pssm: np.ndarray | None) -> "Options":
        """A copy whose ns_opt_t.pssm points at `pssm` (al x 22 int8, rows in query order; nasw.h:73)."""
        n = self.with_flag(self.c.flag)
        if pssm is None:
            n.pssm_arr = None
            n.c.pssm = None
        else:
            n.pssm_arr = np.ascontiguousarray(pssm, dtype=np.int8).reshape(-1)
            n.c.pssm = n.pssm_arr.ctypes.data_as(C.POINTER(C.c_int8))
        return n

    @classmethod
    def nasw_defaults(cls, **kw) -> "Options":
        """ns_opt_init() defaults (nasw-tab.c:131-147): fs=17, MAMMAL splice model, plain BLOSUM62."""
        args = dict(go=11, ge=1, io=29, fs=17, xdrop=100, end_bonus=5, sp_model=NS_S_MAMMAL,
                    sp_null_bonus=-7, ie_coef=0.5, matrix=BLOSUM62)
        args.update(kw)
        return cls(**args)


def cigar_str(words) -> str:
    return "".join(f"{w >> 4}{NS_CIGAR_STR[w & 0xf]}" for w in words)


class ExtraJob(C.Structure):
    """pl_extra_job_t"""
    _fields_ = [("cigar_off", C.c_int64), ("nt_off", C.c_int64), ("aa_off", C.c_int64), ("pssm_off", C.c_int64),
                ("l_nt", C.c_int64), ("vs", C.c_int64), ("ve", C.c_int64), ("feat_off", C.c_int64),
                ("qs", C.c_int32), ("qe", C.c_int32), ("n_cigar", C.c_int32), ("has_stop", C.c_int32),
                ("feat_cap", C.c_int32), ("pad", C.c_int32)]


class Feat(C.Structure):
    """pl_feat_t (mp_feat_t, protlocus.h:230-237)"""
    _fields_ = [("vs", C.c_int64), ("ve", C.c_int64), ("qs", C.c_int32), ("qe", C.c_int32), ("type", C.c_int16),
                ("phase", C.c_int16), ("n_fs", C.c_int32), ("n_stop", C.c_int32), ("score", C.c_int32),
                ("n_iden", C.c_int32), ("blen", C.c_int32), ("donor", C.c_char * 2), ("acceptor", C.c_char * 2)]


class ExtraResult(C.Structure):
    """pl_extra_result_t"""
    _fields_ = [("blen", C.c_int32), ("n_iden", C.c_int32), ("n_plus", C.c_int32), ("n_fs", C.c_int32),
                ("n_stop", C.c_int32), ("dp_max", C.c_int32), ("n_exon", C.c_int32), ("n_feat", C.c_int32),
                ("ok", C.c_int32), ("pad", C.c_int32)]


class PsJob(C.Structure):
    """pl_ps_job_t"""
    _fields_ = [("pssm_off", C.c_int64), ("orf_off", C.c_int64), ("L", C.c_int32), ("n", C.c_int32),
                ("diag", C.c_int32), ("band", C.c_int32)]


class ChainOpt(C.Structure):
    """pl_chain_opt_t: the arguments of mp_chain (chain.c:160)."""
    _fields_ = [("max_dist_x", C.c_int32), ("max_dist_y", C.c_int32), ("bw", C.c_int32), ("max_skip", C.c_int32),
                ("max_iter", C.c_int32), ("min_cnt", C.c_int32), ("min_sc", C.c_int32), ("chn_coef_log", C.c_float),
                ("is_spliced", C.c_int32), ("kmer", C.c_int32), ("bbit", C.c_int32), ("pad", C.c_int32)]


def chain_opt(kind: str = "main", max_intron: int = 36000, bbit: int = 8, kmer: int = 6) -> dict:
    """mp_chain's arguments at the reference's defaults (options.c:44-60, index kmer 6, bbit 8):
    "main" = the coarse chain of mp_map_coarse (map.c:630), "pre" = its pre-chain (map.c:618,
    w = 1 << bbit); max_intron = bw, set from the genome size (options.c:31-38)."""
    if kind == "pre":
        w = 1 << bbit
        return dict(max_dist_x=w, max_dist_y=w, bw=w, max_skip=25, max_iter=1000000, min_cnt=2, min_sc=0, coef=0.75,
                    is_spliced=1, kmer=kmer, bbit=bbit)
    return dict(max_dist_x=max_intron, max_dist_y=1000, bw=max_intron, max_skip=25, max_iter=1000000, min_cnt=3,
                min_sc=0, coef=0.75, is_spliced=1, kmer=kmer, bbit=bbit)


def chain_opt_struct(o: dict) -> ChainOpt:
    return ChainOpt(o["max_dist_x"], o["max_dist_y"], o["bw"], o["max_skip"], o["max_iter"], o["min_cnt"], o["min_sc"],
                    o["coef"], o["is_spliced"], o["kmer"], o["bbit"], 0)
