"""ctypes binding of libplgpu.so (the C ABI declared in include/plgpu.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from .abi import (ChainOpt, ExtraJob, ExtraResult, Feat, PsJob, ExtJob, ExtResult, NsOpt, NsRst, SpliceJob,
                  SpliceResult, chain_opt_struct)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplgpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "plgpu.h")

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C protlocus_b200/csrc` "
                           "(or __graft_entry__.build()); there is no fallback")
    lib = C.CDLL(LIB_PATH)
    lib.ns_gpu_init.argtypes = [C.c_int32]
    lib.ns_gpu_init.restype = C.c_int
    for fn in ("ns_gpu_error", "ns_gpu_name", "pl_last_error"):
        getattr(lib, fn).restype = C.c_char_p
    for fn in ("ns_gpu_dispatch_count", "ns_gpu_launch_count", "pl_kernel_launch_count"):
        getattr(lib, fn).restype = C.c_uint64
    for fn in ("ns_gpu_h2d_seconds", "ns_gpu_kernel_seconds", "ns_gpu_d2h_seconds"):
        getattr(lib, fn).restype = C.c_double
    lib.ns_gpu_submit.argtypes = [C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt), C.c_void_p]
    lib.ns_gpu_submit.restype = C.c_void_p
    lib.ns_gpu_wait.argtypes = [C.c_void_p, C.POINTER(NsRst)]
    lib.ns_gpu_wait.restype = C.c_int
    lib.ns_gpu_global.argtypes = [C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt),
                                  C.c_void_p, C.POINTER(NsRst)]
    lib.ns_gpu_global.restype = C.c_int
    lib.pl_engine_create.argtypes = [C.c_int32, C.c_int64]
    lib.pl_engine_create.restype = C.c_void_p
    lib.pl_engine_destroy.argtypes = [C.c_void_p]
    lib.pl_engine_last_plan.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.pl_splice_batch_host.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                         C.POINTER(SpliceResult), C.c_void_p, C.c_int64]
    lib.pl_splice_batch_host.restype = C.c_int
    lib.pl_splice_batch_device.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                           C.POINTER(C.c_int64), C.c_void_p]
    lib.pl_splice_batch_device.restype = C.c_int
    lib.pl_engine_set_timing.argtypes = [C.c_void_p, C.c_int32]
    lib.pl_engine_times.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4 + [C.POINTER(C.c_int64)] * 2
    lib.pl_engine_stream.argtypes = [C.c_void_p]
    lib.pl_engine_stream.restype = C.c_void_p
    lib.pl_measure_int_peak.argtypes = [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.pl_measure_int_peak.restype = C.c_int
    lib.pl_splice_batch_noalloc.argtypes = [C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                            C.POINTER(C.c_int64), C.c_void_p]
    lib.pl_splice_batch_noalloc.restype = C.c_int
    lib.pl_noalloc_error.restype = C.c_char_p
    lib.pl_ext_stripe_width.argtypes = [C.POINTER(NsOpt), C.c_int32]
    lib.pl_ext_stripe_width.restype = C.c_int32
    lib.pl_ext_batch_host.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(ExtJob), C.c_int32,
                                      C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                      C.c_void_p, C.c_int64, C.POINTER(ExtResult)]
    lib.pl_ext_batch_host.restype = C.c_int
    lib.pl_ext_batch_device.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(ExtJob), C.c_int32,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_ext_batch_device.restype = C.c_int
    lib.pl_ext_last_cells.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.ns_ext_batch_init.argtypes = [C.c_void_p]
    lib.ns_ext_batch_init.restype = C.c_void_p
    lib.ns_ext_batch_add.argtypes = [C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(NsOpt),
                                     C.c_void_p]
    lib.ns_ext_batch_add.restype = C.c_int32
    lib.ns_ext_batch_flush.argtypes = [C.c_void_p]
    lib.ns_ext_batch_flush.restype = C.c_int32
    lib.ns_ext_batch_ready.argtypes = [C.c_void_p, C.c_int32]
    lib.ns_ext_batch_ready.restype = C.c_int
    lib.ns_ext_batch_wait.argtypes = [C.c_void_p]
    lib.ns_ext_batch_get.argtypes = [C.c_void_p, C.c_int32]
    lib.ns_ext_batch_get.restype = C.POINTER(NsRst)
    lib.ns_ext_batch_destroy.argtypes = [C.c_void_p]
    for fn in ("ns_ext_gpu_launch_count", "ns_ext_gpu_request_count"):
        getattr(lib, fn).restype = C.c_uint64
    lib.pl_hmm_profile_create.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_hmm_profile_create.restype = C.c_void_p
    lib.pl_hmm_profile_destroy.argtypes = [C.c_void_p]
    lib.pl_hmm_score_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
    lib.pl_hmm_score_host.restype = C.c_int
    lib.pl_hmm_score_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]
    lib.pl_hmm_score_device.restype = C.c_int
    lib.pl_hmm_score_many_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_hmm_score_many_device.restype = C.c_int
    lib.pl_hmm_score_many_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_hmm_score_many_host.restype = C.c_int
    lib.pl_hmm_last_cells.argtypes = [C.c_void_p]
    lib.pl_hmm_last_cells.restype = C.c_int64
    lib.mp_hmm_dp_score_gpu.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.mp_hmm_dp_score_gpu.restype = C.c_int32
    gl = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64,
          C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    lib.ns_gpu_gapless_score_batch.argtypes = gl
    lib.ns_gpu_gapless_score_batch.restype = C.c_int
    lib.pl_gapless_score_host.argtypes = [C.c_void_p] + gl
    lib.pl_gapless_score_host.restype = C.c_int
    lib.pl_gapless_score_device.argtypes = [C.c_void_p] + gl + [C.c_void_p]
    lib.pl_gapless_score_device.restype = C.c_int
    lib.pl_gapless_last_steps.argtypes = [C.c_void_p]
    lib.pl_gapless_last_steps.restype = C.c_int64
    lib.ns_gpu_gapless_profile.argtypes = [C.c_void_p]
    lib.ns_gpu_gapless_reset_target.argtypes = []
    lib.pl_rc_profile_create.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    lib.pl_rc_profile_create.restype = C.c_void_p
    lib.pl_rc_profile_destroy.argtypes = [C.c_void_p]
    lib.pl_rc_score_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    lib.pl_rc_score_host.restype = C.c_int
    lib.pl_rc_last_cells.argtypes = [C.c_void_p]
    lib.pl_rc_last_cells.restype = C.c_int64
    lib.pl_rc_mathf_eval.argtypes = [C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, C.c_int64, C.c_void_p]
    lib.pl_rc_mathf_eval.restype = C.c_int
    lib.pl_rc_debug_wait_limit.argtypes = [C.c_int64]
    lib.pl_rc_debug_wait_limit.restype = C.c_int
    lib.pl_seed_index_create.argtypes = [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32]
    lib.pl_seed_index_create.restype = C.c_void_p
    lib.pl_seed_index_destroy.argtypes = [C.c_void_p]
    lib.pl_seed_anchors_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                         C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64]
    lib.pl_seed_anchors_host.restype = C.c_int64
    lib.pl_seed_anchors_opt_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p, C.POINTER(SeedOpt), C.c_void_p, C.c_void_p, C.c_int64]
    lib.pl_seed_anchors_opt_host.restype = C.c_int64
    lib.pl_seed_anchors_opt_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                               C.c_void_p, C.POINTER(SeedOpt), C.c_void_p, C.POINTER(C.c_void_p)]
    lib.pl_seed_anchors_opt_device.restype = C.c_int64
    lib.pl_seed_qname_hash.argtypes = [C.c_char_p]
    lib.pl_seed_qname_hash.restype = C.c_uint32
    lib.pl_seed_anchors_hmm_host.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p, C.POINTER(SeedOpt), C.POINTER(SeedHmm), C.c_void_p,
                                             C.c_void_p, C.c_int64]
    lib.pl_seed_anchors_hmm_host.restype = C.c_int64
    lib.pl_seed_anchors_hmm_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                               C.c_void_p, C.POINTER(SeedOpt), C.POINTER(SeedHmm), C.c_void_p,
                                               C.POINTER(C.c_void_p)]
    lib.pl_seed_anchors_hmm_device.restype = C.c_int64
    lib.pl_pf_decide.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_double, C.c_int32,
                                 C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_pf_decide.restype = C.c_int
    lib.pl_pf_select_device.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(NsOpt), C.c_void_p, C.c_int32, C.c_void_p,
                                        C.c_void_p, C.c_double, C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_pf_select_device.restype = C.c_int
    lib.pl_engine_last_pairs.argtypes = [C.c_void_p]
    lib.pl_engine_last_pairs.restype = C.c_int32
    lib.pl_engine_set_pairing.argtypes = [C.c_void_p, C.c_int32]
    lib.pl_engine_set_graphs.argtypes = [C.c_void_p, C.c_int32]
    lib.pl_engine_graph_replays.argtypes = [C.c_void_p]
    lib.pl_engine_graph_replays.restype = C.c_int64
    lib.pl_group_create.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    lib.pl_group_create.restype = C.c_void_p
    lib.pl_group_destroy.argtypes = [C.c_void_p]
    lib.pl_group_engine.argtypes = [C.c_void_p, C.c_int32]
    lib.pl_group_engine.restype = C.c_void_p
    lib.pl_group_splice_host.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                         C.POINTER(SpliceResult), C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    lib.pl_group_splice_host.restype = C.c_int
    lib.pl_group_plan.argtypes = [C.POINTER(SpliceJob), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    lib.pl_group_plan.restype = C.c_int
    lib.pl_group_gather.argtypes = [C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                    C.POINTER(SpliceResult), C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    lib.pl_group_gather.restype = C.c_int
    lib.pl_debug_fault.argtypes = [C.c_int32, C.c_int32]
    lib.pl_debug_fault.restype = C.c_int
    lib.pl_ext_failed_count.restype = C.c_uint64
    lib.pl_extra_cal_host.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.POINTER(ExtraJob), C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.POINTER(ExtraResult),
                                      C.POINTER(Feat), C.c_int64]
    lib.pl_extra_cal_host.restype = C.c_int
    lib.pl_ps_band_cells.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    lib.pl_ps_band_cells.restype = C.c_int64
    lib.pl_ps_gapped_host.argtypes = [C.c_void_p, C.POINTER(PsJob), C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_int64, C.c_int32, C.c_int32, C.c_void_p]
    lib.pl_ps_gapped_host.restype = C.c_int
    lib.pl_extra_cal_device.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.POINTER(ExtraJob), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_extra_cal_device.restype = C.c_int
    lib.pl_ps_gapped_device.argtypes = [C.c_void_p, C.POINTER(PsJob), C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                        C.c_int32, C.c_void_p, C.c_void_p]
    lib.pl_ps_gapped_device.restype = C.c_int
    lib.pl_chain_host.argtypes = [C.c_void_p, C.POINTER(ChainOpt), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_chain_host.restype = C.c_int
    lib.pl_chain_fill_device.argtypes = [C.c_void_p, C.POINTER(ChainOpt), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_chain_fill_device.restype = C.c_int
    lib.pl_chain_finish.argtypes = [C.POINTER(ChainOpt), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_int32), C.c_void_p]
    lib.pl_chain_finish.restype = C.c_int
    lib.pl_chain_last_pairs.argtypes = [C.c_void_p]
    lib.pl_chain_last_pairs.restype = C.c_int64
    lib.pl_engine_set_tuning.argtypes = [C.c_void_p, C.c_int32, C.c_double]
    lib.pl_engine_get_tuning.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    lib.pl_engine_autotune.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    lib.pl_engine_autotune.restype = C.c_int
    lib.pl_pf_model_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64]
    lib.pl_pf_model_create.restype = C.c_void_p
    lib.pl_pf_model_destroy.argtypes = [C.c_void_p]
    lib.pl_pf_model_size.argtypes = [C.c_void_p]
    lib.pl_pf_model_size.restype = C.c_int64
    lib.pl_pf_model_get.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.pl_pf_model_get.restype = C.c_int
    lib.pl_pf_model_set.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.pl_pf_model_set.restype = C.c_int
    lib.pl_pf_features_device.argtypes = [C.c_void_p, C.POINTER(NsOpt), C.POINTER(SpliceJob), C.c_int32, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.pl_pf_features_device.restype = C.c_int
    lib.pl_pf_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    lib.pl_pf_predict.restype = C.c_int
    lib.pl_pf_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
    lib.pl_pf_train.restype = C.c_int
    lib.pl_pf_gemm.argtypes = [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                               C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                               C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    lib.pl_pf_gemm.restype = C.c_int
    _lib = lib
    return lib


def declared_symbols(header: str = HEADER) -> list[str]:
    """Function names declared in include/plgpu.h."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", text, flags=re.M)
    return sorted({n for n in names if n not in ("if", "while", "for", "return", "sizeof")})


def error() -> str:
    return load().pl_last_error().decode()


_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def chain_pack(queries):
    """(off int64, n int32, anchors uint64) of a list of per-query anchor arrays."""
    n = np.array([len(x) for x in queries], np.int32)
    off = np.zeros(len(queries), np.int64)
    if len(queries) > 1:
        off[1:] = np.cumsum(n[:-1], dtype=np.int64)
    a = np.concatenate([np.asarray(x, np.uint64) for x in queries]) if len(queries) else np.zeros(0, np.uint64)
    return off, n, np.ascontiguousarray(a, np.uint64)


def chain_unpack(off, n_u, u, a_out):
    out = []
    for q in range(len(off)):
        k = int(n_u[q])
        uq = u[off[q]: off[q] + k].copy()
        tot = int((uq & np.uint64(0xFFFFFFFF)).sum()) if k else 0
        out.append((uq, a_out[off[q]: off[q] + tot].copy()))
    return out


def chain_finish(opt: dict, a, f, p):
    """The host half of mp_chain for one query from a fill's f and p (pl_chain_finish)."""
    a = np.ascontiguousarray(a, np.uint64)
    f = np.ascontiguousarray(f, np.int32)
    p = np.ascontiguousarray(p, np.int32)
    n = len(a)
    u = np.zeros(max(n, 1), np.uint64)
    a_out = np.zeros(max(n, 1), np.uint64)
    n_u = C.c_int32()
    o = chain_opt_struct(opt)
    if not load().pl_chain_finish(C.byref(o), n, a.ctypes.data, f.ctypes.data, p.ctypes.data, u.ctypes.data,
                                  C.byref(n_u), a_out.ctypes.data):
        raise RuntimeError("pl_chain_finish: " + error())
    k = n_u.value
    tot = int((u[:k] & np.uint64(0xFFFFFFFF)).sum()) if k else 0
    return u[:k].copy(), a_out[:tot].copy()


class Engine:
    """A pl_engine_t on one device (bulk global spliced DP)."""

    def __init__(self, device: int = 0, trace_budget_bytes: int = 0):
        self.lib = load()
        self.h = self.lib.pl_engine_create(device, trace_budget_bytes)
        if not self.h:
            raise RuntimeError("pl_engine_create failed: " + error())

    def close(self):
        if self.h:
            self.lib.pl_engine_destroy(self.h)
            self.h = None

    def set_pairing(self, on):
        """False: off; True: pairs within the per-CTA share of the batch; 2: every eligible job."""
        self.lib.pl_engine_set_pairing(self.h, 2 if on == 2 else int(bool(on)))

    def last_pairs(self) -> int:
        return int(self.lib.pl_engine_last_pairs(self.h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_timing(self, on: bool = True):
        """(Re)start CUDA-event timing of the batch phases."""
        if not self.lib.pl_engine_set_timing(self.h, int(on)):
            raise RuntimeError("pl_engine_set_timing failed: " + error())

    def times(self):
        v = [C.c_double() for _ in range(4)]
        n = [C.c_int64() for _ in range(2)]
        self.lib.pl_engine_times(self.h, *[C.byref(x) for x in v], *[C.byref(x) for x in n])
        return {"prep_ms": v[0].value, "dp_ms": v[1].value, "traceback_ms": v[2].value,
                "compact_ms": v[3].value, "dp_launches": n[0].value, "cells": n[1].value}

    @property
    def stream(self) -> int:
        return self.lib.pl_engine_stream(self.h) or 0

    @staticmethod
    def extra_pack(alns):
        """Packs alignments for extra_run: list of dicts with cigar (words), nt4 (0-4 codes from
        r->vs), aa (bytes from r->qs), vs, ve, qs, qe, has_stop and optional pssm rows."""
        n = len(alns)
        jobs = (ExtraJob * n)()
        cig, nts, aas, pss = [], [], [], []
        co = no = ao = po = fo = 0
        for q, a in enumerate(alns):
            J = jobs[q]
            c = np.asarray(a["cigar"], np.uint32)
            J.cigar_off, J.n_cigar = co, len(c)
            J.nt_off, J.l_nt = no, len(a["nt4"])
            J.aa_off = ao
            J.pssm_off = po if a.get("pssm") is not None else -1
            J.vs, J.ve, J.qs, J.qe, J.has_stop = a["vs"], a["ve"], a["qs"], a["qe"], int(a["has_stop"])
            J.feat_off, J.feat_cap = fo, len(c) + 2
            cig.append(c)
            nts.append(np.asarray(a["nt4"], np.uint8))
            aas.append(a["aa"])
            co, no, ao, fo = co + len(c), no + len(a["nt4"]), ao + len(a["aa"]), fo + len(c) + 2
            if a.get("pssm") is not None:
                p = np.asarray(a["pssm"], np.int8).reshape(-1)
                pss.append(p)
                po += p.size
        return {"n": n, "jobs": jobs, "n_cig": co, "n_nt": no, "n_aa": ao, "n_pssm": po, "n_feat": fo,
                "cig": np.ascontiguousarray(np.concatenate(cig) if cig else np.zeros(1, np.uint32)),
                "nt": np.ascontiguousarray(np.concatenate(nts) if nts else np.zeros(1, np.uint8)),
                "aa": np.frombuffer(b"".join(aas) or b"X", np.uint8).copy(),
                "pssm": np.ascontiguousarray(np.concatenate(pss)) if pss else None,
                "res": (ExtraResult * max(n, 1))(), "feats": (Feat * max(fo, 1))()}

    def extra_run(self, pk, go: int, ge: int, fs: int, mat, codon, aa20):
        """pl_extra_cal_host over a packed batch; results stay in pk["res"] / pk["feats"]."""
        m = np.ascontiguousarray(np.asarray(mat, np.int8))
        cd = np.ascontiguousarray(np.asarray(codon, np.uint8))
        a20 = np.ascontiguousarray(np.asarray(aa20, np.uint8))
        if not self.lib.pl_extra_cal_host(self.h, go, ge, fs, 22, m.ctypes.data, cd.ctypes.data, a20.ctypes.data,
                                          pk["jobs"], pk["n"], pk["cig"].ctypes.data, pk["n_cig"], pk["nt"].ctypes.data,
                                          pk["n_nt"], pk["aa"].ctypes.data, pk["n_aa"],
                                          None if pk["pssm"] is None else pk["pssm"].ctypes.data, pk["n_pssm"],
                                          pk["res"], pk["feats"], pk["n_feat"]):
            raise RuntimeError("pl_extra_cal_host: " + error())
        return pk

    def extra_upload(self, pk):
        """Device copies (torch tensors) of a packed batch's inputs and outputs, for extra_run_device."""
        import torch
        d = {k: torch.from_numpy(np.ascontiguousarray(pk[k])).to("cuda") for k in ("cig", "nt", "aa")}
        d["pssm"] = torch.from_numpy(pk["pssm"]).to("cuda") if pk["pssm"] is not None else None
        d["res"] = torch.zeros(max(pk["n"], 1) * C.sizeof(ExtraResult), dtype=torch.uint8, device="cuda")
        d["feats"] = torch.zeros(max(pk["n_feat"], 1) * C.sizeof(Feat), dtype=torch.uint8, device="cuda")
        return d

    def extra_run_device(self, pk, d, go: int, ge: int, fs: int, mat, codon, aa20, stream=None):
        """pl_extra_cal_device over a packed batch whose buffers are on the device (extra_upload)."""
        m = np.ascontiguousarray(np.asarray(mat, np.int8))
        cd = np.ascontiguousarray(np.asarray(codon, np.uint8))
        a20 = np.ascontiguousarray(np.asarray(aa20, np.uint8))
        if not self.lib.pl_extra_cal_device(self.h, go, ge, fs, 22, m.ctypes.data, cd.ctypes.data, a20.ctypes.data,
                                            pk["jobs"], pk["n"], d["cig"].data_ptr(), d["nt"].data_ptr(),
                                            d["aa"].data_ptr(), d["pssm"].data_ptr() if d["pssm"] is not None else None,
                                            d["res"].data_ptr(), d["feats"].data_ptr(), stream):
            raise RuntimeError("pl_extra_cal_device: " + error())

    def ps_run_device(self, pk, d_pssm, d_orf, d_score, go: int = 11, ge: int = 1, stream=None):
        """pl_ps_gapped_device: pssm / orf / score buffers already on the device (torch tensors)."""
        if not self.lib.pl_ps_gapped_device(self.h, pk["jobs"], pk["n"], d_pssm.data_ptr(), d_orf.data_ptr(), go, ge,
                                            d_score.data_ptr(), stream):
            raise RuntimeError("pl_ps_gapped_device: " + error())

    def extra_cal(self, alns, go: int, ge: int, fs: int, mat, codon, aa20):
        """Alignment statistics and exon features on the device (see extra_pack).
        Returns [(ExtraResult, [Feat])]."""
        pk = self.extra_run(self.extra_pack(alns), go, ge, fs, mat, codon, aa20)
        jobs, res, feats = pk["jobs"], pk["res"], pk["feats"]
        return [(res[q], [feats[jobs[q].feat_off + k] for k in range(min(res[q].n_feat, jobs[q].feat_cap))])
                for q in range(pk["n"])]

    @staticmethod
    def ps_pack(cands):
        """Packs (pssm [L x 22] int8, orf codes, diag, band) candidates for ps_run."""
        n = len(cands)
        jobs = (PsJob * n)()
        ps, orfs = [], []
        po = oo = 0
        for q, (pssm, orf, diag, band) in enumerate(cands):
            p = np.ascontiguousarray(np.asarray(pssm, np.int8).reshape(-1, 22))
            o = np.ascontiguousarray(np.asarray(orf, np.uint8))
            jobs[q].pssm_off, jobs[q].orf_off, jobs[q].L, jobs[q].n = po, oo, p.shape[0], o.size
            jobs[q].diag, jobs[q].band = int(diag), int(band)
            ps.append(p.reshape(-1))
            orfs.append(o)
            po, oo = po + p.size, oo + o.size
        return {"n": n, "jobs": jobs, "n_pssm": po, "n_orf": oo,
                "pssm": np.ascontiguousarray(np.concatenate(ps) if ps else np.zeros(1, np.int8)),
                "orf": np.ascontiguousarray(np.concatenate(orfs) if orfs else np.zeros(1, np.uint8)),
                "score": np.zeros(max(n, 1), np.int32)}

    def ps_run(self, pk, go: int = 11, ge: int = 1) -> np.ndarray:
        if not self.lib.pl_ps_gapped_host(self.h, pk["jobs"], pk["n"], pk["pssm"].ctypes.data, pk["n_pssm"],
                                          pk["orf"].ctypes.data, pk["n_orf"], go, ge, pk["score"].ctypes.data):
            raise RuntimeError("pl_ps_gapped_host: " + error())
        return pk["score"][: pk["n"]]

    def chain(self, opt: dict, queries):
        """mp_chain over many queries on the device (pl_chain_host).  queries: list of sorted
        uint64 anchor arrays.  Returns per query (u words, chained anchors) as numpy arrays."""
        off, n, a = chain_pack(queries)
        n_q, n_a = len(queries), len(a)
        u = np.zeros(max(n_a, 1), np.uint64)
        a_out = np.zeros(max(n_a, 1), np.uint64)
        n_u = np.zeros(max(n_q, 1), np.int32)
        o = chain_opt_struct(opt)
        if not self.lib.pl_chain_host(self.h, C.byref(o), n_q, off.ctypes.data, n.ctypes.data, a.ctypes.data, n_a,
                                      u.ctypes.data, n_u.ctypes.data, a_out.ctypes.data):
            raise RuntimeError("pl_chain_host: " + error())
        return chain_unpack(off, n_u, u, a_out)

    def ps_gapped(self, cands, go: int = 11, ge: int = 1) -> np.ndarray:
        """Prescreen banded gapped scores of (pssm [L x 22] int8, orf codes, diag, band) candidates."""
        return self.ps_run(self.ps_pack(cands), go, ge)

    def set_tuning(self, r4_rows: int = -1, coop_ratio: float = 0.0):
        """Rows-per-lane bin boundary and cooperative-job ratio of the global DP (see plgpu.h)."""
        self.lib.pl_engine_set_tuning(self.h, int(r4_rows), float(coop_ratio))

    def tuning(self):
        r, c = C.c_int32(), C.c_double()
        self.lib.pl_engine_get_tuning(self.h, C.byref(r), C.byref(c))
        return {"r4_rows": r.value, "coop_ratio": c.value}

    def last_plan(self):
        w, c, d = C.c_int32(), C.c_int32(), C.c_int32()
        self.lib.pl_engine_last_plan(self.h, C.byref(w), C.byref(c), C.byref(d))
        return {"waves": w.value, "coop": c.value, "dp_launches": d.value}

    def align_host(self, opt, pairs, ss=None):
        """pairs: list of (nt bytes, protein bytes); ss: None or list of (bytes|None).
        Returns a list of (score, cigar words, width)."""
        n = len(pairs)
        jobs = (SpliceJob * n)()
        nt_parts, aa_parts, ss_parts = [], [], []
        pos_nt = pos_aa = 0
        prot_off = {}  # one copy of each protein: jobs that share it (both strands) can run as int16x2 pairs
        for q, (nt, aa) in enumerate(pairs):
            if aa not in prot_off:
                prot_off[aa] = pos_aa
                aa_parts.append(aa)
                pos_aa += len(aa)
            jobs[q].nt_off, jobs[q].aa_off, jobs[q].nl, jobs[q].al = pos_nt, prot_off[aa], len(nt), len(aa)
            s = ss[q] if ss is not None else None
            jobs[q].ss_off = pos_nt if s is not None else -1
            nt_parts.append(nt)
            ss_parts.append(s if s is not None else bytes(len(nt)))
            pos_nt += len(nt)
        ntb = np.frombuffer(b"".join(nt_parts), dtype=np.uint8)
        aab = np.frombuffer(b"".join(aa_parts), dtype=np.uint8)
        ssb = np.frombuffer(b"".join(ss_parts), dtype=np.uint8) if ss is not None else None
        cap = sum(len(a) + len(b) + 8 for a, b in pairs)
        cig = np.zeros(max(cap, 1), dtype=np.uint32)
        res = (SpliceResult * n)()
        ok = self.lib.pl_splice_batch_host(self.h, opt.ptr, jobs, n, ntb.ctypes.data, ntb.size, aab.ctypes.data,
                                           aab.size, ssb.ctypes.data if ssb is not None else None,
                                           ssb.size if ssb is not None else 0, res, cig.ctypes.data, cig.size)
        if not ok:
            raise RuntimeError("pl_splice_batch_host failed: " + error())
        out = []
        for q in range(n):
            r = res[q]
            if r.status != 0:
                raise RuntimeError(f"job {q}: status {r.status}")
            out.append((r.score, cig[r.cigar_off:r.cigar_off + r.n_cigar].tolist(), r.mode))
        return out


    def ext_host(self, opt, reqs):
        """Batched extension DP through pl_ext_batch_host.  reqs: list of dicts with
        keys nt, aa (bytes), flag (NS_F_EXT_LEFT/RIGHT or 0), optional ss (bytes),
        pssm (al x 22 int8 array) and width (8/16, default: this host's rule).
        Returns a list of (score, nt_len, aa_len)."""
        n = len(reqs)
        jobs = (ExtJob * n)()
        nt_parts, aa_parts, ss_parts, ps_parts = [], [], [], []
        pn = pa = pss = pps = 0
        for q, r in enumerate(reqs):
            nt, aa = r["nt"], r["aa"]
            j = jobs[q]
            j.nt_off, j.aa_off, j.nl, j.al = pn, pa, len(nt), len(aa)
            j.flag, j.width = r.get("flag", 0), r.get("width", 0)
            j.ss_off = j.pssm_off = -1
            nt_parts.append(nt)
            aa_parts.append(aa)
            pn += len(nt)
            pa += len(aa)
            if r.get("ss") is not None:
                j.ss_off = pss
                ss_parts.append(bytes(r["ss"]))
                pss += len(r["ss"])
            if r.get("pssm") is not None:
                m = np.ascontiguousarray(r["pssm"], dtype=np.int8).reshape(-1)
                j.pssm_off = pps
                ps_parts.append(m.tobytes())
                pps += m.size
        ntb = np.frombuffer(b"".join(nt_parts) or b"\0", dtype=np.uint8)
        aab = np.frombuffer(b"".join(aa_parts) or b"\0", dtype=np.uint8)
        ssb = np.frombuffer(b"".join(ss_parts), dtype=np.uint8) if ss_parts else None
        psb = np.frombuffer(b"".join(ps_parts), dtype=np.int8) if ps_parts else None
        res = (ExtResult * max(n, 1))()
        ok = self.lib.pl_ext_batch_host(self.h, opt.ptr, jobs, n, ntb.ctypes.data, ntb.size, aab.ctypes.data,
                                        aab.size, ssb.ctypes.data if ssb is not None else None,
                                        ssb.size if ssb is not None else 0,
                                        psb.ctypes.data if psb is not None else None,
                                        psb.size if psb is not None else 0, res)
        if not ok:
            raise RuntimeError("pl_ext_batch_host failed: " + error())
        out = []
        for q in range(n):
            if res[q].status != 0:
                raise RuntimeError(f"ext job {q}: status {res[q].status}")
            out.append((res[q].score, res[q].nt_len, res[q].aa_len))
        return out

    def ext_last_cells(self):
        a, b = C.c_int64(), C.c_int64()
        self.lib.pl_ext_last_cells(self.h, C.byref(a), C.byref(b))
        return a.value, b.value


    def hmm_score(self, profile: "HmmProfile", regions):
        """Integer profile DP of each region (nt4 code arrays) against one profile: list of int scores."""
        n = len(regions)
        lens = np.array([len(r) for r in regions], dtype=np.int32)
        offs = np.zeros(n, dtype=np.int32)
        if n > 1:
            offs[1:] = np.cumsum(lens[:-1])
        nt = np.concatenate([np.asarray(r, dtype=np.uint8) for r in regions]) if n else np.zeros(0, np.uint8)
        nt = np.ascontiguousarray(nt if nt.size else np.zeros(1, np.uint8))
        score = np.zeros(max(n, 1), dtype=np.int32)
        if not self.lib.pl_hmm_score_host(self.h, profile.h, n, nt.ctypes.data, int(lens.sum()), offs.ctypes.data,
                                          lens.ctypes.data, score.ctypes.data):
            raise RuntimeError("pl_hmm_score_host failed: " + error())
        return score[:n].tolist()

    def hmm_score_many(self, profiles, regions) -> np.ndarray:
        """pl_hmm_score_many_device: every profile against one region set (nt4 code arrays);
        returns an int32 array [profile, region]."""
        import torch
        n = len(regions)
        lens = np.array([len(r) for r in regions], dtype=np.int32)
        offs = np.zeros(n, dtype=np.int32)
        if n > 1:
            offs[1:] = np.cumsum(lens[:-1])
        nt = np.concatenate([np.asarray(r, dtype=np.uint8) for r in regions]) if n else np.zeros(1, np.uint8)
        d_nt = torch.from_numpy(np.ascontiguousarray(nt)).to("cuda")
        d_sc = torch.zeros(max(1, len(profiles) * n), dtype=torch.int32, device="cuda")
        handles = (C.c_void_p * len(profiles))(*[p.h for p in profiles])
        if not self.lib.pl_hmm_score_many_device(self.h, handles, len(profiles), n, d_nt.data_ptr(), offs.ctypes.data,
                                                 lens.ctypes.data, d_sc.data_ptr(), None):
            raise RuntimeError("pl_hmm_score_many_device failed: " + error())
        return d_sc.cpu().numpy()[: len(profiles) * n].reshape(len(profiles), n)

    def gapless_score(self, w: dict, block_width: int, kmer: int, xdrop: int, mat, codon) -> np.ndarray:
        """pl_gapless_score_host on workload dict w: one int32 score per candidate."""
        args, keep = gapless_args(w, block_width, kmer, xdrop, mat, codon)
        sc = np.zeros(len(w["candidates"]), dtype=np.int32)
        if not self.lib.pl_gapless_score_host(self.h, *args, sc.ctypes.data):
            raise RuntimeError("pl_gapless_score_host failed: " + error())
        return sc


    def rc_score(self, profiles, peptides, do_null2: bool = True):
        """Recheck Forward scores.  profiles: list of RcProfile; peptides: list of (profile index,
        residue-code array).  Returns (bits, bias) float32 arrays."""
        n = len(peptides)
        pid = np.array([p for p, _ in peptides], dtype=np.int32)
        lens = np.array([len(d) for _, d in peptides], dtype=np.int32)
        offs = np.zeros(n, dtype=np.int64)
        if n > 1:
            offs[1:] = np.cumsum(lens[:-1])
        dsq = np.ascontiguousarray(np.concatenate([np.asarray(d, dtype=np.uint8) for _, d in peptides]))
        handles = (C.c_void_p * len(profiles))(*[p.h for p in profiles])
        bits = np.zeros(n, dtype=np.float32)
        bias = np.zeros(n, dtype=np.float32)
        if not self.lib.pl_rc_score_host(self.h, handles, len(profiles), n, pid.ctypes.data, dsq.ctypes.data, dsq.size,
                                         offs.ctypes.data, lens.ctypes.data, int(do_null2), bits.ctypes.data,
                                         bias.ctypes.data):
            raise RuntimeError("pl_rc_score_host failed: " + error())
        return bits, bias


class SeedOpt(C.Structure):
    """pl_seed_opt_t"""
    _fields_ = [("max_occ", C.c_int32), ("repeat_cap", C.c_int32), ("anchor_budget", C.c_int64),
                ("qname_hash", C.c_void_p)]


class SeedHmm(C.Structure):
    """pl_seed_hmm_t"""
    _fields_ = [("emit", C.c_void_p), ("n_state", C.c_int64), ("e_off", C.c_void_p), ("e_len", C.c_void_p),
                ("pos_loss", C.c_int32), ("win_loss", C.c_int32), ("seed_max", C.c_int32), ("pad", C.c_int32)]


class SeedIndex:
    """A pl_seed_index_t: the mapper's k-mer index (ki int64 bucket starts, kb uint32 block ids) on a device."""

    def __init__(self, ki, kb, kmer: int, mod_bit: int, device: int = 0):
        self.lib = load()
        ki = np.ascontiguousarray(ki, dtype=np.int64)
        kb = np.ascontiguousarray(kb, dtype=np.uint32)
        self.h = self.lib.pl_seed_index_create(device, ki.ctypes.data, ki.size, kb.ctypes.data, kb.size, kmer, mod_bit)
        if not self.h:
            raise RuntimeError("pl_seed_index_create: " + error())

    def close(self):
        if self.h:
            self.lib.pl_seed_index_destroy(self.h)
            self.h = None


def seed_anchors(eng, index: SeedIndex, proteins, max_occ: int, repeat_cap: int = 0, budget: int = 0, names=None,
                 profiles=None, pos_loss: int = 6, win_loss: int = 8, seed_max: int = 16):
    """Anchors of a list of proteins (bytes) through pl_seed_anchors_opt_host: a list of sorted uint64 arrays.
    repeat_cap > 0: the accuracy mode's repeat rescue, with the proteins' names (bytes).
    profiles: per protein its profile's match emissions (m x 20 int16, HMMER column order), the
    proteins their consensus: HMM-profile queries through pl_seed_anchors_hmm_host, with the
    profile-derived seeds' options (hmm_seed_pos_loss, hmm_seed_win_loss, hmm_seed_max)."""
    n = len(proteins)
    hmm = None
    if profiles is not None:
        if len(profiles) != n:
            raise ValueError("one profile per protein")
        tabs = [np.ascontiguousarray(e, dtype=np.int16).reshape(-1, 20) for e in profiles]
        e_len = np.array([t.shape[0] for t in tabs], dtype=np.int32)
        e_off = np.zeros(n, dtype=np.int64)
        if n > 1:
            e_off[1:] = np.cumsum(e_len[:-1])
        emit = np.ascontiguousarray(np.concatenate(tabs) if n and e_len.sum() else np.zeros((1, 20), np.int16))
        hmm = SeedHmm(emit.ctypes.data, int(e_len.sum()), e_off.ctypes.data, e_len.ctypes.data, pos_loss, win_loss,
                      seed_max, 0)
    qh = np.array([eng.lib.pl_seed_qname_hash(nm) for nm in (names or [b""] * n)], dtype=np.uint32)
    opt = SeedOpt(max_occ, repeat_cap, budget, qh.ctypes.data if n else None)
    lens = np.array([len(p) for p in proteins], dtype=np.int32)
    offs = np.zeros(n, dtype=np.int64)
    if n > 1:
        offs[1:] = np.cumsum(lens[:-1])
    seq = np.frombuffer(b"".join(proteins), dtype=np.uint8) if n else np.zeros(1, np.uint8)
    seq = np.ascontiguousarray(seq if seq.size else np.zeros(1, np.uint8))
    a_off = np.zeros(n + 1, dtype=np.int64)
    cap = 1 << 20
    for _ in range(2):
        a = np.zeros(max(cap, 1), dtype=np.uint64)
        if hmm is None:
            tot = eng.lib.pl_seed_anchors_opt_host(eng.h, index.h, n, seq.ctypes.data, int(lens.sum()),
                                                   offs.ctypes.data, lens.ctypes.data, C.byref(opt),
                                                   a_off.ctypes.data, a.ctypes.data, cap)
        else:
            tot = eng.lib.pl_seed_anchors_hmm_host(eng.h, index.h, n, seq.ctypes.data, int(lens.sum()),
                                                   offs.ctypes.data, lens.ctypes.data, C.byref(opt), C.byref(hmm),
                                                   a_off.ctypes.data, a.ctypes.data, cap)
        if tot < 0:
            raise RuntimeError("pl_seed_anchors_host: " + error())
        if tot <= cap:
            return [a[a_off[q]:a_off[q + 1]].copy() for q in range(n)]
        cap = int(tot)
    raise RuntimeError("pl_seed_anchors_host: capacity")


class RcProfile:
    """A pl_rc_profile_t: recheck's search profile (msc M x 21, tsc M x 8, float32) on a device."""

    def __init__(self, msc, tsc, device: int = 0):
        self.lib = load()
        m = np.ascontiguousarray(msc, dtype=np.float32).reshape(-1, 21)
        t = np.ascontiguousarray(tsc, dtype=np.float32).reshape(-1, 8)
        self.M = m.shape[0]
        self.h = self.lib.pl_rc_profile_create(device, self.M, m.ctypes.data, t.ctypes.data)
        if not self.h:
            raise RuntimeError("pl_rc_profile_create failed: " + error())

    def close(self):
        if self.h:
            self.lib.pl_rc_profile_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gapless_args(w: dict, block_width: int, kmer: int, xdrop: int, mat, codon):
    """The ns_gpu_gapless_score_batch argument list (after the engine) for workload dict w."""
    m = np.ascontiguousarray(mat, dtype=np.int8)
    cd = np.ascontiguousarray(codon, dtype=np.uint8)
    keep = (m, cd)
    args = [w["packed"].ctypes.data, int(w["bases"]), w["queries"].ctypes.data, int(w["queries"].size),
            w["candidates"].ctypes.data, len(w["candidates"]), w["anchors"].ctypes.data, len(w["anchors"]),
            block_width, kmer, xdrop, m.ctypes.data, int(round(m.size ** 0.5)), cd.ctypes.data]
    return args, keep


def gapless_reference_entry(w: dict, block_width: int, kmer: int, xdrop: int, mat, codon) -> np.ndarray:
    """ns_gpu_gapless_score_batch (the reference's entry point; needs gpu_init first)."""
    args, keep = gapless_args(w, block_width, kmer, xdrop, mat, codon)
    sc = np.zeros(len(w["candidates"]), dtype=np.int32)
    if not load().ns_gpu_gapless_score_batch(*args, sc.ctypes.data):
        raise RuntimeError("ns_gpu_gapless_score_batch failed: " + load().ns_gpu_error().decode())
    return sc


class HmmProfile:
    """A pl_hmm_profile_t: the reference parser's tables (emit m x 20, trans m x 7, HMMER order) on a device."""

    def __init__(self, emit, trans, codon_alpha, device: int = 0):
        self.lib = load()
        e = np.ascontiguousarray(emit, dtype=np.int16).reshape(-1, 20)
        t = np.ascontiguousarray(trans, dtype=np.int16).reshape(-1, 7)
        c = np.ascontiguousarray(codon_alpha, dtype=np.uint8)
        self.m = e.shape[0]
        self.h = self.lib.pl_hmm_profile_create(device, self.m, e.ctypes.data, t.ctypes.data, c.ctypes.data)
        if not self.h:
            raise RuntimeError("pl_hmm_profile_create failed: " + error())

    def close(self):
        if self.h:
            self.lib.pl_hmm_profile_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ext_stripe_width(opt, al: int) -> int:
    return int(load().pl_ext_stripe_width(opt.ptr, al))


class ExtBatch:
    """The reference's batch object (ns_ext_batch_*): add / flush / ready / wait / get."""

    def __init__(self):
        self.lib = load()
        self.h = self.lib.ns_ext_batch_init(None)
        if not self.h:
            raise RuntimeError("ns_ext_batch_init returned NULL: " + error())
        self._keep = []

    def add(self, nt: bytes, aa: bytes, opt, ss: bytes | None = None) -> int:
        ntb, aab = C.create_string_buffer(nt, len(nt)), C.create_string_buffer(aa, len(aa))
        ssb = C.create_string_buffer(bytes(ss), len(ss)) if ss is not None else None
        self._keep += [ntb, aab, ssb, opt]  # inputs must stay valid until fetched (nasw.h:201-202)
        return self.lib.ns_ext_batch_add(self.h, ntb, len(nt), aab, len(aa), opt.ptr, ssb)

    def flush(self) -> int:
        return self.lib.ns_ext_batch_flush(self.h)

    def ready(self, rid: int) -> bool:
        return bool(self.lib.ns_ext_batch_ready(self.h, rid))

    def wait(self):
        self.lib.ns_ext_batch_wait(self.h)

    def get(self, rid: int):
        p = self.lib.ns_ext_batch_get(self.h, rid)
        if not p:
            raise RuntimeError(f"extension request {rid} failed: " + self.lib.ns_gpu_error().decode())
        r = p.contents
        return (r.score, r.nt_len, r.aa_len)

    def close(self):
        if self.h:
            self.lib.ns_ext_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def group_plan(jobs, n_devices: int):
    """pl_group_plan over a SpliceJob array: (device slot of each job, DP cells per slot)."""
    n = len(jobs)
    dev = np.zeros(max(n, 1), np.int32)
    cells = np.zeros(n_devices, np.int64)
    if not load().pl_group_plan(jobs, n, n_devices, dev.ctypes.data, cells.ctypes.data):
        raise RuntimeError("pl_group_plan: " + error())
    return dev[:n], cells


def group_gather(dev_of_job, per_device, cigar_cap: int | None = None):
    """pl_group_gather: per_device[d] = (list of (score, cigar words) in the order of slot d's
    jobs).  Returns (SpliceResult array in job order, dense CIGAR words, total words)."""
    n = len(dev_of_job)
    n_dev = len(per_device)
    keep = []
    res_ptrs = (C.c_void_p * n_dev)()
    cig_ptrs = (C.c_void_p * n_dev)()
    for d, items in enumerate(per_device):
        r = (SpliceResult * max(len(items), 1))()
        words, off = [], 0
        for k, (score, cig) in enumerate(items):
            r[k].score, r[k].n_cigar, r[k].cigar_off, r[k].mode, r[k].status = score, len(cig), off, 16, 0
            words += list(cig)
            off += len(cig)
        w = np.array(words + [0], np.uint32)
        keep += [r, w]
        res_ptrs[d] = C.cast(r, C.c_void_p)
        cig_ptrs[d] = w.ctypes.data
    cap = cigar_cap if cigar_cap is not None else sum(len(c) for items in per_device for _, c in items)
    out = (SpliceResult * max(n, 1))()
    cig = np.zeros(max(cap, 1), np.uint32)
    total = C.c_int64()
    dv = np.ascontiguousarray(dev_of_job, np.int32)
    if not load().pl_group_gather(n, dv.ctypes.data, n_dev, res_ptrs, cig_ptrs, out, cig.ctypes.data, cap,
                                  C.byref(total)):
        raise RuntimeError("pl_group_gather: " + error())
    return out, cig, total.value


def measure_int_peak(device: int = 0):
    """Measured integer-pipe lane-op rates (int32, int16x2) of the device."""
    a, b = C.c_double(), C.c_double()
    if not load().pl_measure_int_peak(device, C.byref(a), C.byref(b)):
        raise RuntimeError("pl_measure_int_peak failed")
    return a.value, b.value


def gpu_init(device: int = 0) -> bool:
    return bool(load().ns_gpu_init(device))


def gpu_global(ns: bytes, aa: bytes, opt, ss: bytes | None = None):
    """ns_gpu_global(): returns (ok, score, nt_len, aa_len, cigar words)."""
    lib = load()
    r = NsRst()
    ssb = C.create_string_buffer(bytes(ss), len(ss)) if ss is not None else None
    ok = lib.ns_gpu_global(None, ns, len(ns), aa, len(aa), opt.ptr, ssb, C.byref(r))
    cig = [r.cigar[k] for k in range(r.n_cigar)] if ok and r.n_cigar else []
    if r.cigar:
        _libc.free(C.cast(r.cigar, C.c_void_p))
    return bool(ok), r.score, r.nt_len, r.aa_len, cig
