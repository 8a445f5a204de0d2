"""ctypes binding of libkira_gpu.so (include/kira_gpu.h).

Loading is strict: if the library is missing or cannot be loaded the import
raises, so no caller can silently run anything but the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libkira_gpu.so")

KIRA_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "NotBuilt", 2: "Driver", 3: "Runtime", 4: "NoDevice", 5: "ReadTooLong",
    6: "Timeout", 7: "Invalid", 8: "OutOfMemory", 9: "Capacity", 10: "ScratchLimit",
    11: "Pending",
}
KIRA_ERR_TIMEOUT = 6
KIRA_ERR_SCRATCH_LIMIT = 10
KIRA_PENDING = 11
KIRA_PAIR_SW = 3
KIRA_PAIR_OUT_OF_BOUNDS = 4
NOALLOC_SCRATCH_BYTES = 32 << 20
PAIR_PENDING, PAIR_CERTIFIED, PAIR_MYERS_REJECT, PAIR_SW = 0, 1, 2, 3
READ_BYTES_MAX = 64
ABORT_DISABLED = -268435456  # i32::MIN / 8
INT32_MAX = 2**31 - 1

# Every symbol include/kira_gpu.h declares.
EXPORTS = (
    "kira_gpu_is_available", "kira_gpu_init", "kira_gpu_destroy", "kira_gpu_last_error",
    "kira_gpu_arena_bytes", "kira_gpu_sieve_batch", "kira_gpu_ref_upload",
    "kira_gpu_myers_batch", "kira_gpu_bsw_batch", "kira_gpu_verify_batch",
    "kira_gpu_verify_dev", "kira_gpu_profile", "kira_gpu_stage_times",
    "kira_gpu_bsw_shapes", "kira_gpu_set_bsw_shape", "kira_gpu_bsw_batch_noalloc",
    "kira_gpu_align_batch_simd", "kira_gpu_set_plain", "kira_gpu_set_trace_budget",
    "kira_gpu_set_graphs", "kira_gpu_set_chunk_pairs", "kira_gpu_nm_md", "kira_gpu_wfa_batch",
    "kira_gpu_set_wfa_lanes", "kira_gpu_prefilter_batch", "kira_gpu_exact_match_batch",
    "kira_server_create", "kira_server_destroy", "kira_server_ref_upload",
    "kira_server_submit_verify", "kira_server_submit_bsw", "kira_server_poll",
    "kira_server_wait", "kira_server_info", "kira_server_release", "kira_server_stats",
    "kira_server_last_error", "kira_server_profile", "kira_gpu_launch_count",
    "kira_gpu_alu_probe", "kira_gpu_verify_batch_compact", "kira_gpu_bsw_rounds",
)
SIMD_SCALAR, SIMD_AVX2, SIMD_AVX_VNNI, SIMD_NEON = 0, 1, 2, 3
VERIFY_NO_QGRAM = 1
STAGES = ("sieve_certify", "myers", "bsw_dp", "bsw_traceback", "cigar_compact")


class SieveJob(C.Structure):
    _fields_ = [("read_packed", C.c_void_p), ("read_bytes", C.c_uint32),
                ("read_nucs", C.c_uint32), ("ref_packed", C.c_void_p),
                ("ref_bytes", C.c_uint32), ("ref_nucs", C.c_uint32),
                ("max_mismatches", C.c_uint32)]


class SieveResult(C.Structure):
    _fields_ = [("shift", C.c_int32), ("mismatches", C.c_int32),
                ("second_mismatches", C.c_int32)]


class Pairs(C.Structure):
    _fields_ = [("n", C.c_uint32), ("max_read_len", C.c_uint32), ("max_win_len", C.c_uint32),
                ("max_bandwidth", C.c_uint32), ("read_seq", C.c_void_p),
                ("read_seq_bytes", C.c_uint64), ("read_off", C.c_void_p),
                ("read_len", C.c_void_p), ("win_seq", C.c_void_p),
                ("win_seq_bytes", C.c_uint64), ("win_off", C.c_void_p),
                ("win_len", C.c_void_p), ("band_offset", C.c_void_p),
                ("abort_score", C.c_void_p), ("bandwidth", C.c_void_p)]


class SwCfg(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("match_score", "mismatch", "gap_open", "gap_extend", "bandwidth", "xdrop",
                 "clip_penalty", "adaptive", "max_drift", "dp_xdrop")]


class VerifyParams(C.Structure):
    _fields_ = [("sw", SwCfg), ("sieve_threshold", C.c_int32), ("myers_k", C.c_int32),
                ("cert_strict", C.c_int32), ("flags", C.c_int32)]


class WfaParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("mismatch", "gap_open", "gap_extend", "match_score", "scored", "max_score",
                 "budget_pct", "adaptive_drop", "text_begin_free", "traceback")]


class Chain(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("ref_start", "ref_end", "read_start", "read_end")]


class PrefilterCfg(C.Structure):
    _fields_ = [("match_score", C.c_int32), ("mismatch", C.c_int32), ("xdrop", C.c_int32),
                ("accept_enable", C.c_int32), ("accept_only_top1", C.c_int32),
                ("accept_span_slack", C.c_uint32), ("accept_min_identity", C.c_float),
                ("accept_max_mismatches", C.c_uint32),
                ("accept_require_score_margin", C.c_int32),
                ("long_read_threshold", C.c_uint32), ("multi_alignments_enabled", C.c_int32),
                ("tail", C.c_int32), ("min_identity_x10000", C.c_int32),
                ("exact_first", C.c_int32)]


class ServerCfg(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("max_batch_pairs", C.c_uint32),
                ("mem_fraction", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("n_pairs", C.c_uint32), ("cigar_used", C.c_uint64),
                ("t_submit_ns", C.c_int64), ("t_start_ns", C.c_int64), ("t_done_ns", C.c_int64),
                ("batch_id", C.c_uint64), ("batch_requests", C.c_uint32),
                ("reserved", C.c_uint32)]


class CigarBuf(C.Structure):
    _fields_ = [("ops", C.c_void_p), ("cap", C.c_uint64), ("used", C.c_uint64)]


SW_RESULT_DTYPE = np.dtype([("score", "<i4"), ("ref_start", "<u4"), ("ref_end", "<u4"),
                            ("read_start", "<i4"), ("read_end", "<i4"), ("cigar_off", "<u4"),
                            ("n_cigar", "<u4"), ("status", "u1"), ("early_abort", "u1"),
                            ("reserved", "<u2")])
DETAIL_DTYPE = np.dtype([("sieve_shift", "<i4"), ("sieve_mism", "<i4"),
                         ("sieve_second", "<i4"), ("myers_dist", "<i4"), ("myers_end", "<i4")])
WFA_RESULT_DTYPE = np.dtype([("cost", "<i4"), ("score", "<i4"), ("text_start", "<u4"),
                             ("text_end", "<u4"), ("cigar_off", "<u4"), ("n_cigar", "<u4"),
                             ("found", "<u4"), ("reserved", "<u4")])
assert SW_RESULT_DTYPE.itemsize == 32 and DETAIL_DTYPE.itemsize == 20
assert WFA_RESULT_DTYPE.itemsize == 32
PREFILTER_RESULT_DTYPE = np.dtype([("result", "u1"), ("reason", "u1"), ("other", "u1"),
                                   ("has_metrics", "u1"), ("len", "<u2"), ("mism", "<u2"),
                                   ("matches", "<u2"), ("identity_x10000", "<u2"),
                                   ("score", "<i4"), ("read_start", "<u4"), ("ref_start", "<u4"),
                                   ("nm", "<u4"), ("cigar_off", "<u4"), ("n_cigar", "<u4"),
                                   ("md_off", "<u4"), ("md_len", "<u4"), ("reserved", "<u4")])
CHAIN_DTYPE = np.dtype([("ref_start", "<u4"), ("ref_end", "<u4"), ("read_start", "<u4"),
                        ("read_end", "<u4")])
assert PREFILTER_RESULT_DTYPE.itemsize == 48 and CHAIN_DTYPE.itemsize == 16
PREFILTER_ACCEPT, PREFILTER_REJECT, PREFILTER_FALLBACK, PREFILTER_EXACT = 0, 1, 2, 3

_lib = None


def lib():
    """Load libkira_gpu.so; raises when it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m kira_ls_aligner_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.kira_gpu_is_available.restype = C.c_int
    L.kira_gpu_init.argtypes = [C.c_int, C.POINTER(vp)]
    L.kira_gpu_destroy.argtypes = [vp]
    L.kira_gpu_destroy.restype = None
    L.kira_gpu_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.kira_gpu_arena_bytes.argtypes = [vp]
    L.kira_gpu_arena_bytes.restype = C.c_uint64
    L.kira_gpu_sieve_batch.argtypes = [vp, C.POINTER(SieveJob), C.c_uint32,
                                       C.POINTER(SieveResult)]
    L.kira_gpu_ref_upload.argtypes = [vp, vp, C.c_uint64]
    L.kira_gpu_myers_batch.argtypes = [vp, C.POINTER(Pairs), C.c_uint32, vp, vp]
    L.kira_gpu_bsw_batch.argtypes = [vp, C.POINTER(Pairs), C.POINTER(SwCfg), vp,
                                     C.POINTER(CigarBuf), C.POINTER(C.c_uint64)]
    L.kira_gpu_verify_batch.argtypes = [vp, C.POINTER(Pairs), C.POINTER(VerifyParams), vp,
                                        C.POINTER(CigarBuf), vp, C.POINTER(C.c_uint64)]
    L.kira_gpu_verify_batch_compact.argtypes = [vp, C.POINTER(Pairs), C.POINTER(VerifyParams),
                                                vp, vp, C.c_uint64, C.POINTER(C.c_uint64),
                                                C.POINTER(CigarBuf), C.POINTER(C.c_uint64)]
    L.kira_gpu_verify_dev.argtypes = [vp, C.POINTER(Pairs), C.POINTER(VerifyParams), vp, vp,
                                      C.c_uint64, vp, vp, vp, vp]
    L.kira_gpu_profile.argtypes = [vp, C.c_int]
    L.kira_gpu_bsw_shapes.argtypes = [vp, vp, vp, C.c_int]
    L.kira_gpu_set_plain.argtypes = [vp, C.c_int]
    L.kira_gpu_set_trace_budget.argtypes = [vp, C.c_uint64]
    L.kira_gpu_set_graphs.argtypes = [vp, C.c_int, vp, vp]
    L.kira_gpu_set_chunk_pairs.argtypes = [vp, C.c_int64]
    L.kira_gpu_nm_md.argtypes = [vp, C.POINTER(Pairs), vp, vp, C.c_uint64, vp, vp, vp,
                                 C.c_uint64, C.POINTER(C.c_uint64)]
    L.kira_gpu_wfa_batch.argtypes = [vp, C.POINTER(Pairs), C.POINTER(WfaParams), vp, vp, vp,
                                     C.POINTER(CigarBuf)]
    L.kira_gpu_set_wfa_lanes.argtypes = [vp, C.c_int]
    L.kira_gpu_prefilter_batch.argtypes = [vp, C.POINTER(Pairs), vp, vp, vp,
                                           C.POINTER(PrefilterCfg), vp, C.POINTER(CigarBuf), vp,
                                           C.c_uint64, C.POINTER(C.c_uint64)]
    L.kira_gpu_exact_match_batch.argtypes = [vp, C.POINTER(Pairs), vp, vp]
    L.kira_gpu_align_batch_simd.argtypes = [vp, C.POINTER(Pairs), C.POINTER(SwCfg), C.c_int,
                                            C.c_int, vp, C.POINTER(CigarBuf)]
    L.kira_gpu_bsw_batch_noalloc.argtypes = [C.POINTER(Pairs), C.POINTER(SwCfg), vp, vp,
                                             C.c_uint64, vp, vp]
    L.kira_gpu_set_bsw_shape.argtypes = [vp, C.c_uint32, C.c_int]
    L.kira_gpu_stage_times.argtypes = [vp, C.POINTER(C.c_float), C.c_int]
    L.kira_server_create.argtypes = [C.POINTER(ServerCfg), C.POINTER(vp)]
    L.kira_server_destroy.argtypes = [vp]
    L.kira_server_destroy.restype = None
    L.kira_server_ref_upload.argtypes = [vp, vp, C.c_uint64]
    L.kira_server_submit_verify.argtypes = [vp, C.POINTER(Pairs), C.POINTER(VerifyParams), vp,
                                            vp, C.c_uint64, C.POINTER(C.c_uint64)]
    L.kira_server_submit_bsw.argtypes = [vp, C.POINTER(Pairs), C.POINTER(SwCfg), vp, vp,
                                         C.c_uint64, C.POINTER(C.c_uint64)]
    L.kira_server_poll.argtypes = [vp, C.c_uint64]
    L.kira_server_wait.argtypes = [vp, C.c_uint64, C.c_int64]
    L.kira_server_info.argtypes = [vp, C.c_uint64, C.POINTER(RequestInfo)]
    L.kira_server_release.argtypes = [vp, C.c_uint64]
    L.kira_server_stats.argtypes = [vp, vp, vp, vp]
    L.kira_server_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.kira_server_profile.argtypes = [vp, C.POINTER(C.c_double)]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or C.c_int
    L.kira_gpu_destroy.restype = None
    L.kira_server_destroy.restype = None
    L.kira_gpu_arena_bytes.restype = C.c_uint64
    L.kira_gpu_launch_count.argtypes = []
    L.kira_gpu_launch_count.restype = C.c_uint64
    L.kira_gpu_bsw_rounds.argtypes = [vp]
    L.kira_gpu_bsw_rounds.restype = C.c_uint32
    L.kira_gpu_alu_probe.argtypes = [C.c_int, C.c_int, C.c_uint32, C.POINTER(C.c_double)]
    _lib = L
    return L


def ptr(a) -> int | None:
    """Address of a numpy array / torch tensor (None for None)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
