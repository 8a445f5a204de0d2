"""ctypes binding of the CPU oracle (``oracle/lib/libkira_oracle.so``).

Test infrastructure only: the parity checker for the CUDA library and the timed
CPU baseline of ``bench.py``. The product package never imports this module.

The C functions restate kira-ls-aligner v0.8.3:
``src/alignment/bitpacked.rs``, ``src/alignment/myers.rs``,
``src/alignment/mod.rs:1331-2135``, ``src/alignment/sw_int8_vnni.rs``,
``src/alignment/mod.rs:688-776`` and ``src/alignment/router.rs:191-203``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libkira_oracle.so")

I32_MIN = -(2**31)
# i32::MIN / 8 (exact in Rust): the abort bound that disables the abort test.
ABORT_DISABLED = -268435456
OP_CHARS = "MIDNS"


class OrcCfg(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("match_score", "mismatch", "gap_open", "gap_extend", "bandwidth", "xdrop",
                 "clip_penalty")]


class OrcSwResult(C.Structure):
    _fields_ = [("ref_start", C.c_uint32), ("ref_end", C.c_uint32), ("read_start", C.c_int32),
                ("read_end", C.c_int32), ("score", C.c_int32), ("n_cigar", C.c_uint32),
                ("early_abort", C.c_uint32), ("pad", C.c_uint32), ("cells", C.c_uint64)]


class OrcVerifyParams(C.Structure):
    _fields_ = [("cfg", OrcCfg), ("sieve_threshold", C.c_int32), ("myers_k", C.c_int32),
                ("abort_score", C.c_int32), ("adaptive", C.c_int32), ("max_drift", C.c_int32),
                ("dp_xdrop", C.c_int32), ("cert_strict", C.c_int32)]


class OrcVerifyResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("sieve_shift", C.c_int32), ("sieve_mism", C.c_int32),
                ("sieve_second", C.c_int32), ("myers_dist", C.c_int32), ("myers_end", C.c_int32),
                ("sw", OrcSwResult)]


class OrcWfaCfg(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("mismatch", "gap_open", "gap_extend", "match_score", "scored", "max_score",
                 "adaptive_drop", "text_begin_free", "traceback")]


class OrcChain(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("ref_start", "ref_end", "read_start", "read_end")]


class OrcPrefilterCfg(C.Structure):
    _fields_ = [("match_score", C.c_int32), ("mismatch", C.c_int32), ("xdrop", C.c_int32),
                ("accept_enable", C.c_int32), ("accept_only_top1", C.c_int32),
                ("accept_span_slack", C.c_uint32), ("identity_floor", C.c_int32),
                ("accept_max_mismatches", C.c_uint32),
                ("accept_require_score_margin", C.c_int32),
                ("long_read_threshold", C.c_uint32), ("multi_alignments_enabled", C.c_int32),
                ("tail", C.c_int32), ("min_id_override", C.c_int32)]


class OrcPrefilterOut(C.Structure):
    _fields_ = [("result", C.c_int32), ("reason", C.c_int32), ("other", C.c_int32),
                ("has_metrics", C.c_int32), ("len", C.c_uint32), ("mism", C.c_uint32),
                ("matches", C.c_uint32), ("identity_x10000", C.c_uint32), ("score", C.c_int32),
                ("read_start", C.c_uint32), ("ref_start", C.c_uint32), ("nm", C.c_uint32),
                ("n_cigar", C.c_uint32), ("cigar", C.c_uint32 * 3)]


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", _HERE, "all"])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        u8p = C.POINTER(C.c_uint8)
        L.orc_pack.restype = C.c_int
        L.orc_pack.argtypes = [C.c_char_p, C.c_size_t, u8p]
        L.orc_shift_bits_right.argtypes = [C.c_char_p, C.c_size_t, C.c_int, u8p]
        L.orc_pre_shift.argtypes = [C.c_char_p, C.c_size_t, u8p]
        L.orc_mismatch_count.restype = C.c_size_t
        L.orc_mismatch_count.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t]
        L.orc_scan_best_with_second_raw.argtypes = [
            C.c_char_p, C.c_size_t, C.c_size_t, C.c_int, C.c_char_p, C.c_size_t, C.c_size_t,
            C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_scan.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t, C.c_int, C.c_char_p,
                               C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(C.c_int64),
                               C.POINTER(C.c_int64)]
        L.orc_gpu_sieve_semantics.argtypes = [C.c_char_p, C.c_uint32, C.c_char_p, C.c_uint32,
                                              C.c_uint32, C.POINTER(C.c_int32),
                                              C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_byte_scan.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_size_t,
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_nm_md.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_size_t,
                                C.c_size_t, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32),
                                C.c_char_p, C.c_uint32]
        L.orc_nm_md.restype = C.c_uint32
        L.orc_md_builder.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint32,
                                     C.POINTER(C.c_uint32), C.c_char_p, C.c_uint32]
        L.orc_md_builder.restype = C.c_uint32
        L.orc_myers.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_size_t, C.c_int,
                                C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.orc_banded_sw.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_int32,
                                    C.POINTER(OrcCfg), C.c_int32, C.c_int, C.c_int32, C.c_int32,
                                    C.POINTER(OrcSwResult), C.POINTER(C.c_uint32), C.c_uint32]
        L.orc_banded_sw_matrix.argtypes = [
            C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_int32, C.POINTER(OrcCfg),
            C.c_int32, C.c_int, C.c_int32, C.c_int32, C.POINTER(OrcSwResult),
            C.POINTER(C.c_uint32), C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_size_t]
        pp = C.POINTER(C.c_char_p)
        for name in ("orc_sw_batch_avx2", "orc_sw_batch_int8"):
            f = getattr(L, name)
            f.argtypes = [C.c_int, pp, pp, C.c_size_t, C.c_size_t, C.POINTER(C.c_int32),
                          C.POINTER(C.c_int32), C.POINTER(OrcCfg), C.c_int, C.c_int32, C.c_int32,
                          C.POINTER(OrcSwResult), C.POINTER(C.c_uint32), C.c_uint32]
        L.orc_sw_full_window_model.argtypes = [C.c_int, pp, pp, C.c_size_t, C.c_size_t,
                                               C.POINTER(C.c_int32), C.POINTER(OrcCfg), C.c_int,
                                               C.POINTER(OrcSwResult), C.POINTER(C.c_uint32),
                                               C.c_uint32]
        L.orc_int8_path_viable.argtypes = [C.c_size_t, C.POINTER(OrcCfg)]
        L.orc_align_batch_simd.argtypes = [C.c_int, pp, C.POINTER(C.c_uint32), pp,
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32), C.POINTER(OrcCfg), C.c_int,
                                           C.c_int, C.c_int, C.c_int32, C.c_int32,
                                           C.POINTER(OrcSwResult), C.POINTER(C.c_uint32),
                                           C.c_uint32]
        L.orc_spectral_certified.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t,
                                             C.c_int64, C.c_size_t, C.c_int]
        L.orc_spectral_max_mismatches.restype = C.c_size_t
        L.orc_spectral_max_mismatches.argtypes = [C.c_size_t]
        L.orc_myers_reject_bound.restype = C.c_size_t
        L.orc_myers_reject_bound.argtypes = [C.c_size_t]
        L.orc_verify_pair.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                      C.POINTER(OrcVerifyParams), C.POINTER(OrcVerifyResult),
                                      C.POINTER(C.c_uint32), C.c_uint32]
        vp = C.c_void_p
        L.orc_verify_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp,
                                       C.POINTER(OrcVerifyParams), C.c_int, vp, vp, C.c_uint32]
        L.orc_banded_sw_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp, vp,
                                          C.POINTER(OrcCfg), C.c_int32, C.c_int, C.c_int32,
                                          C.c_int32, C.c_int, vp, vp, C.c_uint32]
        L.orc_sw_avx2_batch.argtypes = [C.c_uint32, vp, vp, C.c_uint32, vp, vp, C.c_uint32,
                                        C.POINTER(OrcCfg), C.c_int, vp, vp, C.c_uint32]
        L.orc_myers_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_uint32, C.c_int,
                                      vp, vp]
        L.orc_sieve_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, vp]
        L.orc_prefilter.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                    C.POINTER(OrcChain), C.c_int, C.c_int32,
                                    C.POINTER(OrcPrefilterCfg), C.POINTER(OrcPrefilterOut),
                                    C.c_char_p, C.c_size_t]
        L.orc_prefilter_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          C.POINTER(OrcPrefilterCfg), C.c_int, C.c_int, vp, vp,
                                          C.c_uint32]
        L.orc_exact_match_exists.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                             C.POINTER(OrcChain)]
        L.orc_identical_nm.restype = C.c_uint32
        L.orc_identical_nm.argtypes = [C.c_char_p, C.c_size_t]
        L.orc_wfa.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                              C.POINTER(OrcWfaCfg), vp, vp, vp, vp, C.c_uint32, vp]
        L.orc_wfa_batch.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp, C.POINTER(OrcWfaCfg),
                                    C.c_int, vp, vp, vp, vp, vp, vp, C.c_uint32]
        _lib = L
    return _lib


# ---------------------------------------------------------------------------
# Python-shaped wrappers (mirror the reference function shapes)
# ---------------------------------------------------------------------------

def cfg(match_score=1, mismatch=4, gap_open=6, gap_extend=1, bandwidth=33, xdrop=100,
        clip_penalty=5) -> OrcCfg:
    return OrcCfg(match_score, mismatch, gap_open, gap_extend, bandwidth, xdrop, clip_penalty)


def pack(seq: bytes):
    """PackedDna::pack (bitpacked.rs:37-45) -> (bits, len, valid)."""
    out = (C.c_uint8 * max(1, (len(seq) + 3) // 4))()
    valid = lib().orc_pack(seq, len(seq), out)
    return bytes(out)[: (len(seq) + 3) // 4], len(seq), bool(valid)


def shift_bits_right(bits: bytes, off: int) -> bytes:
    out = (C.c_uint8 * max(1, len(bits)))()
    lib().orc_shift_bits_right(bits, len(bits), off, out)
    return bytes(out)[: len(bits)]


def pre_shift(bits: bytes):
    n = len(bits)
    out = (C.c_uint8 * max(1, 4 * n))()
    lib().orc_pre_shift(bits, n, out)
    raw = bytes(out)
    return [raw[p * n:(p + 1) * n] for p in range(4)]


def scan_best_with_second(read: bytes, text: bytes):
    """scan_best_with_second over PackedDna of both sequences -> None | (shift, mism, second|None)."""
    rb, rl, rv = pack(read)
    tb, tl, _ = pack(text)
    ph = b"".join(pre_shift(tb))
    s, m, sec = C.c_int64(), C.c_int64(), C.c_int64()
    ok = lib().orc_scan_best_with_second_raw(rb, len(rb), rl, int(rv), ph, len(tb), tl,
                                             C.byref(s), C.byref(m), C.byref(sec))
    if not ok:
        return None
    return s.value, m.value, (None if sec.value < 0 else sec.value)


def scan(read: bytes, text: bytes, max_mism: int):
    """bitpacked::scan (bitpacked.rs:122-133) -> None | (shift, mism)."""
    rb, rl, rv = pack(read)
    tb, tl, _ = pack(text)
    ph = b"".join(pre_shift(tb))
    s, m = C.c_int64(), C.c_int64()
    ok = lib().orc_scan(rb, len(rb), rl, int(rv), ph, len(tb), tl, max_mism, C.byref(s),
                        C.byref(m))
    return (s.value, m.value) if ok else None


def gpu_sieve_semantics(read_bits: bytes, read_nucs: int, ref_bits: bytes, ref_nucs: int,
                        max_mism: int):
    s, m, sec = C.c_int32(), C.c_int32(), C.c_int32()
    lib().orc_gpu_sieve_semantics(read_bits, read_nucs, ref_bits, ref_nucs, max_mism,
                                  C.byref(s), C.byref(m), C.byref(sec))
    return s.value, m.value, sec.value


def byte_scan(read: bytes, win: bytes, max_mism: int):
    s, m = C.c_int64(), C.c_int64()
    ok = lib().orc_byte_scan(read, len(read), win, len(win), max_mism, C.byref(s), C.byref(m))
    return (s.value, m.value) if ok else None


def bounded_edit_distance(pattern: bytes, text: bytes, max_k: int, path: int = 0):
    """myers::bounded_edit_distance (myers.rs:47-70) -> None | (dist, end)."""
    d, e = C.c_uint64(), C.c_uint64()
    ok = lib().orc_myers(pattern, len(pattern), text, len(text), max_k, path, C.byref(d),
                         C.byref(e))
    return (d.value, e.value) if ok else None


@dataclass
class SwRes:
    ref_start: int
    ref_end: int
    read_start: int
    read_end: int
    score: int
    cigar: list  # [(len, op_char)]
    early_abort: bool
    cells: int = 0

    def key(self):
        return (self.ref_start, self.ref_end, self.read_start, self.read_end, self.score,
                tuple(self.cigar), self.early_abort)

    def cigar_str(self) -> str:
        return "".join(f"{n}{c}" for n, c in self.cigar)


def decode_cigar(words) -> list:
    return [(int(w) >> 4, OP_CHARS[int(w) & 0xF]) for w in words]


def _swres(r: OrcSwResult, cig) -> SwRes:
    return SwRes(r.ref_start, r.ref_end, r.read_start, r.read_end, r.score,
                 decode_cigar(cig[: r.n_cigar]), bool(r.early_abort), r.cells)


def banded_sw(read: bytes, ref: bytes, offset: int, c: OrcCfg, abort_score=ABORT_DISABLED,
              adaptive=True, max_drift=16, dp_xdrop=None) -> SwRes:
    """banded_sw_with (mod.rs:1370-1650)."""
    cap = len(read) + len(ref) + 2
    cig = (C.c_uint32 * cap)()
    out = OrcSwResult()
    lib().orc_banded_sw(read, len(read), ref, len(ref), offset, C.byref(c), abort_score,
                        int(adaptive), max_drift, c.xdrop if dp_xdrop is None else dp_xdrop,
                        C.byref(out), cig, cap)
    return _swres(out, cig)


def _ptrs(seqs):
    arr = (C.c_char_p * len(seqs))()
    for i, s in enumerate(seqs):
        arr[i] = s
    return arr


def sw_batch(kind: str, reads, wins, c: OrcCfg, aborts=None, offsets=None, adaptive=True,
             max_drift=16, dp_xdrop=None):
    """Full-window batch kernels: kind in {"avx2", "int8", "model16", "model8"}."""
    n = len(reads)
    q, r = len(reads[0]), len(wins[0])
    cap = q + r + 2
    cig = (C.c_uint32 * (cap * n))()
    outs = (OrcSwResult * n)()
    ab = (C.c_int32 * n)(*(aborts if aborts is not None else [ABORT_DISABLED] * n))
    off = (C.c_int32 * n)(*(offsets if offsets is not None else [0] * n))
    L = lib()
    xd = c.xdrop if dp_xdrop is None else dp_xdrop
    if kind == "avx2":
        rc = L.orc_sw_batch_avx2(n, _ptrs(reads), _ptrs(wins), q, r, ab, off, C.byref(c),
                                 int(adaptive), max_drift, xd, outs, cig, cap)
    elif kind == "int8":
        rc = L.orc_sw_batch_int8(n, _ptrs(reads), _ptrs(wins), q, r, ab, off, C.byref(c),
                                 int(adaptive), max_drift, xd, outs, cig, cap)
    else:
        bits = 16 if kind == "model16" else 8
        rc = L.orc_sw_full_window_model(n, _ptrs(reads), _ptrs(wins), q, r, ab, C.byref(c), bits,
                                        outs, cig, cap)
    res = [_swres(outs[k], cig[k * cap:(k + 1) * cap]) for k in range(n)]
    return rc, res


SIMD_SCALAR, SIMD_AVX2, SIMD_VNNI, SIMD_NEON = 0, 1, 2, 3


def align_batch_simd(reads, wins, c: OrcCfg, mode: int, detected: int, aborts=None,
                     offsets=None, adaptive=True, max_drift=16, dp_xdrop=None):
    """align_batch_simd (mod.rs:1111-1169) SW results (before build_alignment)."""
    n = len(reads)
    if n == 0:
        return []
    cap = max(len(x) for x in reads) + max(len(x) for x in wins) + 2
    cig = (C.c_uint32 * (cap * n))()
    outs = (OrcSwResult * n)()
    ab = (C.c_int32 * n)(*(aborts if aborts is not None else [ABORT_DISABLED] * n))
    off = (C.c_int32 * n)(*(offsets if offsets is not None else [0] * n))
    rl = (C.c_uint32 * n)(*[len(x) for x in reads])
    wl = (C.c_uint32 * n)(*[len(x) for x in wins])
    lib().orc_align_batch_simd(n, _ptrs(reads), rl, _ptrs(wins), wl, ab, off, C.byref(c), mode,
                               detected, int(adaptive), max_drift,
                               c.xdrop if dp_xdrop is None else dp_xdrop, outs, cig, cap)
    return [_swres(outs[k], cig[k * cap:(k + 1) * cap]) for k in range(n)]


def int8_path_viable(read_len: int, c: OrcCfg) -> bool:
    return bool(lib().orc_int8_path_viable(read_len, C.byref(c)))


def cpu_has_avx2() -> bool:
    return bool(lib().orc_cpu_has_avx2())


def cpu_has_avx_vnni() -> bool:
    return bool(lib().orc_cpu_has_avx_vnni())


def spectral_certified(read: bytes, ref_aligned: bytes, mism: int, second, max_mism: int,
                       strict=False) -> bool:
    return bool(lib().orc_spectral_certified(read, ref_aligned, len(read), mism,
                                             -1 if second is None else second, max_mism,
                                             int(strict)))


def spectral_max_mismatches(n: int) -> int:
    return lib().orc_spectral_max_mismatches(n)


def myers_reject_bound(n: int) -> int:
    return lib().orc_myers_reject_bound(n)


def verify_params(c: OrcCfg, sieve_threshold=12, myers_k=8, abort_score=ABORT_DISABLED,
                  adaptive=True, max_drift=16, dp_xdrop=None, cert_strict=False):
    return OrcVerifyParams(c, sieve_threshold, myers_k, abort_score, int(adaptive), max_drift,
                           c.xdrop if dp_xdrop is None else dp_xdrop, int(cert_strict))


def verify_pair(read: bytes, win: bytes, p: OrcVerifyParams):
    cap = len(read) + len(win) + 2
    cig = (C.c_uint32 * cap)()
    out = OrcVerifyResult()
    lib().orc_verify_pair(read, len(read), win, len(win), C.byref(p), C.byref(out), cig, cap)
    return out, decode_cigar(cig[: out.sw.n_cigar])


VERIFY_DTYPE = np.dtype([("status", "<i4"), ("sieve_shift", "<i4"), ("sieve_mism", "<i4"),
                         ("sieve_second", "<i4"), ("myers_dist", "<i4"), ("myers_end", "<i4"),
                         ("ref_start", "<u4"), ("ref_end", "<u4"), ("read_start", "<i4"),
                         ("read_end", "<i4"), ("score", "<i4"), ("n_cigar", "<u4"),
                         ("early_abort", "<u4"), ("pad", "<u4"), ("cells", "<u8")])
SW_DTYPE = np.dtype([("ref_start", "<u4"), ("ref_end", "<u4"), ("read_start", "<i4"),
                     ("read_end", "<i4"), ("score", "<i4"), ("n_cigar", "<u4"),
                     ("early_abort", "<u4"), ("pad", "<u4"), ("cells", "<u8")])
assert VERIFY_DTYPE.itemsize == C.sizeof(OrcVerifyResult)
assert SW_DTYPE.itemsize == C.sizeof(OrcSwResult)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def verify_batch(reads, read_off, read_len, wins, win_off, win_len, p: OrcVerifyParams,
                 nthreads: int, cap_per_pair: int):
    """Threaded composed verification over flat arrays (numpy)."""
    n = len(read_off)
    out = np.zeros(n, VERIFY_DTYPE)
    cig = np.zeros(n * cap_per_pair, np.uint32)
    lib().orc_verify_batch(n, _p(reads), _p(read_off), _p(read_len), _p(wins), _p(win_off),
                           _p(win_len), C.byref(p), nthreads, _p(out), _p(cig), cap_per_pair)
    return out, cig.reshape(n, cap_per_pair)


def banded_sw_batch(reads, read_off, read_len, wins, win_off, win_len, offsets, c: OrcCfg,
                    nthreads: int, cap_per_pair: int, abort_score=ABORT_DISABLED, adaptive=True,
                    max_drift=16, dp_xdrop=None):
    n = len(read_off)
    out = np.zeros(n, SW_DTYPE)
    cig = np.zeros(n * cap_per_pair, np.uint32)
    lib().orc_banded_sw_batch(n, _p(reads), _p(read_off), _p(read_len), _p(wins), _p(win_off),
                              _p(win_len), _p(offsets), C.byref(c), abort_score, int(adaptive),
                              max_drift, c.xdrop if dp_xdrop is None else dp_xdrop, nthreads,
                              _p(out), _p(cig), cap_per_pair)
    return out, cig.reshape(n, cap_per_pair)


def sw_avx2_batch(reads, read_off, q, wins, win_off, r, c: OrcCfg, nthreads: int,
                  cap_per_pair: int):
    n = len(read_off)
    out = np.zeros(n, SW_DTYPE)
    cig = np.zeros(n * cap_per_pair, np.uint32)
    lib().orc_sw_avx2_batch(n, _p(reads), _p(read_off), q, _p(wins), _p(win_off), r, C.byref(c),
                            nthreads, _p(out), _p(cig), cap_per_pair)
    return out, cig.reshape(n, cap_per_pair)


def myers_batch(reads, read_off, read_len, wins, win_off, win_len, max_k, nthreads):
    n = len(read_off)
    dist = np.zeros(n, np.int64)
    end = np.zeros(n, np.int64)
    lib().orc_myers_batch(n, _p(reads), _p(read_off), _p(read_len), _p(wins), _p(win_off),
                          _p(win_len), max_k, nthreads, _p(dist), _p(end))
    return dist, end


def sieve_batch(reads, read_off, read_len, wins, win_off, win_len, nthreads):
    n = len(read_off)
    s = np.zeros(n, np.int32)
    m = np.zeros(n, np.int32)
    sec = np.zeros(n, np.int32)
    lib().orc_sieve_batch(n, _p(reads), _p(read_off), _p(read_len), _p(wins), _p(win_off),
                          _p(win_len), nthreads, _p(s), _p(m), _p(sec))
    return s, m, sec


CIGAR_CODES = {"M": 0, "I": 1, "D": 2, "N": 3, "S": 4}


def nm_md(read: bytes, ref: bytes, read_start: int, ref_start: int, cigar) -> tuple:
    """nm_md_from_cigar (md.rs:162-205); cigar as [(len, 'M'|'I'|'D'|'N'|'S')] or
    packed words. Returns (NM, MD)."""
    words = [w if isinstance(w, int) else (w[0] << 4) | CIGAR_CODES[w[1]] for w in cigar]
    arr = np.asarray(words or [0], np.uint32)
    nm = C.c_uint32()
    cap = 4 * (len(read) + len(ref)) + 64
    buf = C.create_string_buffer(cap)
    n = lib().orc_nm_md(read, len(read), ref, len(ref), read_start, ref_start,
                        arr.ctypes.data, len(words), C.byref(nm), buf, cap)
    return nm.value, buf.raw[:n].decode()


def md_builder(script: str, read: bytes = b"", ref: bytes = b"", lens=None) -> tuple:
    """MdBuilder driven op by op (see orc_md_builder)."""
    lens = np.asarray(lens if lens is not None else [0] * len(script), np.uint32)
    nm = C.c_uint32()
    buf = C.create_string_buffer(4096)
    n = lib().orc_md_builder(script.encode(), read or b"\0", ref or b"\0", lens.ctypes.data,
                             len(script), C.byref(nm), buf, 4096)
    return nm.value, buf.raw[:n].decode()


def nm_md_batch(reads, read_off, read_len, wins, win_off, win_len, read_start, ref_start,
                cig_off, n_cig, ops, nthreads: int, md_stride: int = 2048):
    n = len(read_off)
    nm = np.zeros(n, np.uint32)
    md_len = np.zeros(n, np.uint32)
    md = np.zeros(n * md_stride, np.uint8)
    lib().orc_nm_md_batch(n, _p(reads), _p(read_off), _p(read_len), _p(wins), _p(win_off),
                          _p(win_len), _p(read_start), _p(ref_start), _p(cig_off), _p(n_cig),
                          _p(ops), nthreads, _p(nm), _p(md_len), _p(md), md_stride)
    return nm, md_len, md.reshape(n, md_stride)


# ---------------------------------------------------------------------------
# WFA (src/alignment/wfa.rs)
# ---------------------------------------------------------------------------

@dataclass
class WfaRes:
    score: int        # WFA cost (the loss for the scored cost model)
    cigar: list       # [(len, op_char)]; empty for score-only
    text_start: int
    text_end: int

    def cigar_str(self) -> str:
        return "".join(f"{n}{c}" for n, c in self.cigar)


def wfa_cfg(mismatch=4, gap_open=6, gap_extend=1, max_score=100, adaptive_drop=None,
            text_begin_free=0, match_score=0, scored=False, traceback=True) -> OrcWfaCfg:
    return OrcWfaCfg(mismatch, gap_open, gap_extend, match_score, int(scored), max_score,
                     -1 if adaptive_drop is None else adaptive_drop, text_begin_free,
                     int(traceback))


def wfa(pattern: bytes, text: bytes, c: OrcWfaCfg):
    """wfa_align / wfa_score_only and their scored forms (wfa.rs:549-745) -> None | WfaRes."""
    cap = 2 * len(pattern) + len(text) + 8
    cig = (C.c_uint32 * cap)()
    sc, ts, te, nc = C.c_int32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    rc = lib().orc_wfa(pattern, len(pattern), text, len(text), C.byref(c), C.byref(sc),
                       C.byref(ts), C.byref(te), cig, cap, C.byref(nc))
    if rc < 0:
        raise ValueError("invalid WFA costs")
    if rc == 0:
        return None
    return WfaRes(sc.value, decode_cigar(cig[: nc.value]), ts.value, te.value)


def wfa_scored(pattern: bytes, text: bytes, a: int, b: int, o: int, e: int, max_score: int,
               adaptive_drop=None, text_begin_free=0, traceback=True):
    """wfa_align_scored (wfa.rs:57-65); with traceback=False the value of
    wfa_score_only_scored (wfa.rs:69-79): the affine score m*a - loss."""
    r = wfa(pattern, text, wfa_cfg(b, o, e, max_score, adaptive_drop, text_begin_free, a, True,
                                   traceback))
    if r is None or traceback:
        return r
    return len(pattern) * a - r.score


def wfa_batch(reads: np.ndarray, read_off, read_len, wins: np.ndarray, win_off, win_len,
              c: OrcWfaCfg, threads: int = 0, cap_per_pair: int = 64):
    """Per-pair orc_wfa on host threads -> (found, score, text_start, text_end, n_cigar, cigar)."""
    n = len(read_len)
    ro = np.ascontiguousarray(read_off, np.uint64)
    rl = np.ascontiguousarray(read_len, np.uint32)
    wo = np.ascontiguousarray(win_off, np.uint64)
    wl = np.ascontiguousarray(win_len, np.uint32)
    rs = np.ascontiguousarray(reads, np.uint8)
    ws = np.ascontiguousarray(wins, np.uint8)
    found = np.zeros(n, np.int32)
    score = np.zeros(n, np.int32)
    ts = np.zeros(n, np.uint32)
    te = np.zeros(n, np.uint32)
    nc = np.zeros(n, np.uint32)
    cig = np.zeros((n, cap_per_pair), np.uint32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    lib().orc_wfa_batch(n, p(rs), p(ro), p(rl), p(ws), p(wo), p(wl), C.byref(c),
                        threads or os.cpu_count() or 1, p(found), p(score), p(ts), p(te),
                        p(nc), p(cig), cap_per_pair)
    return found, score, ts, te, nc, cig


# ---------------------------------------------------------------------------
# Ungapped prefilter (src/alignment/prefilter.rs) and exact matches (mod.rs:779-832)
# ---------------------------------------------------------------------------
PREFILTER_REASONS = ("accept", "disabled", "not_short_preset", "not_top1",
                     "max_alignments_not_one", "span_too_small", "mism_too_high", "id_too_low",
                     "indel_suspect", "other")
PREFILTER_OTHER = (None, "read_len0", "non_monotonic", "anchor0", "span0", "neg_start",
                   "span_oob", "margin_fail")


def identity_floor(accept_min_identity: float) -> int:
    """(accept_min_identity * 100.0).round() as u16 (f32 arithmetic, saturating)."""
    v = float(np.float32(accept_min_identity) * np.float32(100.0))
    if v != v:
        return 0
    r = np.floor(abs(v) + 0.5) * (1 if v >= 0 else -1)
    return int(min(max(r, 0), 65535))


def prefilter_cfg(match_score=1, mismatch=4, xdrop=50, accept_enable=True, accept_only_top1=True,
                  accept_span_slack=5, accept_min_identity=98.0, accept_max_mismatches=2,
                  accept_require_score_margin=0, long_read_threshold=300,
                  multi_alignments_enabled=False, tail=True, min_id_override=None):
    return OrcPrefilterCfg(match_score, mismatch, xdrop, int(accept_enable),
                           int(accept_only_top1), accept_span_slack,
                           identity_floor(accept_min_identity), accept_max_mismatches,
                           accept_require_score_margin, long_read_threshold,
                           int(multi_alignments_enabled), int(tail),
                           -1 if min_id_override is None else min_id_override)


@dataclass
class PrefilterRes:
    result: str            # accept | reject | fallback
    reason: str
    metrics: tuple | None  # (len, mism, matches, identity_x10000, score, read_start, ref_start)
    nm: int = 0
    md: str = ""
    cigar: list = None


def prefilter(read: bytes, ref: bytes, chain, c: OrcPrefilterCfg, is_top1=True,
              score_margin=2**31 - 1) -> PrefilterRes:
    """prefilter_chain (prefilter.rs:93-294); chain = (ref_start, ref_end, read_start, read_end)."""
    ch = OrcChain(*chain)
    out = OrcPrefilterOut()
    md = C.create_string_buffer(len(read) * 4 + 32)
    n = lib().orc_prefilter(read, len(read), ref, len(ref), C.byref(ch), int(is_top1),
                            score_margin, C.byref(c), C.byref(out), md, len(md))
    if n < 0:
        raise ValueError("chain outside the read or reference")
    reason = PREFILTER_REASONS[out.reason]
    if out.reason == 9:
        reason = PREFILTER_OTHER[out.other]
    met = None
    if out.has_metrics:
        met = (out.len, out.mism, out.matches, out.identity_x10000, out.score, out.read_start,
               out.ref_start)
    res = PrefilterRes(("accept", "reject", "fallback")[out.result], reason, met)
    if out.result == 0:
        res.nm = out.nm
        res.md = md.raw[:n].decode()
        res.cigar = decode_cigar(list(out.cigar)[: out.n_cigar])
    return res


def exact_match_exists(read: bytes, ref: bytes, chain) -> bool:
    return bool(lib().orc_exact_match_exists(read, len(read), ref, len(ref),
                                             C.byref(OrcChain(*chain))))


def identical_nm(bases: bytes) -> int:
    return int(lib().orc_identical_nm(bases, len(bases)))


def prefilter_batch(reads, read_off, read_len, wins, win_off, win_len, chains, is_top1,
                    score_margin, c: OrcPrefilterCfg, exact_first=True, threads=0,
                    md_stride=0):
    """orc_prefilter_batch on host threads -> array of OrcPrefilterOut (and MD bytes)."""
    n = len(read_len)
    arrs = [np.ascontiguousarray(a, dt) for a, dt in
            ((reads, np.uint8), (read_off, np.uint64), (read_len, np.uint32), (wins, np.uint8),
             (win_off, np.uint64), (win_len, np.uint32), (chains, np.uint32))]
    top = None if is_top1 is None else np.ascontiguousarray(is_top1, np.uint8)
    mar = None if score_margin is None else np.ascontiguousarray(score_margin, np.int32)
    out = (OrcPrefilterOut * max(n, 1))()
    md = np.zeros(max(n * md_stride, 1), np.uint8) if md_stride else None
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = lib().orc_prefilter_batch(n, *[p(a) for a in arrs], p(top), p(mar), C.byref(c),
                                   int(exact_first), threads or os.cpu_count() or 1, out,
                                   p(md), md_stride)
    if rc < 0:
        raise ValueError("a chain lies outside its read or window")
    return out, md
