"""Host runtime over the C ABI: context, error mapping and pair batches.

The classes here are the host side of the drop-in boundary; every compute call
goes through libkira_gpu.so (there is no CPU path in this package).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

OP_CHARS = "MIDNS"


# --- CudaError (src/cuda/mod.rs:17-34) --------------------------------------
class CudaError(Exception):
    status = -1


class NotBuilt(CudaError):
    status = 1


class DriverError(CudaError):
    status = 2


class RuntimeFailure(CudaError):
    status = 3


class NoDevice(CudaError):
    status = 4


class ReadTooLong(CudaError):
    status = 5

    def __init__(self, msg: str, length: int = 0, maximum: int = A.READ_BYTES_MAX):
        super().__init__(msg)
        self.len = length
        self.max = maximum


class Timeout(CudaError):
    status = 6


class InvalidArgument(CudaError):
    status = 7


class OutOfMemory(CudaError):
    status = 8


class CapacityError(CudaError):
    status = 9


_ERRORS = {c.status: c for c in (NotBuilt, DriverError, RuntimeFailure, NoDevice, ReadTooLong,
                                 Timeout, InvalidArgument, OutOfMemory, CapacityError)}


def raise_for(rc: int, msg: str) -> None:
    if rc == A.KIRA_OK:
        return
    cls = _ERRORS.get(rc, CudaError)
    raise cls(f"[{A.STATUS_NAMES.get(rc, rc)}] {msg}")


def is_available() -> bool:
    """cuda::is_available (src/cuda/mod.rs:39-49)."""
    return bool(A.lib().kira_gpu_is_available())


# --- configuration -----------------------------------------------------------
@dataclass
class AlignmentConfig:
    """AlignmentConfig (src/alignment/mod.rs:24-35) plus the DP knobs the reference
    reads from KIRA_ADAPTIVE_BAND / KIRA_ADAPTIVE_MAX_DRIFT / KIRA_DP_XDROP."""
    match_score: int = 1
    mismatch: int = 4
    gap_open: int = 6
    gap_extend: int = 1
    bandwidth: int = 33
    xdrop: int = 100
    clip_penalty: int = 5
    adaptive: bool = True
    max_drift: int = 16
    dp_xdrop: int = -1

    def to_c(self) -> A.SwCfg:
        return A.SwCfg(self.match_score, self.mismatch, self.gap_open, self.gap_extend,
                       self.bandwidth, self.xdrop, self.clip_penalty, int(self.adaptive),
                       self.max_drift, self.dp_xdrop)


@dataclass
class VerifyParams:
    cfg: AlignmentConfig = field(default_factory=AlignmentConfig)
    sieve_threshold: int = 12
    myers_k: int = 8
    cert_strict: bool = False
    qgram_filter: bool = True  # exact 4-gram prefilter before Myers (same results)

    def to_c(self) -> A.VerifyParams:
        return A.VerifyParams(self.cfg.to_c(), self.sieve_threshold, self.myers_k,
                              int(self.cert_strict),
                              0 if self.qgram_filter else A.VERIFY_NO_QGRAM)


@dataclass
class WfaParams:
    """WfaPenalties / AlignmentConfig and WfaOptions (src/alignment/wfa.rs:9-111).

    scored=True selects WfaCosts::scored (wfa_align_scored / wfa_score_only_scored)
    with match_score > 0; max_score < 0 uses router::wfa_score_budget per read
    (budget_pct < 0: 25); adaptive_drop None is the exact search."""
    mismatch: int = 4
    gap_open: int = 6
    gap_extend: int = 1
    max_score: int = -1
    adaptive_drop: int | None = None
    text_begin_free: int = 0
    traceback: bool = True
    scored: bool = False
    match_score: int = 0
    budget_pct: int = -1

    @classmethod
    def scored_from(cls, cfg: "AlignmentConfig", **kw) -> "WfaParams":
        return cls(cfg.mismatch, cfg.gap_open, cfg.gap_extend, scored=True,
                   match_score=cfg.match_score, **kw)

    def to_c(self) -> A.WfaParams:
        return A.WfaParams(self.mismatch, self.gap_open, self.gap_extend, self.match_score,
                           int(self.scored), self.max_score, self.budget_pct,
                           -1 if self.adaptive_drop is None else self.adaptive_drop,
                           self.text_begin_free, int(self.traceback))


@dataclass
class PrefilterConfig:
    """prefilter_chain's arguments (src/alignment/prefilter.rs:93-108), defaults of the
    `mem` command (src/cli/args/mem.rs:460-477), and the KIRA_UNGAP_TAIL /
    KIRA_UNGAP_MINID knobs; exact_first runs exact_match_alignment first as stage 4
    does (stage4_alignment.rs:728-735)."""
    match_score: int = 1
    mismatch: int = 4
    xdrop: int = 100
    accept_enable: bool = True
    accept_only_top1: bool = True
    accept_span_slack: int = 15
    accept_min_identity: float = 98.5
    accept_max_mismatches: int = 5
    accept_require_score_margin: int = 0
    long_read_threshold: int = 500
    multi_alignments_enabled: bool = False
    tail: bool = True
    min_identity_x10000: int = -1
    exact_first: bool = True

    def to_c(self) -> A.PrefilterCfg:
        return A.PrefilterCfg(self.match_score, self.mismatch, self.xdrop, int(self.accept_enable),
                              int(self.accept_only_top1), self.accept_span_slack,
                              self.accept_min_identity, self.accept_max_mismatches,
                              self.accept_require_score_margin, self.long_read_threshold,
                              int(self.multi_alignments_enabled), int(self.tail),
                              self.min_identity_x10000, int(self.exact_first))


def _chains(chains) -> np.ndarray:
    """kira_chain records from a CHAIN_DTYPE array or an (n, 4) integer array of
    (ref_start, ref_end, read_start, read_end)."""
    a = np.asarray(chains)
    if a.dtype == A.CHAIN_DTYPE:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(a, np.uint32).reshape(-1, 4).view(A.CHAIN_DTYPE).reshape(-1)


# --- pair batches --------------------------------------------------------------
@dataclass
class PairBatch:
    """Flat (read x window) pairs: ASCII arenas plus per-pair offsets/lengths."""
    read_seq: np.ndarray
    read_off: np.ndarray
    read_len: np.ndarray
    win_seq: np.ndarray | None
    win_off: np.ndarray
    win_len: np.ndarray
    band_offset: np.ndarray | None = None
    abort_score: np.ndarray | None = None
    bandwidth: np.ndarray | None = None

    @property
    def n(self) -> int:
        return int(len(self.read_off))

    @classmethod
    def from_pairs(cls, reads, wins, band_offset=None, abort_score=None, bandwidth=None):
        """Build from equal-length lists of byte strings (a read may repeat)."""
        uniq: dict[bytes, int] = {}
        chunks, roff = [], []
        pos = 0
        for r in reads:
            r = bytes(r)
            if r not in uniq:
                uniq[r] = pos
                chunks.append(r)
                pos += len(r)
            roff.append(uniq[r])
        wchunks, woff = [], []
        wpos = 0
        for w in wins:
            w = bytes(w)
            woff.append(wpos)
            wchunks.append(w)
            wpos += len(w)

        def arr(x, dt):
            return None if x is None else np.ascontiguousarray(np.asarray(x, dtype=dt))

        return cls(np.frombuffer(b"".join(chunks) + b"\0", np.uint8).copy(),
                   np.asarray(roff, np.uint64), np.asarray([len(r) for r in reads], np.uint32),
                   np.frombuffer(b"".join(wchunks) + b"\0", np.uint8).copy(),
                   np.asarray(woff, np.uint64), np.asarray([len(w) for w in wins], np.uint32),
                   arr(band_offset, np.int32), arr(abort_score, np.int32),
                   arr(bandwidth, np.int32))

    def to_c(self) -> A.Pairs:
        p = A.Pairs()
        p.n = self.n
        p.read_seq = A.ptr(self.read_seq)
        p.read_seq_bytes = int(self.read_seq.nbytes)
        p.read_off = A.ptr(self.read_off)
        p.read_len = A.ptr(self.read_len)
        p.win_seq = A.ptr(self.win_seq)
        p.win_seq_bytes = 0 if self.win_seq is None else int(self.win_seq.nbytes)
        p.win_off = A.ptr(self.win_off)
        p.win_len = A.ptr(self.win_len)
        p.band_offset = A.ptr(self.band_offset)
        p.abort_score = A.ptr(self.abort_score)
        p.bandwidth = A.ptr(self.bandwidth)
        return p


def default_sw_cigar_cap(batch: "PairBatch") -> int:
    """CIGAR capacity that covers gapped alignments without a retry: 8 ops per pair
    or one op per 4 read bases, whichever is larger (a retry with the exact need
    follows only past that)."""
    bases = int(np.asarray(batch.read_len, np.uint64).sum()) if batch.n else 0
    return max(16, 8 * batch.n, bases // 4)


def decode_cigar(ops) -> list:
    return [(int(w) >> 4, OP_CHARS[int(w) & 0xF]) for w in ops]


def cigar_string(cig) -> str:
    return "".join(f"{n}{c}" for n, c in cig)


@dataclass
class SwPublicResult:
    """SwPublicResult (src/alignment/mod.rs:910-920), window coordinates."""
    ref_start: int
    ref_end: int
    read_start: int
    read_end: int
    score: int
    cigar: list
    early_abort: bool
    status: int = A.PAIR_SW

    def key(self):
        return (self.ref_start, self.ref_end, self.read_start, self.read_end, self.score,
                tuple(self.cigar), self.early_abort)


def results_to_list(res: np.ndarray, ops: np.ndarray) -> list:
    out = []
    for r in res:
        o, n = int(r["cigar_off"]), int(r["n_cigar"])
        out.append(SwPublicResult(int(r["ref_start"]), int(r["ref_end"]), int(r["read_start"]),
                                  int(r["read_end"]), int(r["score"]),
                                  decode_cigar(ops[o:o + n]), bool(r["early_abort"]),
                                  int(r["status"])))
    return out


# --- context -------------------------------------------------------------------
class GpuContext:
    """One kira_ctx (one device, one stream, one grow-only arena)."""

    def __init__(self, device: int = 0):
        self._lib = A.lib()
        h = C.c_void_p()
        rc = self._lib.kira_gpu_init(device, C.byref(h))
        if rc != A.KIRA_OK:
            raise_for(rc, f"kira_gpu_init(device={device}) failed")
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kira_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def last_error(self) -> str:
        buf = C.create_string_buffer(1024)
        self._lib.kira_gpu_last_error(self._h, buf, 1024)
        return buf.value.decode(errors="replace")

    def check(self, rc: int) -> None:
        if rc != A.KIRA_OK:
            raise_for(rc, self.last_error())

    def arena_bytes(self) -> int:
        return int(self._lib.kira_gpu_arena_bytes(self._h))

    # -- sieve drop-in
    def sieve_batch(self, jobs: list) -> np.ndarray:
        n = len(jobs)
        arr = (A.SieveJob * max(n, 1))()
        keep = []
        for i, j in enumerate(jobs):
            rb = np.frombuffer(bytes(j.read_packed) or b"\0", np.uint8)
            wb = np.frombuffer(bytes(j.ref_shifted[0]) or b"\0", np.uint8)
            keep += [rb, wb]
            arr[i] = A.SieveJob(rb.ctypes.data, len(j.read_packed), j.read_nucs, wb.ctypes.data,
                                len(j.ref_shifted[0]), j.ref_nucs, j.max_mismatches)
        out = (A.SieveResult * max(n, 1))()
        self.check(self._lib.kira_gpu_sieve_batch(self._h, arr, n, out))
        return np.array([(o.shift, o.mismatches, o.second_mismatches) for o in out[:n]],
                        dtype=np.int64).reshape(n, 3)

    def ref_upload(self, seq) -> None:
        a = np.frombuffer(bytes(seq), np.uint8) if not isinstance(seq, np.ndarray) else seq
        self.check(self._lib.kira_gpu_ref_upload(self._h, A.ptr(a), int(a.nbytes)))

    # -- Myers
    def myers_batch(self, batch: PairBatch, max_k: int):
        dist = np.empty(batch.n, np.int32)
        end = np.empty(batch.n, np.int32)
        pc = batch.to_c()
        self.check(self._lib.kira_gpu_myers_batch(self._h, C.byref(pc), max_k, A.ptr(dist),
                                                  A.ptr(end)))
        return dist, end

    # -- banded SW
    def bsw_batch(self, batch: PairBatch, cfg: AlignmentConfig, cigar_cap: int | None = None):
        n = batch.n
        res = np.zeros(n, A.SW_RESULT_DTYPE)
        cap = cigar_cap if cigar_cap is not None else default_sw_cigar_cap(batch)
        ops = np.zeros(cap, np.uint32)
        cb = A.CigarBuf(A.ptr(ops), cap, 0)
        cells = C.c_uint64()
        pc = batch.to_c()
        cc = cfg.to_c()
        rc = self._lib.kira_gpu_bsw_batch(self._h, C.byref(pc), C.byref(cc), A.ptr(res),
                                          C.byref(cb), C.byref(cells))
        if rc == 9 and cigar_cap is None:
            return self.bsw_batch(batch, cfg, int(cb.used) + 16)
        self.check(rc)
        return res, ops[: cb.used], int(cells.value)

    # -- align_batch_simd (full-window batch SW drop-in)
    def align_batch_simd(self, batch: PairBatch, cfg: AlignmentConfig, mode: int,
                         detected: int, cigar_cap: int | None = None):
        n = batch.n
        res = np.zeros(max(n, 1), A.SW_RESULT_DTYPE)
        cap = cigar_cap if cigar_cap is not None else max(16, 8 * n)
        ops = np.zeros(cap, np.uint32)
        cb = A.CigarBuf(A.ptr(ops), cap, 0)
        pc = batch.to_c()
        cc = cfg.to_c()
        rc = self._lib.kira_gpu_align_batch_simd(self._h, C.byref(pc), C.byref(cc), mode,
                                                 detected, A.ptr(res), C.byref(cb))
        if rc == 9 and cigar_cap is None:
            return self.align_batch_simd(batch, cfg, mode, detected, int(cb.used) + 16)
        self.check(rc)
        return res[:n], ops[: cb.used]

    # -- NM / MD:Z of a batch's alignments
    def nm_md(self, batch: PairBatch, res: np.ndarray, ops: np.ndarray,
              md_cap: int | None = None):
        """(nm per pair, list of MD strings) for the results `res` / CIGAR `ops`
        an alignment call returned on `batch` (nm 0xFFFFFFFF without alignment)."""
        n = batch.n
        res = np.ascontiguousarray(res)
        ops = np.ascontiguousarray(ops, np.uint32)
        nm = np.zeros(max(n, 1), np.uint32)
        off = np.zeros(n + 1, np.uint32)
        cap = md_cap if md_cap is not None else max(64, 8 * n)
        md = np.zeros(cap, np.uint8)
        used = C.c_uint64()
        pc = batch.to_c()
        rc = self._lib.kira_gpu_nm_md(self._h, C.byref(pc), A.ptr(res), A.ptr(ops) if len(ops) else None,
                                      len(ops), A.ptr(nm), A.ptr(off), A.ptr(md), cap, C.byref(used))
        if rc == 9 and md_cap is None:
            return self.nm_md(batch, res, ops, int(used.value) + 16)
        self.check(rc)
        text = md.tobytes()
        return nm[:n], [text[off[i]:off[i + 1]].decode() for i in range(n)]

    # -- WFA
    def wfa_batch(self, batch: PairBatch, params: WfaParams, max_score=None,
                  text_begin_free=None, cigar_cap: int | None = None):
        """kira_gpu_wfa_batch -> (results [WFA_RESULT_DTYPE], CIGAR ops). Optional
        per-pair int32 arrays override params.max_score / params.text_begin_free."""
        n = batch.n
        res = np.zeros(max(n, 1), A.WFA_RESULT_DTYPE)
        cap = cigar_cap if cigar_cap is not None else max(16, 4 * n)
        ops = np.zeros(max(cap, 1), np.uint32)
        cb = A.CigarBuf(A.ptr(ops), cap, 0)
        ms = None if max_score is None else np.ascontiguousarray(max_score, np.int32)
        tf = None if text_begin_free is None else np.ascontiguousarray(text_begin_free, np.int32)
        pc = batch.to_c()
        wp = params.to_c()
        rc = self._lib.kira_gpu_wfa_batch(self._h, C.byref(pc), C.byref(wp), A.ptr(ms),
                                          A.ptr(tf), A.ptr(res), C.byref(cb))
        if rc == 9 and cigar_cap is None:
            return self.wfa_batch(batch, params, max_score, text_begin_free, int(cb.used) + 16)
        self.check(rc)
        return res[:n], ops[: cb.used]

    # -- ungapped prefilter and exact matches
    def prefilter_batch(self, batch: PairBatch, chains: np.ndarray, cfg: PrefilterConfig,
                        is_top1=None, score_margin=None, cigar_cap: int | None = None,
                        md_cap: int | None = None):
        """kira_gpu_prefilter_batch -> (results [PREFILTER_RESULT_DTYPE], CIGAR ops,
        MD bytes). chains is a CHAIN_DTYPE array (window coordinates)."""
        n = batch.n
        ch = _chains(chains)
        res = np.zeros(max(n, 1), A.PREFILTER_RESULT_DTYPE)
        ccap = cigar_cap if cigar_cap is not None else max(16, 3 * n)
        mcap = md_cap if md_cap is not None else max(64, 8 * n)
        ops = np.zeros(max(ccap, 1), np.uint32)
        md = np.zeros(max(mcap, 1), np.uint8)
        cb = A.CigarBuf(A.ptr(ops), ccap, 0)
        used = C.c_uint64()
        top = None if is_top1 is None else np.ascontiguousarray(is_top1, np.uint8)
        mar = None if score_margin is None else np.ascontiguousarray(score_margin, np.int32)
        pc, pf = batch.to_c(), cfg.to_c()
        rc = self._lib.kira_gpu_prefilter_batch(self._h, C.byref(pc), A.ptr(ch), A.ptr(top),
                                                A.ptr(mar), C.byref(pf), A.ptr(res),
                                                C.byref(cb), A.ptr(md), mcap, C.byref(used))
        if rc == 9 and cigar_cap is None and md_cap is None:
            return self.prefilter_batch(batch, chains, cfg, is_top1, score_margin,
                                        int(cb.used) + 16, int(used.value) + 64)
        self.check(rc)
        return res[:n], ops[: cb.used], md[: used.value]

    def exact_match_batch(self, batch: PairBatch, chains: np.ndarray) -> np.ndarray:
        """kira_gpu_exact_match_batch -> uint8 per chain (exact_match_exists)."""
        n = batch.n
        ch = _chains(chains)
        out = np.zeros(max(n, 1), np.uint8)
        pc = batch.to_c()
        self.check(self._lib.kira_gpu_exact_match_batch(self._h, C.byref(pc), A.ptr(ch),
                                                        A.ptr(out)))
        return out[:n]

    # -- composed verification
    def verify_batch(self, batch: PairBatch, params: VerifyParams, detail: bool = False,
                     cigar_cap: int | None = None):
        n = batch.n
        res = np.zeros(n, A.SW_RESULT_DTYPE)
        det = np.zeros(n, A.DETAIL_DTYPE) if detail else None
        cap = cigar_cap if cigar_cap is not None else max(16, 4 * n)
        ops = np.zeros(cap, np.uint32)
        cb = A.CigarBuf(A.ptr(ops), cap, 0)
        cells = C.c_uint64()
        pc = batch.to_c()
        vp = params.to_c()
        rc = self._lib.kira_gpu_verify_batch(self._h, C.byref(pc), C.byref(vp), A.ptr(res),
                                             C.byref(cb), A.ptr(det), C.byref(cells))
        if rc == 9 and cigar_cap is None:
            return self.verify_batch(batch, params, detail, int(cb.used) + 16)
        self.check(rc)
        return res, ops[: cb.used], det, int(cells.value)


# --- serving (continuous batching) ----------------------------------------------
@dataclass
class RequestInfo:
    status: int
    n_pairs: int
    cigar_used: int
    t_submit_ns: int
    t_start_ns: int
    t_done_ns: int
    batch_id: int
    batch_requests: int

    @property
    def latency_s(self) -> float:
        return (self.t_done_ns - self.t_submit_ns) / 1e9


class Ticket:
    """One submitted request: owns its result buffers and keeps its inputs alive
    until the server has finished with them."""

    def __init__(self, server: "Server", tid: int, batch: PairBatch, res, ops, keep):
        self.server, self.id, self.batch = server, tid, batch
        self.res, self.ops, self._keep = res, ops, keep

    def poll(self) -> int:
        return int(self.server._lib.kira_server_poll(self.server._h, self.id))

    def done(self) -> bool:
        return self.poll() != A.KIRA_PENDING

    def wait(self, timeout_s: float = 60.0):
        """Results (per-pair structured array, this request's CIGAR ops); raises
        Timeout when the bounded wait expires, or the request's error."""
        rc = int(self.server._lib.kira_server_wait(self.server._h, self.id,
                                                   int(timeout_s * 1000)))
        if rc != A.KIRA_OK:
            raise_for(rc, f"request {self.id}: {self.server.last_error()}")
        return self.res, self.ops[: self.info().cigar_used]

    def info(self) -> RequestInfo:
        i = A.RequestInfo()
        raise_for(self.server._lib.kira_server_info(self.server._h, self.id, C.byref(i)),
                  f"no ticket {self.id}")
        return RequestInfo(i.status, i.n_pairs, i.cigar_used, i.t_submit_ns, i.t_start_ns,
                           i.t_done_ns, i.batch_id, i.batch_requests)

    def release(self) -> None:
        self.server._lib.kira_server_release(self.server._h, self.id)


class Server:
    """kira_server: `slots` concurrent batches over one device-resident reference;
    requests of the same kind and parameters that queue up are run as one batch."""

    def __init__(self, device: int = 0, slots: int = 2, max_batch_pairs: int = 1 << 20,
                 mem_fraction: float = 0.5):
        self._lib = A.lib()
        h = C.c_void_p()
        cfg = A.ServerCfg(device, slots, max_batch_pairs, mem_fraction)
        raise_for(self._lib.kira_server_create(C.byref(cfg), C.byref(h)),
                  f"kira_server_create(device={device}, slots={slots}) failed")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kira_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def last_error(self) -> str:
        buf = C.create_string_buffer(1024)
        self._lib.kira_server_last_error(self._h, buf, 1024)
        return buf.value.decode(errors="replace")

    def ref_upload(self, seq) -> None:
        a = np.frombuffer(bytes(seq), np.uint8) if not isinstance(seq, np.ndarray) else seq
        raise_for(self._lib.kira_server_ref_upload(self._h, A.ptr(a), int(a.nbytes)),
                  self.last_error())

    def _submit(self, fn, batch: PairBatch, params, cigar_cap):
        n = batch.n
        res = np.zeros(max(n, 1), A.SW_RESULT_DTYPE)
        cap = cigar_cap if cigar_cap is not None else max(16, 4 * n)
        ops = np.zeros(cap, np.uint32)
        pc = batch.to_c()
        cp = params.to_c()
        t = C.c_uint64()
        raise_for(fn(self._h, C.byref(pc), C.byref(cp), A.ptr(res), A.ptr(ops), cap, C.byref(t)),
                  "submit refused")
        return Ticket(self, int(t.value), batch, res[:n], ops, (pc, cp))

    def submit_verify(self, batch: PairBatch, params: VerifyParams,
                      cigar_cap: int | None = None) -> Ticket:
        return self._submit(self._lib.kira_server_submit_verify, batch, params, cigar_cap)

    def submit_bsw(self, batch: PairBatch, cfg: AlignmentConfig,
                   cigar_cap: int | None = None) -> Ticket:
        if cigar_cap is None:
            cigar_cap = default_sw_cigar_cap(batch)
        return self._submit(self._lib.kira_server_submit_bsw, batch, cfg, cigar_cap)

    def stats(self) -> dict:
        b, p, q = C.c_uint64(), C.c_uint64(), C.c_uint32()
        self._lib.kira_server_stats(self._h, C.byref(b), C.byref(p), C.byref(q))
        ms = (C.c_double * 4)()
        self._lib.kira_server_profile(self._h, ms)
        return {"batches": b.value, "pairs": p.value, "queued": q.value,
                "host_ms": {"staging": ms[0], "pipeline": ms[1], "scatter": ms[2],
                            "admission": ms[3]}}
