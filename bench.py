"""Benchmark of the composed verification path (sieve -> certificate -> Myers ->
banded SW with CIGAR) on the batched short-read workload: 2M (read x window)
pairs, 150 bp reads, 250 bp windows, 8 candidates per read, band 33, scoring
+1/-4/-6/-1, sieve threshold 12, Myers k 8; seeded synthetic data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0. `value` = pairs/s with inputs resident in HBM
(kira_gpu_verify_dev, CUDA events on the launching stream, L2 flushed between
steps); `e2e` = pairs/s through the host API (kira_gpu_verify_batch_compact: a
status byte per pair, rows and CIGARs of the aligned pairs; kira_gpu_verify_batch
with a row per pair beside it) with pinned host inputs and outputs, H2D + D2H inside
the timed region. After the timed steps the line's `parity` block checks every pair's
row and CIGAR against the oracle. Multi-GPU: one process per GPU, one job sharded into
contiguous ranges (weak scaling, no data-path collective), time = max over ranks.
The line also folds in a short uneven-batch run (`uneven`) and a serving run
(`serving`); `--workload` runs the other configurations on their own.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "batched_2M_150x250_band33"
METRIC = "pairs/s (composed sieve+Myers+banded-SW verification, bit-exact)"
UNIT = "pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--reads", type=int, default=250_000,
                    help="reads per GPU (x8 candidate windows = pairs per GPU)")
    ap.add_argument("--ref-len", type=int, default=100_000_000, help="reference bases")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the oracle pass (parity check and cpu_baseline)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the uneven-batch and serving runs folded into the headline line")
    ap.add_argument("--backend", choices=["nccl", "gloo"], default="nccl",
                    help="process-group backend of a multi-GPU run")
    ap.add_argument("--dry-run", action="store_true",
                    help="multi-rank plumbing only (launch, shards, gather, timing reduction), "
                         "no GPU work; for CPU tests with --backend gloo")
    ap.add_argument("--shape", type=int, default=-1,
                    help="install this banded-SW launch shape instead of autotuning")
    ap.add_argument("--workload", choices=["batched", "uneven", "serving", "gapfill", "nmmd",
                                           "wfa", "prefilter"],
                    default="batched",
                    help="batched: the headline 2M-pair verification; uneven: 500k banded-SW "
                         "pairs of mixed length and band (bucketed vs one-launch path); "
                         "serving: Poisson request stream through the server vs one request "
                         "per call; gapfill: long-read gap-fill segments at band 256; nmmd: "
                         "NM + MD:Z of the batched alignments; wfa: the cascade's WFA step "
                         "(scored costs, router budget) with and without traceback; "
                         "prefilter: stage-4 exact match + ungapped prefilter per chain")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: requests per second")
    ap.add_argument("--duration", type=float, default=5.0, help="serving: seconds of arrivals")
    ap.add_argument("--slots", type=int, default=4, help="serving: concurrent batches")
    ap.add_argument("--long-reads", type=int, default=20_000,
                    help="gapfill: simulated long reads (split into gap-fill segments)")
    ap.add_argument("--wfa-pairs", type=int, default=1_000_000, help="wfa: pairs per call")
    ap.add_argument("--wfa-drop", type=int, default=-1, help="wfa: adaptive drop (< 0 exact)")
    ap.add_argument("--chains", type=int, default=2_000_000, help="prefilter: chains per call")
    ap.add_argument("--wfa-lanes", type=int, default=0,
                    help="wfa: lanes per pair (8, 16, 32; 0 = library default)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


VERIFY_CFG = dict(match=1, mismatch=4, gap_open=6, gap_extend=1, band=33, xdrop=100, clip=5,
                  sieve_threshold=12, myers_k=8)
PARITY_FIELDS = ("status", "score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar",
                 "early_abort", "cigar", "cells")


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    c = VERIFY_CFG
    op = O.verify_params(O.cfg(c["match"], c["mismatch"], c["gap_open"], c["gap_extend"],
                               c["band"], c["xdrop"], c["clip"]), c["sieve_threshold"],
                         c["myers_k"])
    return O, op


def oracle_verify(w, nthreads: int, cap: int = 16):
    """The oracle port of the reference CPU path (sieve -> certificate -> Myers ->
    banded_sw_with per pair) over every pair of `w`, on `nthreads` host threads;
    windows read straight from the reference. Returns (rows, CIGAR ops per pair,
    seconds). Pairs whose CIGAR exceeds `cap` ops are re-run with room for all."""
    O, op = _oracle()
    t = time.perf_counter()
    out, cig = O.verify_batch(w.reads, w.read_off, w.read_len, w.reference, w.win_off, w.win_len,
                              op, nthreads, cap)
    el = time.perf_counter() - t
    big = np.nonzero(out["n_cigar"] > cap)[0]
    wide = {}
    if len(big):
        o2, c2 = O.verify_batch(w.reads, w.read_off[big].copy(), w.read_len[big].copy(),
                                w.reference, w.win_off[big].copy(), w.win_len[big].copy(), op,
                                nthreads, 1024)
        wide = {int(p): c2[k] for k, p in enumerate(big)}
    return out, cig, wide, el


def parity_block(res, ops, cells, w, nthreads: int):
    """Every pair of this rank's workload against the oracle, field by field, and the
    CIGAR op by op; `cells` = the GPU's executed band cells of one step."""
    out, cig, wide, el = oracle_verify(w, nthreads)
    by = {}
    for f in PARITY_FIELDS[:8]:
        by[f] = int((res[f].astype(np.int64) != out[f].astype(np.int64)).sum())
    n = res["n_cigar"].astype(np.int64)
    sel = np.nonzero((n == out["n_cigar"].astype(np.int64)) & (n > 0))[0]
    cnt = n[sel]
    bad = set()
    if len(sel):
        pair = np.repeat(sel, cnt)
        t = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        got = ops[res["cigar_off"][pair].astype(np.int64) + t]
        narrow = cig.shape[1]
        want = np.where(t < narrow, cig[pair, np.minimum(t, narrow - 1)], 0)
        for k in np.nonzero(t >= narrow)[0]:
            want[k] = wide[int(pair[k])][t[k]]
        bad = set(np.unique(pair[got != want]).tolist())
    by["cigar"] = len(bad)
    by["cells"] = int(int(out["cells"].sum()) != int(cells))
    return {"checked": int(len(res)), "mismatches": int(sum(by.values())), "by_field": by,
            "fields": list(PARITY_FIELDS)}, el


def run_reference(args, rank, world):
    """Reference arm: the reference CPU path (the oracle port: the reference is Rust
    and cannot be built here) on all host threads, over the same 2M-pair workload
    as the GPU arm's rank 0, every pair every step. Under torchrun only rank 0 runs."""
    if rank != 0:
        return None
    from kira_ls_aligner_b200 import synth
    w = synth.batched(n_reads=args.reads, ref_len=args.ref_len)
    nthreads = os.cpu_count() or 1
    O, op = _oracle()
    a = (w.reads, w.read_off, w.read_len, w.reference, w.win_off, w.win_len)
    for _ in range(args.warmup):
        O.verify_batch(*a, op, nthreads, 16)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.verify_batch(*a, op, nthreads, 16)
        times.append(time.perf_counter() - t)
    n = w.n_pairs
    v = n * len(times) / sum(times)
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded; no public dataset)",
        "config": _config(args, w, world, "reference CPU path on all host threads"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"all {n} pairs of the workload every step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _config(args, w, world, parallelism):
    return {"workload": WORKLOAD, "pairs_per_gpu": 8 * args.reads, "read_len": 150,
            "window_len": 250, "candidates_per_read": 8, "band": 33, "sieve_threshold": 12,
            "myers_k": 8, "scoring": "+1/-4/-6/-1, xdrop 100, clip 5, adaptive band (drift 16)",
            "reference_bp": int(len(w.reference)), "seed": "0xB200",
            "l2": "flushed between steps (256 MB write)", "parallelism": parallelism}


def run_uneven(args, rank, local, world):
    """Uneven-length banded SW: 500k pairs, reads U[50,300], band U{16,32,64,128},
    window = read + 2 x band. Bucketed path (band classes, tuned shapes, dynamic
    fetch) vs the one-launch path, both through the host API (H2D + D2H per call)."""
    import torch

    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, PairBatch, _abi, autotune, synth
    if rank != 0:
        return None
    torch.cuda.set_device(local)
    w = synth.uneven(resident=True)
    n = w.n_pairs
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    batch = PairBatch(pin(w.reads), pin(w.read_off), pin(w.read_len), None,
                      pin(w.win_off), pin(w.win_len), pin(w.band_offset), None,
                      pin(w.bandwidth))
    cfg = AlignmentConfig(1, 4, 6, 1, 33, 100, 5, True, 16)
    ctx = GpuContext(local)
    ctx.ref_upload(w.reference)
    L = _abi.lib()
    # Autotune the shape of each band class on a 20k-pair sample of that class
    # (DP stage time from the library's stage events).
    tuned = {}
    for band in (16, 32, 64, 128):
        sub = _subset(w, np.nonzero(w.bandwidth == band)[0][:20000])
        tuned[band] = autotune.tune_bsw_shape(
            ctx, band, lambda: ctx.bsw_batch(sub, cfg), device_name=torch.cuda.get_device_name(local))
    # Both forms through the C entry point on the same preallocated pinned host
    # outputs (result rows and CIGAR ops), as the e2e verification call does.
    from kira_ls_aligner_b200.runtime import default_sw_cigar_cap
    res_h = torch.empty(n * 32, dtype=torch.uint8).pin_memory()
    ops_cap = default_sw_cigar_cap(batch)
    ops_h = torch.empty(ops_cap, dtype=torch.int32).pin_memory()
    cb = _abi.CigarBuf(ops_h.data_ptr(), ops_cap, 0)
    pc, cc, cells_h = batch.to_c(), cfg.to_c(), C.c_uint64()

    def call():
        ctx.check(L.kira_gpu_bsw_batch(ctx.handle, C.byref(pc), C.byref(cc), res_h.data_ptr(),
                                       C.byref(cb), C.byref(cells_h)))

    out = {}
    for mode in ("plain", "bucketed"):
        ctx.check(L.kira_gpu_set_plain(ctx.handle, 1 if mode == "plain" else 0))
        # The bucketed form replays its per-class launches from a CUDA graph.
        ctx.check(L.kira_gpu_set_graphs(ctx.handle, 0 if mode == "plain" else 1, None, None))
        for _ in range(args.warmup):
            call()
        ts = [_timed(call) for _ in range(args.steps)]
        res, ops, cells = ctx.bsw_batch(batch, cfg)
        ctx.check(L.kira_gpu_profile(ctx.handle, 1))
        ctx.bsw_batch(batch, cfg)
        buf = (C.c_float * 8)()
        k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
        ctx.check(L.kira_gpu_profile(ctx.handle, 0))
        stages = dict(zip(("upload", "bucketing", "bsw_dp", "bsw_traceback", "cigar_compact"),
                          [round(float(x), 3) for x in buf[:k]]))
        if mode == "bucketed":
            graphs = graph_counts(ctx)
        out[mode] = {"stage_ms": stages, "pairs_per_s": n / (sum(ts) / len(ts) / 1e3),
                     "ms_per_call": sum(ts) / len(ts), "gcups": cells / (sum(ts) / len(ts) / 1e3) / 1e9,
                     "cells": int(cells), "checksum": int(res["score"].astype(np.int64).sum())}
    assert out["plain"]["checksum"] == out["bucketed"]["checksum"]
    ctx.close()
    return {
        "metric": "pairs/s (uneven-length banded SW with CIGAR, bit-exact)",
        "value": out["bucketed"]["pairs_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out["bucketed"]["ms_per_call"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded)",
        "config": {"workload": w.name, "pairs": n, "read_len": "U[50,300]",
                   "band": "U{16,32,64,128}", "window": "read + 2*band", "errors": "U[0,3%] 8:1:1",
                   "path": "host API (kira_gpu_bsw_batch), pinned inputs (reads + "
                           "descriptors; windows from the resident reference) and pinned "
                           "outputs (rows + CIGAR ops), H2D + D2H per call"},
        "bucketed": out["bucketed"], "plain": out["plain"],
        "speedup_vs_plain": out["bucketed"]["pairs_per_s"] / out["plain"]["pairs_per_s"],
        "cuda_graphs": graphs,
        "autotune": tuned}


def run_nmmd(args, rank, local, world):
    """NM and MD:Z of the batched workload's alignments (2M pairs, 150 / 250 bp):
    kira_gpu_nm_md through the host API (pairs, results and CIGARs in, NM,
    offsets and MD text out) against the oracle on all host threads."""
    import torch

    from kira_ls_aligner_b200 import GpuContext, PairBatch, VerifyParams, _abi, synth
    if rank != 0:
        return
    torch.cuda.set_device(local)
    w = synth.batched(n_reads=args.reads)
    ctx = GpuContext(local)
    ctx.ref_upload(w.reference)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    b = PairBatch(pin(w.reads), pin(w.read_off), pin(w.read_len), None, pin(w.win_off),
                  pin(w.win_len))
    res, ops, _, _ = ctx.verify_batch(b, VerifyParams(sieve_threshold=12, myers_k=8))
    res = pin(res.view(np.uint8)).view(_abi.SW_RESULT_DTYPE)
    L = _abi.lib()
    n = w.n_pairs
    nm = pin(np.zeros(n, np.uint32))
    off = pin(np.zeros(n + 1, np.uint32))
    mdb = pin(np.zeros(64 * n, np.uint8))
    used = C.c_uint64()
    pc = b.to_c()
    ops = pin(np.ascontiguousarray(ops, np.uint32))

    def call():  # the C entry point on preallocated host buffers
        ctx.check(L.kira_gpu_nm_md(ctx.handle, C.byref(pc), _abi.ptr(res), _abi.ptr(ops),
                                   len(ops), _abi.ptr(nm), _abi.ptr(off), _abi.ptr(mdb),
                                   mdb.nbytes, C.byref(used)))
    for _ in range(args.warmup):
        call()
    ts = [_timed(call) for _ in range(args.steps)]
    ctx.check(L.kira_gpu_profile(ctx.handle, 1))
    call()
    buf = (C.c_float * 8)()
    k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
    ctx.check(L.kira_gpu_profile(ctx.handle, 0))
    stage = [float(x) for x in buf[:k]]
    ms = sum(ts) / len(ts)
    aligned = int((res["n_cigar"] > 0).sum())
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as O
        sel = np.nonzero(res["n_cigar"] > 0)[0][:200_000]
        nthreads = os.cpu_count() or 1
        t = time.perf_counter()
        O.nm_md_batch(w.reads, w.read_off[sel].copy(), w.read_len[sel].copy(), w.reference,
                      w.win_off[sel].copy(), w.win_len[sel].copy(),
                      res["read_start"][sel].copy(), res["ref_start"][sel].copy(),
                      res["cigar_off"][sel].copy(), res["n_cigar"][sel].copy(), ops, nthreads,
                      md_stride=512)
        el = time.perf_counter() - t
        cpu = {"value": len(sel) / el, "unit": "aligned pairs/s", "cores": nthreads,
               "kind": "port", "sample": f"{len(sel)} aligned pairs of the workload"}
    print(json.dumps({
        "metric": "pairs/s (NM + MD:Z from the device CIGARs, bit-exact)",
        "value": w.n_pairs / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": "nmmd_batched_2M_150x250", "pairs": w.n_pairs,
                   "aligned_pairs": aligned, "md_bytes": int(used.value),
                   "path": "host API, pinned inputs, H2D + D2H per call"},
        "aligned_pairs_per_s": aligned / (ms / 1e3),
        "stage_ms": {"upload": stage[0] if k > 0 else None,
                     "nm_and_lengths": stage[1] if k > 1 else None,
                     "md_text": stage[3] if k > 3 else None},
        "cpu_baseline": cpu}))
    ctx.close()


def run_wfa(args, rank, local, world):
    """The cascade's WFA step (try_fast_dp_alignment, mod.rs:344-439): 150 bp reads
    against read + 33 bp of text at the seed-implied start over a resident
    reference, scored costs +1/-4/-6/-1, router budget (25 % of the read x 5),
    exact search. Both wfa_align_scored (traceback + CIGAR) and
    wfa_score_only_scored (locus_alignment_score) through the host API with
    pinned inputs (H2D + D2H inside the timed region); `value` is the traceback
    form, the kernel time from the library's stage events."""
    import torch

    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, PairBatch, WfaParams, _abi, synth
    if rank != 0:
        return
    torch.cuda.set_device(local)
    w = synth.wfa_cascade(args.wfa_pairs)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    b = PairBatch(pin(w.reads), pin(w.read_off), pin(w.read_len), None, pin(w.win_off),
                  pin(w.win_len))
    ctx = GpuContext(local)
    ctx.ref_upload(w.reference)
    L = _abi.lib()
    ctx.check(L.kira_gpu_set_wfa_lanes(ctx.handle, args.wfa_lanes))
    n = w.n_pairs
    drop = None if args.wfa_drop < 0 else args.wfa_drop
    out = {}
    for mode, tb in (("traceback", True), ("score_only", False)):
        p = WfaParams.scored_from(AlignmentConfig(), adaptive_drop=drop, traceback=tb)
        res = pin(np.zeros(n * _abi.WFA_RESULT_DTYPE.itemsize, np.uint8)).view(
            _abi.WFA_RESULT_DTYPE)
        ops = pin(np.zeros(8 * n, np.uint32))
        cb = _abi.CigarBuf(_abi.ptr(ops), len(ops), 0)
        pc, wp = b.to_c(), p.to_c()

        def call():  # the C entry point on preallocated host buffers
            ctx.check(L.kira_gpu_wfa_batch(ctx.handle, C.byref(pc), C.byref(wp), None, None,
                                           _abi.ptr(res), C.byref(cb)))
        for _ in range(args.warmup):
            call()
        ts = [_timed(call) for _ in range(args.steps)]
        ctx.check(L.kira_gpu_profile(ctx.handle, 1))
        kern = []
        for _ in range(3):
            call()
            buf = (C.c_float * 8)()
            k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
            kern.append([float(x) for x in buf[:k]])
        ctx.check(L.kira_gpu_profile(ctx.handle, 0))
        ms = sum(ts) / len(ts)
        kms = statistics.median(s[1] for s in kern)
        cost = res["cost"][res["found"] == 1].astype(np.float64)
        out[mode] = {"e2e_pairs_per_s": n / (ms / 1e3), "ms_per_call": ms,
                     "kernel_ms": kms, "kernel_pairs_per_s": n / (kms / 1e3),
                     "stage_ms": dict(zip(("upload", "wavefronts", "cigar_compact", "download"),
                                          [round(x, 3) for x in kern[-1]])),
                     "found": int(res["found"].sum()), "mean_cost": float(cost.mean()),
                     "cigar_ops": int(cb.used),
                     "checksum": int(res["cost"].astype(np.int64).sum())}
    assert out["traceback"]["checksum"] == out["score_only"]["checksum"]
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as O
        nthreads = os.cpu_count() or 1
        m = min(n, 200_000)
        c = O.wfa_cfg(4, 6, 1, 185, drop, 0, 1, True, True)
        wins = w.reference
        t = time.perf_counter()
        O.wfa_batch(w.reads, w.read_off[:m], w.read_len[:m], wins, w.win_off[:m], w.win_len[:m],
                    c, nthreads, 64)
        el = time.perf_counter() - t
        cpu = {"value": m / el, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"first {m} pairs of the workload, traceback form"}
    tb = out["traceback"]
    h2d = int(w.read_len.sum()) + n * (8 + 4 + 8 + 4)
    print(json.dumps({
        "metric": "pairs/s (WFA step of the cascade: scored wfa_align with CIGAR, bit-exact)",
        "value": tb["kernel_pairs_per_s"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tb["kernel_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16/int32",
        "data": "synthetic (seeded)",
        "config": {"workload": w.name, "pairs": n, "read_len": 150, "text_len": 183,
                   "costs": "scored 1/4/6/1", "max_score": "router budget (185)",
                   "adaptive_drop": drop, "errors": "U[0,4%] 4:1:1",
                   "lanes_per_pair": args.wfa_lanes or "default",
                   "path": "resident reference, host API, pinned inputs"},
        "e2e": {"value": tb["e2e_pairs_per_s"], "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 32 * n + 4 * tb["cigar_ops"]},
        "modes": out, "cpu_baseline": cpu}))
    ctx.close()


def run_prefilter(args, rank, local, world):
    """Stage 4's step before the cascade (stage4_alignment.rs:728-776): per chain
    exact_match_alignment, else prefilter_chain (ungapped x-drop extension, span
    Hamming count, accept cascade, [S]M[S] CIGAR + NM + MD:Z for accepts), with
    the `mem` defaults. 2M chains of 150 bp reads over a resident 50 Mbp contig;
    host API with pinned inputs (H2D + D2H inside the timed region); the kernel
    time is passes 1 + 2 from the library's stage events."""
    import torch

    from kira_ls_aligner_b200 import GpuContext, PairBatch, PrefilterConfig, _abi, synth
    if rank != 0:
        return
    torch.cuda.set_device(local)
    w = synth.prefilter_chains(args.chains)
    n = w.n_pairs
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    b = PairBatch(pin(w.reads), pin(w.read_off), pin(w.read_len), None,
                  pin(np.zeros(n, np.uint64)), pin(np.full(n, len(w.reference), np.uint32)))
    chains = pin(w.chains)  # (n, 4) uint32 = kira_chain
    top1, margin = pin(w.is_top1), pin(w.score_margin)
    ctx = GpuContext(local)
    ctx.ref_upload(w.reference)
    L = _abi.lib()
    cfg = PrefilterConfig()
    res = pin(np.zeros(n * _abi.PREFILTER_RESULT_DTYPE.itemsize, np.uint8)).view(
        _abi.PREFILTER_RESULT_DTYPE)
    ops = pin(np.zeros(3 * n, np.uint32))
    md = pin(np.zeros(16 * n, np.uint8))
    cb = _abi.CigarBuf(_abi.ptr(ops), len(ops), 0)
    used = C.c_uint64()
    pc, pf = b.to_c(), cfg.to_c()

    def call():  # the C entry point on preallocated pinned host buffers
        ctx.check(L.kira_gpu_prefilter_batch(ctx.handle, C.byref(pc), _abi.ptr(chains),
                                             _abi.ptr(top1), _abi.ptr(margin), C.byref(pf),
                                             _abi.ptr(res), C.byref(cb), _abi.ptr(md), md.nbytes,
                                             C.byref(used)))
    for _ in range(args.warmup):
        call()
    ts = [_timed(call) for _ in range(args.steps)]
    ctx.check(L.kira_gpu_profile(ctx.handle, 1))
    stages = []
    for _ in range(3):
        call()
        buf = (C.c_float * 8)()
        k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
        stages.append([float(x) for x in buf[:k]])
    ctx.check(L.kira_gpu_profile(ctx.handle, 0))
    ms = sum(ts) / len(ts)
    st = [statistics.median(s[i] for s in stages) for i in range(len(stages[0]))]
    kms = st[1] + st[3]
    kinds = np.bincount(res["result"], minlength=4)
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as O
        nthreads = os.cpu_count() or 1
        m = min(n, 1_000_000)
        oc = O.prefilter_cfg(1, 4, 100, True, True, 15, 98.5, 5, 0, 500)
        t = time.perf_counter()
        O.prefilter_batch(w.reads, w.read_off[:m], w.read_len[:m], w.reference,
                          np.zeros(m, np.uint64), np.full(m, len(w.reference), np.uint32),
                          w.chains[:m], w.is_top1[:m], w.score_margin[:m], oc, True, nthreads, 32)
        el = time.perf_counter() - t
        cpu = {"value": m / el, "unit": "chains/s", "cores": nthreads, "kind": "port",
               "sample": f"first {m} chains of the workload"}
    h2d = int(w.read_len.sum()) + n * (8 + 4 + 8 + 4 + 16 + 1 + 4)
    print(json.dumps({
        "metric": "chains/s (stage-4 exact match + ungapped prefilter with CIGAR/NM/MD, bit-exact)",
        "value": n / (kms / 1e3), "unit": "chains/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": w.name, "chains": n, "read_len": 150,
                   "reference_bp": int(len(w.reference)), "cfg": "mem defaults",
                   "path": "resident contig, host API, pinned inputs"},
        "e2e": {"value": n / (ms / 1e3), "unit": "chains/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 48 * n + 4 * int(cb.used) + int(used.value)},
        "stage_ms": dict(zip(("upload", "extend_decide", "offsets", "cigar_md", "download"),
                             [round(x, 3) for x in st])),
        "outcomes": {"accept": int(kinds[0]), "reject": int(kinds[1]),
                     "fallback": int(kinds[2]), "exact": int(kinds[3])},
        "cpu_baseline": cpu}))
    ctx.close()


def _slice_short(w, r0, nreads, cands=4):
    """PairBatch of reads [r0, r0 + nreads) of a short-read pool (compact read arena;
    windows stay reference coordinates)."""
    from kira_ls_aligner_b200 import PairBatch
    a, b = r0 * cands, (r0 + nreads) * cands
    base = int(w.read_off[a])
    end = int(w.read_off[b - 1]) + int(w.read_len[b - 1])
    return PairBatch(np.concatenate([w.reads[base:end], np.zeros(16, np.uint8)]),
                     w.read_off[a:b] - np.uint64(base), w.read_len[a:b].copy(), None,
                     w.win_off[a:b].copy(), w.win_len[a:b].copy())


def _slice_long(g, s0, n):
    from kira_ls_aligner_b200 import PairBatch
    base = int(g.read_off[s0])
    end = int(g.read_off[s0 + n - 1]) + int(g.read_len[s0 + n - 1])
    return PairBatch(np.concatenate([g.reads[base:end], np.zeros(16, np.uint8)]),
                     g.read_off[s0:s0 + n] - np.uint64(base), g.read_len[s0:s0 + n].copy(), None,
                     g.win_off[s0:s0 + n].copy(), g.win_len[s0:s0 + n].copy(),
                     g.band_offset[s0:s0 + n].copy(), None, g.bandwidth[s0:s0 + n].copy())


def run_serving(args, rank, local, world):
    """Serving loop: seeded Poisson arrivals (70 % short requests of 1k-64k reads x 4
    windows, 30 % long requests of 50-2000 gap-fill segments at band 256) over a
    1 Gbp device-resident reference. The server (continuous batching over `slots`
    streams) against the plain path (one request per call, in arrival order)."""
    import torch

    from kira_ls_aligner_b200 import (AlignmentConfig, GpuContext, Server, VerifyParams, _abi,
                                      synth)
    if rank != 0:
        return None
    torch.cuda.set_device(local)
    pool = synth.serving_pool()
    sched = synth.arrivals(0xA11, args.rate, args.duration)
    vp = VerifyParams(sieve_threshold=12, myers_k=8)
    cfg = AlignmentConfig(1, 4, 6, 1, 256, 100, 5, True, 16)
    nshort = len(pool.short.read_off) // 4
    nlong = len(pool.long.read_off)
    reqs, rs, ls = [], 0, 0
    for t, kind, n in sched:
        if kind == "short":
            rs = 0 if rs + n > nshort else rs
            reqs.append((t, kind, _slice_short(pool.short, rs, n)))
            rs += n
        else:
            ls = 0 if ls + n > nlong else ls
            reqs.append((t, kind, _slice_long(pool.long, ls, n)))
            ls += n
    total_pairs = sum(b.n for _, _, b in reqs)

    def pct(x, p):
        return float(np.percentile(np.asarray(x), p)) * 1e3

    def serve(open_loop: bool):
        srv = Server(local, slots=args.slots, max_batch_pairs=1 << 20)
        srv.ref_upload(pool.reference)
        # Warm-up (untimed): the whole request stream submitted at once, twice, so that
        # every slot has run full-size batches of both kinds (arenas, pinned staging,
        # the chunked path's twin context and side streams) before the timed run.
        for _ in range(2):
            warm = [srv.submit_verify(b, vp) if kind == "short" else srv.submit_bsw(b, cfg)
                    for _, kind, b in reqs]
            for t in warm:
                t.wait(600)
        b0 = srv.stats()["batches"]
        tickets = []
        t0 = time.perf_counter()
        for t, kind, b in reqs:
            d = t0 + t - time.perf_counter() if open_loop else 0.0
            if d > 0:
                time.sleep(d)
            tickets.append((kind, srv.submit_verify(b, vp) if kind == "short"
                            else srv.submit_bsw(b, cfg)))
        t_sub = time.perf_counter() - t0
        infos = []
        for kind, tk in tickets:
            tk.wait(600)
            infos.append((kind, tk.info()))
        first = min(i.t_submit_ns for _, i in infos)
        last = max(i.t_done_ns for _, i in infos)
        lat = [i.latency_s for _, i in infos]
        out = {"pairs_per_s": total_pairs / ((last - first) / 1e9),
               "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
               "p50_short_ms": pct([i.latency_s for k, i in infos if k == "short"], 50),
               "p99_short_ms": pct([i.latency_s for k, i in infos if k == "short"], 99),
               "p50_long_ms": pct([i.latency_s for k, i in infos if k == "long"], 50),
               "p99_long_ms": pct([i.latency_s for k, i in infos if k == "long"], 99),
               "batches": srv.stats()["batches"] - b0,
               # where the slowest requests spent their time: queued (submit to batch
               # start) and in their batch (start to done)
               "queue_ms_p50_p99": [pct([(i.t_start_ns - i.t_submit_ns) / 1e9 for _, i in infos], q)
                                    for q in (50, 99)],
               "batch_ms_p50_p99": [pct([(i.t_done_ns - i.t_start_ns) / 1e9 for _, i in infos], q)
                                    for q in (50, 99)],
               "host_ms": srv.stats()["host_ms"], "submit_s": t_sub,
               "mean_requests_per_batch": float(np.mean([i.batch_requests for _, i in infos]))}
        srv.close()
        return out

    def plain_run(open_loop: bool):
        ctx = GpuContext(local)
        ctx.ref_upload(pool.reference)
        ctx.check(_abi.lib().kira_gpu_set_plain(ctx.handle, 1))
        for _, kind, b in reqs[:8]:
            ctx.verify_batch(b, vp) if kind == "short" else ctx.bsw_batch(b, cfg)
        plat, pk = [], []
        t0 = time.perf_counter()
        for t, kind, b in reqs:
            arr = t0 + t if open_loop else t0
            d = arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ctx.verify_batch(b, vp) if kind == "short" else ctx.bsw_batch(b, cfg)
            plat.append(time.perf_counter() - arr)
            pk.append(kind)
        span = time.perf_counter() - (t0 + (reqs[0][0] if open_loop else 0.0))
        ctx.close()
        return {"pairs_per_s": total_pairs / span, "p50_ms": pct(plat, 50),
                "p99_ms": pct(plat, 99),
                "p50_short_ms": pct([x for x, k in zip(plat, pk) if k == "short"], 50),
                "p99_short_ms": pct([x for x, k in zip(plat, pk) if k == "short"], 99),
                "p50_long_ms": pct([x for x, k in zip(plat, pk) if k == "long"], 50),
                "p99_long_ms": pct([x for x, k in zip(plat, pk) if k == "long"], 99)}

    # Open loop: each request submitted at its Poisson arrival time (latency);
    # saturated: every request submitted at once (capacity in pairs/s).
    srv_out, srv_sat = serve(True), serve(False)
    plain, plain_sat = plain_run(True), plain_run(False)
    return {
        "metric": "serving pairs/s with p50/p99 request latency (bit-exact)",
        "value": srv_out["pairs_per_s"], "unit": UNIT, "n_gpus": 1, "steps": len(reqs),
        "warmup": 4, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded Poisson arrivals)",
        "config": {"workload": "serving", "rate_req_s": args.rate, "duration_s": args.duration,
                   "requests": len(reqs), "pairs": total_pairs, "slots": args.slots,
                   "short": "1k-64k reads U[100,250] bp x 4 windows (verification)",
                   "long": "50-2000 gap-fill segments U[200,2000] bp, band 256 (banded SW)",
                   "reference_bp": int(len(pool.reference))},
        "server": srv_out, "plain": plain,
        "saturated": {"server_pairs_per_s": srv_sat["pairs_per_s"],
                      "plain_pairs_per_s": plain_sat["pairs_per_s"],
                      "speedup": srv_sat["pairs_per_s"] / plain_sat["pairs_per_s"],
                      "server_batches": srv_sat["batches"],
                      "server_mean_requests_per_batch": srv_sat["mean_requests_per_batch"],
                      "server_host_ms": srv_sat["host_ms"], "server_submit_s": srv_sat["submit_s"]},
        "p99_ratio_plain_over_server": plain["p99_ms"] / srv_out["p99_ms"],
        "p50_ratio_plain_over_server": plain["p50_ms"] / srv_out["p50_ms"]}


def run_gapfill(args, rank, local, world):
    """Long-read gap-fill at the configured size: 20k simulated long reads (lognormal
    length, mean 10 kbp, sd 6 kbp, 1-50 kbp; 5-12 % error at 2:1:1) from a 1 Gbp
    genome with 10 % repeat families, split at exact 15-mer anchors into segments of
    200-2000 bases, each aligned with band 256 (int32 lanes: the scores leave the
    packed int16 range) against the reference between its anchors. One host-API call
    per step over every segment (H2D of the segment bases and descriptors, D2H of
    rows and CIGARs); the trace arena runs in rounds sized by free device memory.
    A sample of segments is checked against the oracle outside the timed region."""
    import torch

    from kira_ls_aligner_b200 import AlignmentConfig, GpuContext, PairBatch, _abi, autotune, synth
    if rank != 0:
        return
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    g = synth.gapfill_reads(args.long_reads)
    gen_s = time.perf_counter() - t0
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    b = PairBatch(pin(g.reads), pin(g.read_off), pin(g.read_len), None, pin(g.win_off),
                  pin(g.win_len), pin(g.band_offset), None, pin(g.bandwidth))
    cfg = AlignmentConfig(1, 4, 6, 1, 256, 100, 5, True, 16)
    ctx = GpuContext(local)
    ctx.ref_upload(g.reference)
    L = _abi.lib()
    # Launch shape of the band-256 class: installed, or autotuned on 4,000 segments
    # drawn across the batch (DP stage time from the library's stage events).
    if args.shape >= 0:
        ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, 256, args.shape))
        tuned = {"best": args.shape, "shape": autotune.shapes()[args.shape], "dp_ms": None}
    else:
        sub = _subset(g, np.linspace(0, g.n_pairs - 1, 4000).astype(np.int64))
        tuned = autotune.tune_bsw_shape(ctx, 256, lambda: ctx.bsw_batch(sub, cfg),
                                        device_name=torch.cuda.get_device_name(local))
    for _ in range(args.warmup):
        res, ops, cells = ctx.bsw_batch(b, cfg)
    ts = [_timed(lambda: ctx.bsw_batch(b, cfg)) for _ in range(args.steps)]
    res, ops, cells = ctx.bsw_batch(b, cfg)
    rounds = int(L.kira_gpu_bsw_rounds(ctx.handle))
    ctx.check(L.kira_gpu_profile(ctx.handle, 1))
    ctx.bsw_batch(b, cfg)
    buf = (C.c_float * 8)()
    k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
    ctx.check(L.kira_gpu_profile(ctx.handle, 0))
    stage = dict(zip(("upload", "bucketing", "bsw_dp", "bsw_traceback", "cigar_compact"),
                     [round(float(x), 3) for x in buf[:k]]))
    ms = sum(ts) / len(ts)
    n = g.n_pairs
    parity = None
    if not args.no_cpu:  # every 37th segment against the oracle's banded_sw_with
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as O
        sel = np.arange(0, n, 37)
        c = O.cfg(1, 4, 6, 1, 256, 100, 5)
        out, cig = O.banded_sw_batch(g.reads, g.read_off[sel].copy(), g.read_len[sel].copy(),
                                     g.reference, g.win_off[sel].copy(), g.win_len[sel].copy(),
                                     g.band_offset[sel].copy(), c, os.cpu_count() or 1, 1024)
        bad = 0
        for t, p in enumerate(sel):
            r = res[p]
            same = all(int(r[f]) == int(out[f][t]) for f in
                       ("score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar",
                        "early_abort"))
            o, m = int(r["cigar_off"]), int(r["n_cigar"])
            if not same or m > 1024 or not np.array_equal(ops[o:o + m], cig[t][:m]):
                bad += 1
        parity = {"checked": int(len(sel)), "mismatches": bad,
                  "fields": ["score", "ref_start", "ref_end", "read_start", "read_end",
                             "n_cigar", "early_abort", "cigar"]}
    print(json.dumps({
        "metric": "pairs/s and GCUPS (long-read gap-fill banded SW with CIGAR, bit-exact)",
        "value": n / (ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
        "config": {"workload": g.name, "long_reads": g.n_reads, "read_bases": g.read_bases,
                   "segments": n, "segment_bases": int(g.read_len.sum()),
                   "segment_len": [int(g.read_len.min()), int(g.read_len.max())],
                   "read_len": "lognormal mean 10 kbp sd 6 kbp, 1-50 kbp",
                   "errors": "U[5%,12%] 2:1:1", "anchors": "exact 15-mers", "band": 256,
                   "reference_bp": int(len(g.reference)), "repeats": "10 %",
                   "path": "resident reference, host API (H2D segments + descriptors, "
                           "D2H rows + CIGARs per call)", "generate_s": round(gen_s, 1)},
        "gcups": cells / (ms / 1e3) / 1e9, "cells": int(cells), "trace_rounds": rounds,
        "autotune": tuned,
        "reads_per_s": g.n_reads / (ms / 1e3), "stage_ms": stage, "parity": parity,
        "checksum": int(res["score"].astype(np.int64).sum())}))
    ctx.close()


def _subset(w, idx):
    """A compact PairBatch of the pairs `idx` of an SwWorkload (own read arena;
    windows stay reference coordinates when the workload's reference is resident)."""
    from kira_ls_aligner_b200 import PairBatch
    rl, wl = w.read_len[idx], w.win_len[idx]
    if w.wins is None:
        reads = np.concatenate([w.reads[int(o):int(o) + int(n)]
                                for o, n in zip(w.read_off[idx], rl)] + [np.zeros(16, np.uint8)])
        ro = np.concatenate([[0], np.cumsum(rl[:-1], dtype=np.uint64)]).astype(np.uint64)
        return PairBatch(reads, ro, rl.copy(), None, w.win_off[idx].copy(), wl.copy(),
                         w.band_offset[idx].copy(), None, w.bandwidth[idx].copy())
    reads = np.concatenate([w.reads[int(o):int(o) + int(n)] for o, n in zip(w.read_off[idx], rl)]
                           + [np.zeros(16, np.uint8)])
    wins = np.concatenate([w.wins[int(o):int(o) + int(n)] for o, n in zip(w.win_off[idx], wl)]
                          + [np.zeros(16, np.uint8)])
    ro = np.concatenate([[0], np.cumsum(rl[:-1], dtype=np.uint64)]).astype(np.uint64)
    wo = np.concatenate([[0], np.cumsum(wl[:-1], dtype=np.uint64)]).astype(np.uint64)
    return PairBatch(reads, ro, rl.copy(), wins, wo, wl.copy(), w.band_offset[idx].copy(), None,
                     w.bandwidth[idx].copy())


def graph_counts(ctx) -> dict:
    from kira_ls_aligner_b200 import _abi
    c, r = C.c_uint64(), C.c_uint64()
    _abi.lib().kira_gpu_set_graphs(ctx.handle, -1, C.byref(c), C.byref(r))
    return {"captures": c.value, "replays": r.value}


def _timed(fn) -> float:
    t = time.perf_counter()
    fn()
    return (time.perf_counter() - t) * 1e3


def relaunch(args) -> int:
    """`--gpus N` without a launcher: run this script under torchrun, one rank per GPU
    (rendezvous on 127.0.0.1); rank 0 prints the line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1", "--master-port",
           str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1 and args.impl == "ours":
        sys.exit(relaunch(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300))
    out = None
    try:
        if args.workload == "uneven":
            out = run_uneven(args, rank, local, world)
        elif args.workload == "serving":
            out = run_serving(args, rank, local, world)
        elif args.workload == "gapfill":
            run_gapfill(args, rank, local, world)
        elif args.workload == "nmmd":
            run_nmmd(args, rank, local, world)
        elif args.workload == "wfa":
            run_wfa(args, rank, local, world)
        elif args.workload == "prefilter":
            run_prefilter(args, rank, local, world)
        elif args.impl == "reference":
            out = run_reference(args, rank, world)
        else:
            out = run_ours(args, rank, local, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


def job_shard(args, rank, world):
    """This rank's contiguous range of the job (world blocks of 8 x reads pairs on one
    reference), cost-balanced by shard.shard_bounds, and its pairs."""
    from kira_ls_aligner_b200 import shard, synth
    block = 8 * args.reads
    n = world * block
    cost = shard.pair_cost(np.full(n, 150, np.uint32), np.full(n, 250, np.uint32), band=33)
    lo, hi = shard.shard_bounds(cost, world)[rank]
    return lo, hi, synth.batched_range(lo, hi, block_pairs=block, ref_len=args.ref_len)


def run_ours(args, rank, local, world, dist):
    lo, hi, w = job_shard(args, rank, world)
    n = w.n_pairs
    if args.dry_run:
        return dry_run(args, rank, world, dist, w, lo, hi)
    import torch

    from kira_ls_aligner_b200 import GpuContext, VerifyParams, _abi, autotune, shard
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    ctx = GpuContext(local)
    L = _abi.lib()
    ctx.ref_upload(w.reference)

    # Device-resident inputs and outputs.
    t_reads = torch.from_numpy(np.concatenate([w.reads, np.zeros(16, np.uint8)])).to(dev)
    t_roff = torch.from_numpy(w.read_off.view(np.int64)).to(dev)
    t_rlen = torch.from_numpy(w.read_len.view(np.int32)).to(dev)
    t_woff = torch.from_numpy(w.win_off.view(np.int64)).to(dev)
    t_wlen = torch.from_numpy(w.win_len.view(np.int32)).to(dev)
    cap = 4 * n
    t_res = torch.empty(n * 32, dtype=torch.uint8, device=dev)
    t_ops = torch.empty(cap, dtype=torch.int32, device=dev)
    t_used = torch.zeros(1, dtype=torch.int64, device=dev)
    t_cells = torch.zeros(1, dtype=torch.int64, device=dev)
    pc = _abi.Pairs()
    pc.n = n
    pc.max_read_len, pc.max_win_len = int(w.read_len.max()), int(w.win_len.max())
    pc.read_seq, pc.read_seq_bytes = t_reads.data_ptr(), int(w.reads.nbytes)
    pc.read_off, pc.read_len = t_roff.data_ptr(), t_rlen.data_ptr()
    pc.win_seq, pc.win_off, pc.win_len = None, t_woff.data_ptr(), t_wlen.data_ptr()
    vp = params.to_c()
    stream = torch.cuda.current_stream(dev)

    def step():
        rc = L.kira_gpu_verify_dev(ctx.handle, C.byref(pc), C.byref(vp), t_res.data_ptr(),
                                   t_ops.data_ptr(), cap, t_used.data_ptr(), None,
                                   t_cells.data_ptr(), C.c_void_p(stream.cuda_stream))
        ctx.check(rc)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    def run_sync():
        step()
        torch.cuda.synchronize(dev)
    if args.shape >= 0:
        ctx.check(L.kira_gpu_set_bsw_shape(ctx.handle, 33, args.shape))
        tuning = {"best": args.shape, "shape": autotune.shapes()[args.shape], "dp_ms": None}
    else:
        tuning = autotune.tune_bsw_shape(ctx, 33, run_sync,
                                         device_name=torch.cuda.get_device_name(dev))
    stage_ms = np.zeros(len(_abi.STAGES))
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)  # let the sampler attach before the timed region
    # keep the GPU busy while the sampler attaches so its first samples see load
    for _ in range(3):
        step()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    total_ms = 0.0
    t_cells.zero_()
    launches = 0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = L.kira_gpu_launch_count()
        e0.record(stream)
        step()
        e1.record(stream)
        launches += L.kira_gpu_launch_count() - c0
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    cells = int(t_cells.item())
    cells_step = cells // max(args.steps, 1)
    # Stage times from the library's stage events, on separate steps after the timed
    # ones (stage timing runs the stages one after another on one stream).
    L.kira_gpu_profile(ctx.handle, 1)
    for _ in range(PROFILED_STEPS):
        flush.zero_()
        step()
        buf = (C.c_float * 8)()
        k = L.kira_gpu_stage_times(ctx.handle, buf, 8)
        stage_ms[:k] += np.array(buf[:k]) * args.steps / PROFILED_STEPS
    L.kira_gpu_profile(ctx.handle, 0)
    total_ms = _max_over_ranks(total_ms, dist, dev)
    ms_per_step = total_ms / args.steps
    value = n * world * args.steps / (total_ms / 1e3)

    # This step's results on the host (outside the timed region).
    res = np.frombuffer(t_res.cpu().numpy().tobytes(), _abi.SW_RESULT_DTYPE)
    used = int(t_used.item())
    ops = t_ops[:used].cpu().numpy().view(np.uint32)
    statuses = np.bincount(res["status"], minlength=4).tolist()

    # e2e through the host API with pinned host inputs.
    e2e = None if args.no_e2e else e2e_run(args, ctx, L, vp, w, n, world, dist, dev)

    # Every rank's results gathered on rank 0 (one collective, outside the timed
    # region), checked against the per-rank checksums.
    gathered = None
    if dist is not None:
        gdev = dev if args.backend == "nccl" else None
        g_res, g_ops = shard.gather_results(res, ops, dist, device=gdev)
        sums = _all_gather_ints([n, int(res["score"].astype(np.int64).sum()), len(ops),
                                 int(ops.astype(np.int64).sum())], dist, gdev)
        if rank == 0:
            ok = (len(g_res) == sum(s[0] for s in sums) and len(g_ops) == sum(s[2] for s in sums)
                  and int(g_res["score"].astype(np.int64).sum()) == sum(s[1] for s in sums)
                  and int(g_ops.astype(np.int64).sum()) == sum(s[3] for s in sums))
            gathered = {"pairs": int(len(g_res)), "cigar_ops": int(len(g_ops)),
                        "checksums_match": bool(ok)}

    # Parity: every pair of this rank's shard against the oracle (all ranks at once,
    # host threads split between them); mismatch counts summed over ranks.
    parity, cpu = None, None
    if not args.no_cpu:
        nthreads = max(1, (os.cpu_count() or 1) // world)
        parity, el = parity_block(res, ops, cells_step, w, nthreads)
        if dist is not None:
            tot = _all_gather_ints([parity["checked"], parity["mismatches"]], dist,
                                   dev if args.backend == "nccl" else None)
            parity["checked_all_ranks"] = sum(t[0] for t in tot)
            parity["mismatches_all_ranks"] = sum(t[1] for t in tot)
        if world == 1:
            cpu = {"value": n / el, "unit": UNIT, "cores": nthreads, "kind": "port",
                   "sample": f"all {n} pairs of the workload, one pass (the parity check's "
                             f"oracle run), {el:.2f} s"}

    roofline = roofline_block(args, L, local, stage_ms, statuses, cells_step, n, tuning)

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        ctx.close()
        ctx = None
        extras = run_extras(args, local)

    if ctx is not None:
        ctx.close()
    if rank != 0:
        return None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded; no public dataset)",
        "config": _config(args, w, world,
                          f"{world} rank(s), one job of {world} x {8 * args.reads} pairs in "
                          f"contiguous cost-balanced shards, no data-path collective"),
        "gcups": cells_step * world / (ms_per_step / 1e3) / 1e9, "cells_per_step": cells_step,
        "autotune": tuning,
        "status_counts": {"certified": statuses[1], "myers_reject": statuses[2],
                          "sw": statuses[3]},
        "parity": parity, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "clocks": clocks, "gpu_launches": int(launches),
        "shard": {"rank0_pairs": [lo, hi], "gathered": gathered},
    }
    out.update(extras)
    return out


def _max_over_ranks(x: float, dist, dev) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _all_gather_ints(vals, dist, dev):
    import torch
    t = torch.tensor(vals, dtype=torch.int64, device=dev)
    parts = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    return [[int(v) for v in p.cpu()] for p in parts]


def e2e_run(args, ctx, L, vp, w, n, world, dist, dev):
    """The same metric through the host API with pinned host buffers: H2D of the
    read arena and pair descriptors, D2H of the results inside the timed region.
    Headline: kira_gpu_verify_batch_compact (a status byte per pair, full rows and
    CIGARs of the aligned pairs); beside it kira_gpu_verify_batch (a 32-byte row for
    every pair)."""
    import torch

    from kira_ls_aligner_b200 import _abi
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    h_reads = pin(np.concatenate([w.reads, np.zeros(16, np.uint8)]))
    h_roff, h_rlen = pin(w.read_off.view(np.int64)), pin(w.read_len.view(np.int32))
    h_woff, h_wlen = pin(w.win_off.view(np.int64)), pin(w.win_len.view(np.int32))
    cap = 4 * n
    res_h = torch.empty(n * 32, dtype=torch.uint8).pin_memory()
    stat_h = torch.empty(n, dtype=torch.uint8).pin_memory()
    ops_h = torch.empty(cap, dtype=torch.int32).pin_memory()
    cb = _abi.CigarBuf(ops_h.data_ptr(), cap, 0)
    hpc = _abi.Pairs()
    hpc.n = n
    hpc.read_seq, hpc.read_seq_bytes = h_reads.data_ptr(), int(w.reads.nbytes)
    hpc.read_off, hpc.read_len = h_roff.data_ptr(), h_rlen.data_ptr()
    hpc.win_seq, hpc.win_off, hpc.win_len = None, h_woff.data_ptr(), h_wlen.data_ptr()
    cells_h, rows_used = C.c_uint64(), C.c_uint64()

    def full_step():
        ctx.check(L.kira_gpu_verify_batch(ctx.handle, C.byref(hpc), C.byref(vp),
                                          res_h.data_ptr(), C.byref(cb), None,
                                          C.byref(cells_h)))

    def compact_step():
        ctx.check(L.kira_gpu_verify_batch_compact(ctx.handle, C.byref(hpc), C.byref(vp),
                                                  stat_h.data_ptr(), res_h.data_ptr(), n,
                                                  C.byref(rows_used), C.byref(cb),
                                                  C.byref(cells_h)))

    def timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        return _max_over_ranks(time.perf_counter() - t0, dist, dev)
    el_full = timed(full_step)
    el = timed(compact_step)
    # Bytes the call copies up: the read arena plus the pair descriptors, packed to
    # 12 bytes a pair (u32 offsets, u16 lengths) when the read arena and the
    # reference are below 4 GiB and every length fits 16 bits, else 24.
    packed = (w.reads.nbytes < 1 << 32 and len(w.reference) < 1 << 32
              and max(int(w.read_len.max()), int(w.win_len.max())) < 1 << 16)
    h2d = int(w.reads.nbytes) + n * (12 if packed else 8 + 4 + 8 + 4)
    tail = 8 + 8 + 16  # op count, cells, flag words
    d2h = n + 32 * int(rows_used.value) + 4 * int(cb.used) + tail + 8
    return {"value": n * world * args.steps / el, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * el / args.steps,
            "api": "kira_gpu_verify_batch_compact",
            "full_rows": {"value": n * world * args.steps / el_full,
                          "ms_per_step": 1e3 * el_full / args.steps,
                          "d2h_bytes_per_step": 32 * n + 4 * int(cb.used) + tail,
                          "api": "kira_gpu_verify_batch"}}


def profile_figure(name: str, key: str):
    """A figure recorded in a committed ncu summary (`key: value` line), or None."""
    import re
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            m = re.search(rf"^{re.escape(key)}:\s*([0-9.eE+-]+)", f.read(), re.M)
        return float(m.group(1)) if m else None
    except OSError:
        return None


PROFILED_STEPS = 5
ALU_PROBES = ("dpx_s16x2_addmax", "iadd3", "lop3", "imad", "lop3+imad", "dpx+imad")


def roofline_block(args, L, local, stage_ms, statuses, cells_step, n, tuning):
    """HBM roofline of the dominant stage (algorithmic bytes / CUDA-event time against
    the measured copy bandwidth) and, beside it, the integer-pipe roofline of the DP
    kernel: the reference recurrence's integer operations per cell (18; 9 on packed
    int16 pairs) at the measured cell rate, against this GPU's integer instruction
    rate measured in the same run (kira_gpu_alu_probe)."""
    from kira_ls_aligner_b200 import _abi, autotune
    peak, peak_kind = measured_peaks()
    dom = int(np.argmax(stage_ms))
    dom_ms = stage_ms[dom] / args.steps
    n_sw = statuses[3]
    n_my = statuses[2] + statuses[3]
    q, wl = 150, 250
    packed = bool(autotune.packed()[tuning["best"]])
    qp, wp = (q + 3) // 4, (wl + 3) // 4
    # Algorithmic bytes per launch of each stage: 2-bit packed sequences and result
    # rows for the sieve and Myers; for the DP the ASCII read and window of every SW
    # pair, its end coordinates, and a 4-bit trace code per executed band cell.
    alg = {0: n * (qp + wp + 12), 1: n_my * (qp + wp + 8), 2: n_sw * (q + wl + 16) + cells_step // 2,
           3: n_sw * (32 + 16) + cells_step // 50, 4: n * (32 + 8) + 4 * n}
    achieved = alg[dom] / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    per_cell = profile_figure("bsw16_dp_batched_800k.md" if packed else "bsw_dp_batched_800k.md",
                              "dram_bytes_per_cell")
    per_pair = profile_figure("verify_filter_batched_800k.md", "dram_bytes_per_pair")
    traffic = {2: None if per_cell is None else per_cell * cells_step,
               0: None if per_pair is None else per_pair * n}.get(dom)
    dp_ms = stage_ms[2] / args.steps
    probes = {}
    for op, name in enumerate(ALU_PROBES):
        v = C.c_double()
        if L.kira_gpu_alu_probe(local, op, 40_000, C.byref(v)) == 0:
            probes[name] = v.value / 1e12
    ops_cell = 9 if packed else 18
    cell_rate = cells_step / (dp_ms / 1e3) if dp_ms > 0 else 0.0
    single = [probes[k] for k in ALU_PROBES[:4] if k in probes]
    ipeak = max(single) if single else None
    return {"bound": "hbm", "kernel": _abi.STAGES[dom], "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "traffic": None if traffic is None
            else int(traffic), "algorithmic_bytes": int(alg[dom]),
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic_source": "ncu DRAM bytes per unit (profiles/), scaled by this run's units",
            "stage_ms_per_step": {s: round(float(t) / args.steps, 4)
                                  for s, t in zip(_abi.STAGES, stage_ms)},
            "int_pipe": {"kernel": "bsw_dp", "gcups": cell_rate / 1e9,
                         "ops_per_cell": ops_cell,
                         "achieved_tops": cell_rate * ops_cell / 1e12,
                         "peak_tops": ipeak, "frac": None if not ipeak
                         else cell_rate * ops_cell / 1e12 / ipeak,
                         "probe_tops": probes,
                         "peak_source": "kira_gpu_alu_probe in this run (fastest single-kind "
                                        "stream: DPX add-max / IADD3 / LOP3 / IMAD)"}}


def run_extras(args, local) -> dict:
    """The batching and serving targets on the same GPU, folded into the headline
    line: the uneven-length batch (bucketed persistent launches + graphs vs one
    launch of the same kernel choice) and a short serving run (p50 / p99 latency,
    server vs one request per call)."""
    import argparse as _ap
    ea = _ap.Namespace(**vars(args))
    ea.steps, ea.warmup = 3, 2
    out = {}
    try:
        u = run_uneven(ea, 0, local, 1)
        out["uneven"] = {"config": u["config"], "pairs_per_s": u["value"],
                         "plain_pairs_per_s": u["plain"]["pairs_per_s"],
                         "speedup_vs_plain": u["speedup_vs_plain"],
                         "bucketed_stage_ms": u["bucketed"]["stage_ms"],
                         "plain_stage_ms": u["plain"]["stage_ms"], "cuda_graphs": u["cuda_graphs"]}
    except Exception as e:  # noqa: BLE001 -- reported, the headline stands
        out["uneven"] = {"error": repr(e)}
    ea.rate, ea.duration = 200.0, 2.0
    try:
        v = run_serving(ea, 0, local, 1)
        out["serving"] = {"config": v["config"], "pairs_per_s": v["value"],
                          "p50_ms": v["server"]["p50_ms"], "p99_ms": v["server"]["p99_ms"],
                          "plain_p50_ms": v["plain"]["p50_ms"],
                          "plain_p99_ms": v["plain"]["p99_ms"],
                          "speedup_vs_plain": v["saturated"]["speedup"],
                          "saturated": v["saturated"]}
    except Exception as e:  # noqa: BLE001
        out["serving"] = {"error": repr(e)}
    return out


def dry_run(args, rank, world, dist, w, lo, hi):
    """The multi-rank plumbing without a GPU: shard, stand-in results, gather on rank
    0, max-over-ranks timing."""
    from kira_ls_aligner_b200 import _abi, shard
    n = w.n_pairs
    res = np.zeros(n, _abi.SW_RESULT_DTYPE)
    res["score"] = (w.win_off % 97).astype(np.int32)
    res["n_cigar"] = 1
    res["cigar_off"] = np.arange(n, dtype=np.uint32)
    ops = (w.read_len.astype(np.uint32) << 4)
    t = time.perf_counter()
    el = _max_over_ranks(time.perf_counter() - t, dist, None)
    gathered = None
    if dist is not None:
        g_res, g_ops = shard.gather_results(res, ops, dist)
        if rank == 0:
            gathered = {"pairs": int(len(g_res)), "cigar_ops": int(len(g_ops)),
                        "offsets_rebased": bool((g_res["cigar_off"] ==
                                                 np.arange(len(g_res))).all())}
    if rank != 0:
        return None
    return {"metric": METRIC, "dry_run": True, "n_gpus": world, "steps": args.steps,
            "shard": {"rank0_pairs": [lo, hi], "gathered": gathered}, "max_s": el}


if __name__ == "__main__":
    main()
