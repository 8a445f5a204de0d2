"""Composed verification (sieve -> certificate -> Myers -> banded SW) on the GPU
vs the oracle's verify_pair on the same seeded pairs: per-pair status, sieve and
Myers details, score, end coordinates and CIGAR, bit-exact."""
import os

import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
NTHREADS = os.cpu_count() or 4


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _oracle(w, arena, woffs, params, sel=None):
    idx = np.arange(w.n_pairs) if sel is None else sel
    c = params.cfg
    op = O.verify_params(O.cfg(c.match_score, c.mismatch, c.gap_open, c.gap_extend, c.bandwidth,
                               c.xdrop, c.clip_penalty), params.sieve_threshold, params.myers_k,
                         adaptive=c.adaptive, max_drift=c.max_drift,
                         cert_strict=params.cert_strict)
    cap = 512
    out, cig = O.verify_batch(w.reads, w.read_off[idx].copy(), w.read_len[idx].copy(), arena,
                              woffs[idx].copy(), w.win_len[idx].copy(), op, NTHREADS, cap)
    return out, cig


def _compare(res, ops, det, out, cig, sel):
    for k, p in enumerate(sel):
        r, o = res[p], out[k]
        assert r["status"] == o["status"], (p, r, o)
        assert det[p]["sieve_shift"] == o["sieve_shift"], p
        assert det[p]["sieve_mism"] == o["sieve_mism"], p
        assert det[p]["sieve_second"] == o["sieve_second"], p
        assert det[p]["myers_dist"] == o["myers_dist"], p
        assert det[p]["myers_end"] == o["myers_end"], p
        got = (r["score"], r["ref_start"], r["ref_end"], r["read_start"], r["read_end"],
               r["n_cigar"], r["early_abort"])
        want = (o["score"], o["ref_start"], o["ref_end"], o["read_start"], o["read_end"],
                o["n_cigar"], o["early_abort"])
        assert got == want, (p, got, want)
        a = int(r["cigar_off"])
        assert np.array_equal(ops[a:a + int(r["n_cigar"])], cig[k][: int(o["n_cigar"])]), p


def _run(ctx, w, params, host_windows=True):
    from kira_ls_aligner_b200 import PairBatch
    arena, woffs = w.windows_arena()
    if host_windows:
        b = PairBatch(w.reads, w.read_off, w.read_len, arena, woffs, w.win_len)
    else:
        ctx.ref_upload(w.reference)
        b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    res, ops, det, cells = ctx.verify_batch(b, params, detail=True)
    return res, ops, det, cells, arena, woffs


def test_small_config_all_pairs(ctx):
    from kira_ls_aligner_b200 import VerifyParams, synth
    w = synth.small()
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    res, ops, det, cells, arena, woffs = _run(ctx, w, params)
    out, cig = _oracle(w, arena, woffs, params)
    _compare(res, ops, det, out, cig, np.arange(w.n_pairs))
    assert cells == int(out["cells"].sum())
    # Every status occurs in this workload.
    assert {1, 2, 3} <= set(np.unique(res["status"]).tolist())


def test_resident_reference_equals_host_windows(ctx):
    from kira_ls_aligner_b200 import VerifyParams, synth
    w = synth.make_workload("t", 3000, 200_000, cands=6, sub_lo=0.0, sub_hi=0.03, seed=99)
    params = VerifyParams(sieve_threshold=-1, myers_k=-1, cert_strict=True)
    a = _run(ctx, w, params, host_windows=True)
    b = _run(ctx, w, params, host_windows=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
    sel = np.arange(0, w.n_pairs, 3)
    out, cig = _oracle(w, a[4], a[5], params, sel)
    _compare(a[0], a[1], a[2], out, cig, sel)


@pytest.mark.parametrize("myers_k,sub_hi,indel", [(8, 0.05, 0.002), (-1, 0.08, 0.004),
                                                  (2, 0.02, 0.001), (30, 0.10, 0.005)])
def test_qgram_prefilter_changes_nothing(ctx, myers_k, sub_hi, indel):
    # The 4-gram filter only removes pairs Myers rejects: on/off give identical
    # statuses, details, scores and CIGARs (and match the oracle on a sample).
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, synth
    w = synth.make_workload("q", 2500, 400_000, cands=8, sub_lo=0.0, sub_hi=sub_hi,
                            indel_rate=indel, repeat_frac=0.2, seed=1000 + max(myers_k, 0))
    arena, woffs = w.windows_arena()
    b = PairBatch(w.reads, w.read_off, w.read_len, arena, woffs, w.win_len)
    on = ctx.verify_batch(b, VerifyParams(sieve_threshold=12, myers_k=myers_k), detail=True)
    off = ctx.verify_batch(b, VerifyParams(sieve_threshold=12, myers_k=myers_k,
                                           qgram_filter=False), detail=True)
    assert np.array_equal(on[0], off[0]) and np.array_equal(on[1], off[1])
    assert np.array_equal(on[2], off[2]) and on[3] == off[3]
    assert (on[0]["status"] == 2).sum() > 0
    sel = np.arange(0, w.n_pairs, 11)
    out, cig = _oracle(w, arena, woffs, VerifyParams(sieve_threshold=12, myers_k=myers_k), sel)
    _compare(on[0], on[1], on[2], out, cig, sel)


@pytest.mark.parametrize("myers_k,thr,sub_hi,indel", [(8, 12, 0.05, 0.002), (0, 12, 0.02, 0.0),
                                                      (1, 3, 0.03, 0.001), (-1, -1, 0.08, 0.004),
                                                      (30, 2, 0.10, 0.005)])
def test_filter_first_sieve_equals_full_sieve(ctx, myers_k, thr, sub_hi, indel):
    # Without detail rows the 4-gram count runs first and the sieve only for the
    # pairs it leaves open (k = 0 or 1 puts the certificate's bound below the
    # filter's, so some pairs are tagged "reject unless certified"). Results equal
    # the detail path, which sieves every pair, in one shot and in chunks, and the
    # oracle on a sample; reads and windows carry some N bases.
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, _abi, synth
    w = synth.make_workload("f", 2500, 400_000, cands=8, sub_lo=0.0, sub_hi=sub_hi,
                            indel_rate=indel, repeat_frac=0.2, seed=3000 + max(myers_k, 0))
    rng = np.random.default_rng(7)
    reads = w.reads.copy()
    for r in rng.choice(2500, 40, replace=False):
        reads[int(w.read_off[8 * r]) + int(rng.integers(0, 150))] = ord("N")
    arena, woffs = w.windows_arena()
    arena = arena.copy()
    arena[rng.choice(len(arena), 60, replace=False)] = ord("N")
    w.reads = reads
    b = PairBatch(reads, w.read_off, w.read_len, arena, woffs, w.win_len)
    params = VerifyParams(sieve_threshold=thr, myers_k=myers_k)
    full = ctx.verify_batch(b, params, detail=True)
    fast = ctx.verify_batch(b, params)
    assert np.array_equal(full[0], fast[0]) and np.array_equal(full[1], fast[1])
    assert full[3] == fast[3]
    st = np.bincount(fast[0]["status"], minlength=4)
    assert st[1] > 0 and st[2] > 0, st
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 3000))
        chunked = ctx.verify_batch(b, params)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    assert np.array_equal(full[0], chunked[0]) and np.array_equal(full[1], chunked[1])
    sel = np.arange(0, w.n_pairs, 17)
    out, cig = _oracle(w, arena, woffs, params, sel)
    _compare(fast[0], fast[1], full[2], out, cig, sel)


@pytest.mark.parametrize("resident,shuffle", [(False, False), (True, False), (True, True)])
def test_chunked_host_path_equals_one_shot(ctx, resident, shuffle):
    # kira_gpu_verify_batch in chunks (copy-in / compute / copy-out streams, read
    # arena and planes uploaded as far as each chunk needs) == the one-shot path.
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, _abi, synth
    w = synth.make_workload("c", 9000, 500_000, cands=4, sub_lo=0.0, sub_hi=0.04, seed=77)
    arena, woffs = w.windows_arena()
    idx = np.arange(w.n_pairs)
    if shuffle:
        idx = np.random.default_rng(5).permutation(w.n_pairs)
    if resident:
        ctx.ref_upload(w.reference)
        b = PairBatch(w.reads, w.read_off[idx].copy(), w.read_len[idx].copy(), None,
                      w.win_off[idx].copy(), w.win_len[idx].copy())
    else:
        b = PairBatch(w.reads, w.read_off[idx].copy(), w.read_len[idx].copy(), arena,
                      woffs[idx].copy(), w.win_len[idx].copy())
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 0))
        one = ctx.verify_batch(b, params, detail=True)
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 3000))
        chunked = ctx.verify_batch(b, params, detail=True)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    assert np.array_equal(one[0], chunked[0]) and np.array_equal(one[1], chunked[1])
    assert np.array_equal(one[2], chunked[2]) and one[3] == chunked[3]
    sel = np.arange(0, w.n_pairs, 13)
    out, cig = _oracle(w, arena, woffs, params, np.asarray(idx)[sel])
    _compare(chunked[0], chunked[1], chunked[2], out, cig, sel)


def test_chunked_host_path_rejects_out_of_range_pair(ctx):
    # A pair in a later chunk whose read lies outside the arena fails the whole
    # call with InvalidArgument (after the earlier chunks drain), and the context
    # keeps working.
    from kira_ls_aligner_b200 import InvalidArgument, PairBatch, VerifyParams, _abi, synth
    w = synth.make_workload("e", 2000, 200_000, cands=4, seed=78)
    arena, woffs = w.windows_arena()
    roff = w.read_off.copy()
    roff[6500] = len(w.reads) + 10
    bad = PairBatch(w.reads, roff, w.read_len, arena, woffs, w.win_len)
    good = PairBatch(w.reads, w.read_off, w.read_len, arena, woffs, w.win_len)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 1000))
        with pytest.raises(InvalidArgument):
            ctx.verify_batch(bad, params)
        res, ops, _, _ = ctx.verify_batch(good, params)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    ref = ctx.verify_batch(good, params)
    assert np.array_equal(res, ref[0]) and np.array_equal(ops, ref[1])


def test_chunked_host_checks_in_sub_ranges(ctx):
    # Chunks of 140k pairs are checked in 2^14-pair sub-ranges on the context's host
    # threads, and alternate between two compute streams: results equal the
    # one-shot path, and a bad pair in the middle of a later chunk still fails the
    # call with InvalidArgument.
    from kira_ls_aligner_b200 import InvalidArgument, PairBatch, VerifyParams, _abi, synth
    w = synth.make_workload("s", 80_000, 2_000_000, cands=4, sub_lo=0.0, sub_hi=0.03, seed=79)
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 0))
        one = ctx.verify_batch(b, params)
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 140_000))
        chunked = ctx.verify_batch(b, params)
        woff = w.win_off.copy()
        woff[140_000 + 70_000] = len(w.reference)
        bad = PairBatch(w.reads, w.read_off, w.read_len, None, woff, w.win_len)
        with pytest.raises(InvalidArgument) as ei:
            ctx.verify_batch(bad, params)
        assert "pair 210000" in str(ei.value)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    assert np.array_equal(one[0], chunked[0]) and np.array_equal(one[1], chunked[1])


def test_uneven_automatic_chunks(ctx):
    # Batches of at least 2^20 pairs go in chunks of 1/8, 1/4, 1/4, 1/4, 1/8 of the batch
    # by default; results equal the one-shot path.
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, _abi, synth
    w = synth.make_workload("u", 270_000, 5_000_000, cands=4, sub_lo=0.0, sub_hi=0.03, seed=80)
    assert w.n_pairs >= 1 << 20
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 0))
        one = ctx.verify_batch(b, params)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    auto = ctx.verify_batch(b, params)
    assert np.array_equal(one[0], auto[0]) and np.array_equal(one[1], auto[1]) and one[3] == auto[3]


def _compare_all(res, ops, det, out, cig):
    """Vectorised form of _compare over every pair (rows, details and CIGAR ops)."""
    for f in ("status", "score", "ref_start", "ref_end", "read_start", "read_end", "n_cigar",
              "early_abort"):
        bad = np.nonzero(res[f].astype(np.int64) != out[f].astype(np.int64))[0]
        assert len(bad) == 0, (f, bad[:5], res[bad[:1]], out[bad[:1]])
    if det is not None:
        for f in ("sieve_shift", "sieve_mism", "sieve_second", "myers_dist", "myers_end"):
            bad = np.nonzero(det[f].astype(np.int64) != out[f].astype(np.int64))[0]
            assert len(bad) == 0, (f, bad[:5])
    n = res["n_cigar"].astype(np.int64)
    sel = np.nonzero(n)[0]
    cnt = n[sel]
    pair = np.repeat(sel, cnt)
    t = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    got = ops[res["cigar_off"][pair].astype(np.int64) + t]
    bad = np.nonzero(got != cig[pair, t])[0]
    assert len(bad) == 0, ("cigar", np.unique(pair[bad])[:5])


def test_batched_config_200k_all_pairs(ctx):
    """The benchmark's own generator (100 Mbp with 5 % repeat families, 8 candidate
    windows per read, seed 0xB200): 200k pairs, every pair against the oracle, in
    the detail form and in the filter-first form the benchmark times."""
    from kira_ls_aligner_b200 import PairBatch, VerifyParams, synth
    w = synth.batched(n_reads=25_000)
    params = VerifyParams(sieve_threshold=12, myers_k=8)
    c = params.cfg
    op = O.verify_params(O.cfg(c.match_score, c.mismatch, c.gap_open, c.gap_extend, c.bandwidth,
                               c.xdrop, c.clip_penalty), 12, 8)
    out, cig = O.verify_batch(w.reads, w.read_off, w.read_len, w.reference, w.win_off, w.win_len,
                              op, NTHREADS, 64)
    assert int(out["n_cigar"].max()) <= 64
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    res, ops, det, cells = ctx.verify_batch(b, params, detail=True)
    _compare_all(res, ops, det, out, cig)
    assert cells == int(out["cells"].sum())
    res2, ops2, _, cells2 = ctx.verify_batch(b, params)
    _compare_all(res2, ops2, None, out, cig)
    assert cells2 == cells
    counts = np.bincount(res["status"], minlength=4)
    assert counts[1] > 0 and counts[2] > 0 and counts[3] > 0
