"""WFA on the GPU (kira_gpu_wfa_batch) against the oracle's restatement of
src/alignment/wfa.rs, pair by pair: found, cost, score, text span and CIGAR
identical. Covers the reference's own WFA test corpora (tests/wfa_semi_global.rs,
tests/wfa2_modes.rs, tests/scored_wfa.rs, wfa.rs:965-1129) run through the GPU,
plain and scored costs, exact and adaptive searches, pinned and ends-free leading
text, traceback and score-only, per-pair budgets, router budgets, a resident
reference, and the edge cases (empty read or window, non-ACGT bytes, budgets
below the optimum, refused costs, CIGAR capacity)."""
import numpy as np
import pytest

import pyoracle as O
from test_oracle_wfa import BASES, Lcg, _mutate, _next32, xorshift

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _batch(pairs):
    from kira_ls_aligner_b200 import PairBatch
    return PairBatch.from_pairs([bytes(p) for p, _ in pairs], [bytes(t) for _, t in pairs])


def _gpu(ctx, pairs, params, max_score=None, tbf=None):
    from kira_ls_aligner_b200 import decode_cigar
    res, ops = ctx.wfa_batch(_batch(pairs), params, max_score=max_score, text_begin_free=tbf)
    out = []
    for r in res:
        if not r["found"]:
            out.append(None)
            continue
        cig = decode_cigar(ops[int(r["cigar_off"]):int(r["cigar_off"]) + int(r["n_cigar"])])
        out.append((int(r["cost"]), int(r["score"]), int(r["text_start"]), int(r["text_end"]),
                    [(n, c) for n, c in cig]))
    return out


def _want(pairs, params, max_score=None, tbf=None):
    out = []
    for i, (p, t) in enumerate(pairs):
        ms = params.max_score if max_score is None else int(max_score[i])
        if ms < 0 and max_score is None:  # router::wfa_score_budget
            pct = 25 if params.budget_pct < 0 else params.budget_pct
            x = params.mismatch + (params.match_score if params.scored else 0)
            e = params.gap_extend + (params.match_score if params.scored else 0)
            ms = max(len(p) * pct // 100 * x, (params.gap_open + e * 4) * 3)
        c = O.wfa_cfg(params.mismatch, params.gap_open, params.gap_extend, ms,
                      params.adaptive_drop, params.text_begin_free if tbf is None else int(tbf[i]),
                      params.match_score, params.scored, params.traceback)
        r = O.wfa(bytes(p), bytes(t), c)
        if r is None:
            out.append(None)
            continue
        score = len(p) * params.match_score - r.score if params.scored else r.score
        out.append((r.score, score, r.text_start if params.traceback else 0, r.text_end, r.cigar))
    return out


def _check(ctx, pairs, params, max_score=None, tbf=None):
    got = _gpu(ctx, pairs, params, max_score, tbf)
    want = _want(pairs, params, max_score, tbf)
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == w, (i, pairs[i], g, w)
    return got


def _pen(**kw):
    from kira_ls_aligner_b200 import WfaParams
    return WfaParams(4, 6, 1, **kw)


# --- the reference's corpora ------------------------------------------------------

def _semi_global_pairs():
    pairs = [(b"ACGTACGT", b"ACGTACGTAA"), (b"ACGTACGT", b"ACATACGT"), (b"ACGTACGT", b"ACGACGT"),
             (b"ACGACGT", b"ACGTACGT"), (b"AAAAAAAA", b"TTTTTTTT")]
    rng = [0xC0FFEE]
    for _ in range(50):
        m = 20 + xorshift(rng) % 80
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = _mutate(rng, pattern, xorshift(rng) % 4)
        for _ in range(5):
            text.append(BASES[xorshift(rng) % 4])
        pairs.append((pattern, bytes(text)))
    rng = Lcg(0x1234_5678_9ABC_DEF0)
    text = bytes(rng.base() for _ in range(260))
    for prefix in (110, 120, 130, 134, 140, 145, 148, 149, 150):
        for tail in (1, 2, 3, 4, 6, 8, 12, 16, 20):
            read = bytearray(text[:prefix])
            for _ in range(tail):
                read.append(rng.base())
            pairs.append((bytes(read), text))
    pairs.append((b"ATAGTCGAGCAGGTAATAACGCCCTTCGTGGCGGAACACCAGGTCGATAAAGCCTTTTAACATGCCACGTACCTGC"
                  b"ATGAACTCCAGCGGCGGGCAGCCTGCGGATAGCGGGGCAAAATGGCGGATTAAAGTATAAAACCGCCTGGGGGT",
                  b"ATAGTCGAGCAGGTAATAACGCCCTTCGTGGCGGAACACCAGGTCGATAAAGCCTTTTAACATGCCACGTACCTGC"
                  b"ATGAACTCCAGCGGCGGGCAGCCTGCGGATAGCGGGTCAAACTGGCGGATTAACGTATCAAGCTGACTGGCGATAA"
                  b"GCGGTTCACTAATCGGCAGATAAAACTCCATCTCCACCTGTTTATTGC"))
    return pairs


def _modes_pairs(seed, n, m_lo, m_span, errs, kinds=3, tail=6):
    rng = [seed]
    pairs = []
    for _ in range(n):
        m = m_lo + xorshift(rng) % m_span
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = _mutate(rng, pattern, xorshift(rng) % errs, kinds)
        for _ in range(tail):
            text.append(BASES[xorshift(rng) % 4])
        pairs.append((pattern, bytes(text)))
    return pairs


@pytest.mark.parametrize("traceback", [True, False])
def test_reference_corpora(ctx, traceback):
    pairs = _semi_global_pairs()
    budgets = np.array([20] * 4 + [5] + [80] * 50 + [400] * 81 + [150], np.int32)
    got = _check(ctx, pairs, _pen(traceback=traceback), max_score=budgets)
    assert got[0][:4] == (0, 0, 0, 8) and got[4] is None
    if traceback:
        assert got[0][4] == [(8, "M")]
        assert got[-1] == (34, 34, 0, 134, [(134, "M"), (16, "I")])
    got = _check(ctx, pairs, _pen(traceback=traceback), max_score=np.full(len(pairs), 14, np.int32))
    assert got[4][0] == 14
    # tests/wfa2_modes.rs corpora: budgets 8 / 30 / 200, adaptive drops 50 and 3
    sp = _modes_pairs(0x9E37_79B9, 200, 20, 120, 6, tail=5)
    for budget in (8, 30, 200):
        _check(ctx, sp, _pen(max_score=budget, traceback=traceback))
    ap = _modes_pairs(0xBADC0FFE, 60, 40, 100, 4)
    exact = _check(ctx, ap, _pen(max_score=200, traceback=traceback))
    wide = _check(ctx, ap, _pen(max_score=200, adaptive_drop=50, traceback=traceback))
    assert [e[0] for e in exact] == [w[0] for w in wide]
    tp = _modes_pairs(0x1357_9BDF, 40, 50, 80, 5, kinds=1)
    _check(ctx, tp, _pen(max_score=400, adaptive_drop=3, traceback=traceback))


def test_ends_free(ctx):
    pattern = b"ACGTACGTACGTACGT"
    text = b"TTTTT" + pattern + b"GG"
    got = _check(ctx, [(pattern, text)] * 2, _pen(max_score=200), tbf=np.array([0, 5], np.int32))
    assert got[0][:3] == (11, 11, 0)
    assert got[1] == (0, 0, 5, 21, [(16, "M")])


def test_scored_corpus(ctx):
    # tests/scored_wfa.rs:88-121 through the GPU: three cost sets, leading free
    # text 0..4 per pair, budget 300 and loss - 1 (None for every pair).
    from kira_ls_aligner_b200 import WfaParams
    rng = [0x6A09E667F3BCC909]
    groups = {0: [], 1: [], 2: []}
    for trial in range(1800):
        qlen = 1 + _next32(rng) % 28
        rlen = 1 + _next32(rng) % 35
        q = bytes(BASES[_next32(rng) % 4] for _ in range(qlen))
        r = bytes(BASES[_next32(rng) % 4] for _ in range(rlen))
        groups[trial % 3].append((q, r, _next32(rng) % 5))
    for g, (a, b, o, e) in enumerate(((1, 4, 6, 1), (2, 3, 2, 1), (3, 2, 0, 2))):
        pairs = [(q, r) for q, r, _ in groups[g]]
        tbf = np.array([lead for _, _, lead in groups[g]], np.int32)
        for tb in (True, False):
            p = WfaParams(b, o, e, max_score=300, scored=True, match_score=a, traceback=tb)
            got = _check(ctx, pairs, p, tbf=tbf)
            assert all(x is not None for x in got)
            below = np.array([x[0] - 1 for x in got], np.int32)
            again = _gpu(ctx, pairs, p, max_score=below, tbf=tbf)
            assert all(x is None for x, c in zip(again, got) if c[0] > 0)


# --- the cascade workload -----------------------------------------------------------

@pytest.mark.parametrize("drop,tbf,traceback,lanes", [
    (None, 0, True, 0), (None, 0, False, 0), (50, 0, True, 0), (None, 5, True, 0),
    (8, 3, False, 0), (None, 0, True, 16), (None, 0, True, 32), (50, 2, False, 32),
    (3, 0, True, 16)])
def test_cascade_workload(ctx, drop, tbf, traceback, lanes):
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch, WfaParams, _abi, synth
    ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, lanes))
    w = synth.wfa_cascade(3000, seed=0x51 + tbf, err_hi=0.08, ref_len=400_000)
    ref = w.reference
    pairs = [(w.reads[int(w.read_off[i]):int(w.read_off[i]) + int(w.read_len[i])].tobytes(),
              ref[int(w.win_off[i]):int(w.win_off[i]) + int(w.win_len[i])].tobytes())
             for i in range(w.n_pairs)]
    p = WfaParams.scored_from(AlignmentConfig(), adaptive_drop=drop, text_begin_free=tbf,
                              traceback=traceback)
    got = _check(ctx, pairs, p)
    assert sum(x is not None for x in got) > 0.9 * len(got)
    if traceback:
        assert any(len(x[4]) > 1 for x in got if x)
    # the same pairs with windows read from the resident reference
    ctx.ref_upload(ref)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, w.win_off, w.win_len)
    res, ops = ctx.wfa_batch(b, p)
    res2, ops2 = ctx.wfa_batch(_batch(pairs), p)
    ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, 0))
    assert np.array_equal(res, res2) and np.array_equal(ops, ops2)


def test_edge_cases(ctx):
    alpha = b"ACGTNacgtRY="
    rng = np.random.default_rng(7)
    pairs = [(b"", b"ACGT"), (b"", b""), (b"ACGT", b""), (b"A", b"A"), (b"A", b"C"),
             (b"ACGTTT", b"AC"), (b"NNNN", b"NNNN"), (b"acgt", b"ACGT")]
    for _ in range(300):
        m = int(rng.integers(1, 60))
        p = bytes(alpha[int(i)] for i in rng.integers(0, len(alpha), m))
        t = bytearray(p[int(rng.integers(0, m)):]) + bytes(
            alpha[int(i)] for i in rng.integers(0, len(alpha), int(rng.integers(0, 40))))
        if len(t) and rng.random() < 0.5:
            t[int(rng.integers(0, len(t)))] = ord("G")
        pairs.append((p, bytes(t)))
    for tb in (True, False):
        for ms in (-1, 0, 3, 60, 100000):
            _check(ctx, pairs, _pen(max_score=ms, traceback=tb))
        _check(ctx, pairs, _pen(max_score=100, adaptive_drop=0, traceback=tb))
        _check(ctx, pairs, _pen(max_score=100, text_begin_free=1000, traceback=tb))
    got = _gpu(ctx, pairs[:3], _pen(max_score=10))
    assert got[0] == (0, 0, 0, 0, []) and got[1] == (0, 0, 0, 0, [])
    assert got[2] == (10, 10, 0, 0, [(4, "I")])


@pytest.mark.parametrize("lanes", [0, 8])
def test_long_reads(ctx, lanes):
    from kira_ls_aligner_b200 import _abi, synth
    ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, lanes))
    w = synth.gapfill(n_segments=60, seed=0x77, seg_lo=400, seg_hi=1500, err_lo=0.01,
                      err_hi=0.03, ref_len=2_000_000)
    pairs = []
    for i in range(w.n_pairs):
        q = w.reads[int(w.read_off[i]):int(w.read_off[i]) + int(w.read_len[i])].tobytes()
        s = int(w.win_off[i]) + int(w.band_offset[i])
        pairs.append((q, w.reference[s:s + len(q) + 64].tobytes()))
    try:
        for tb in (True, False):
            got = _check(ctx, pairs, _pen(max_score=400, traceback=tb))
            assert sum(x is not None for x in got) > 10
    finally:
        ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, 0))


def test_refused_costs_and_capacity(ctx):
    from kira_ls_aligner_b200 import CapacityError, InvalidArgument, WfaParams, _abi
    pairs = _semi_global_pairs()[:20]
    res, ops = ctx.wfa_batch(_batch(pairs), WfaParams(4, 6, 1, max_score=50, scored=True,
                                                      match_score=0))
    assert (res["found"] == 0).all() and (res["cost"] == -1).all() and len(ops) == 0
    with pytest.raises(InvalidArgument):
        ctx.wfa_batch(_batch(pairs), WfaParams(0, 6, 1, max_score=50))
    with pytest.raises(InvalidArgument):
        ctx.wfa_batch(_batch(pairs), WfaParams(4, 6, 0, max_score=50))
    with pytest.raises(CapacityError):
        ctx.wfa_batch(_batch(pairs), _pen(max_score=50), cigar_cap=3)
    with pytest.raises(Exception) as ei:
        ctx.wfa_batch(_batch([(b"A" * 30001, b"A")]), _pen(max_score=5))
    assert "ReadTooLong" in str(ei.value) or "30000" in str(ei.value)
    del _abi


@pytest.mark.parametrize("traceback", [True, False])
def test_chunked_host_path(ctx, traceback):
    # Host batches of several chunks (uploads / kernels / downloads overlapped, CIGAR
    # offsets through the running total) equal the one-shot call; per-pair budgets
    # and leading free text are sliced with the chunks.
    from kira_ls_aligner_b200 import AlignmentConfig, PairBatch, WfaParams, _abi, synth
    w = synth.wfa_cascade(90_000, seed=0x5CA1, err_hi=0.06, ref_len=3_000_000)
    rng = np.random.default_rng(4)
    ms = rng.integers(5, 120, w.n_pairs).astype(np.int32)
    tbf = rng.integers(0, 6, w.n_pairs).astype(np.int32)
    ref = w.reference
    b = PairBatch(w.reads, w.read_off, w.read_len, ref, w.win_off, w.win_len)
    p = WfaParams.scored_from(AlignmentConfig(), traceback=traceback)
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 0))
        one = ctx.wfa_batch(b, p, max_score=ms, text_begin_free=tbf)
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 32768))
        many = ctx.wfa_batch(b, p, max_score=ms, text_begin_free=tbf)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    assert np.array_equal(one[0], many[0]) and np.array_equal(one[1], many[1])
    sel = list(range(0, w.n_pairs, 97))
    pairs = [(w.reads[int(w.read_off[i]):int(w.read_off[i]) + 150].tobytes(),
              ref[int(w.win_off[i]):int(w.win_off[i]) + int(w.win_len[i])].tobytes()) for i in sel]
    want = _want(pairs, p, max_score=ms[sel], tbf=tbf[sel])
    from kira_ls_aligner_b200 import decode_cigar
    res, ops = many
    for j, i in enumerate(sel):
        r = res[i]
        got = None
        if r["found"]:
            cig = decode_cigar(ops[int(r["cigar_off"]):int(r["cigar_off"]) + int(r["n_cigar"])])
            got = (int(r["cost"]), int(r["score"]), int(r["text_start"]), int(r["text_end"]),
                   [(a, c) for a, c in cig])
        assert got == want[j], i


@pytest.mark.parametrize("traceback", [True, False])
def test_wide_window_and_fallbacks(ctx, traceback):
    # Costs with a free gap open and unit extends: 64 diagonals cover fewer than 32
    # scores, so the window kernel uses 128 diagonals (exact up to score 63), and
    # pairs still open then go through the general kernel's fallback list. Every
    # result equals the oracle; the general kernel alone (lanes 32) agrees too.
    from kira_ls_aligner_b200 import WfaParams, _abi, synth
    w = synth.wfa_cascade(3000, seed=0x64D, err_hi=0.3, ref_len=400_000)
    ref = w.reference
    pairs = [(w.reads[int(w.read_off[i]):int(w.read_off[i]) + 150].tobytes(),
              ref[int(w.win_off[i]):int(w.win_off[i]) + int(w.win_len[i])].tobytes())
             for i in range(w.n_pairs)]
    p = WfaParams(2, 0, 1, max_score=120, traceback=traceback)
    got = _check(ctx, pairs, p)
    costs = [x[0] for x in got if x is not None]
    assert max(costs) > 63 and min(costs) < 20  # both the window and the fallback ran
    ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, 32))
    try:
        assert _gpu(ctx, pairs, p) == got
    finally:
        ctx.check(_abi.lib().kira_gpu_set_wfa_lanes(ctx.handle, 0))
