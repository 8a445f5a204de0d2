"""The ungapped prefilter and exact matches on the GPU (kira_gpu_prefilter_batch,
kira_gpu_exact_match_batch) against the oracle's restatement of
src/alignment/prefilter.rs and mod.rs:779-832, chain by chain: result, reason,
UngappedStats, NM, MD:Z and CIGAR identical. Covers the reference's own cases
(tests/prefilter_accept.rs, tests/md_format.rs), a seeded stage-4 corpus over a
resident contig under several configurations, and the edge cases."""
import numpy as np
import pytest

import pyoracle as O

pytestmark = pytest.mark.gpu
READ150 = b"ACGT" * 37 + b"AC"


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _ocfg(cfg):
    return O.prefilter_cfg(cfg.match_score, cfg.mismatch, cfg.xdrop, cfg.accept_enable,
                           cfg.accept_only_top1, cfg.accept_span_slack, cfg.accept_min_identity,
                           cfg.accept_max_mismatches, cfg.accept_require_score_margin,
                           cfg.long_read_threshold, cfg.multi_alignments_enabled, cfg.tail,
                           None if cfg.min_identity_x10000 < 0 else cfg.min_identity_x10000)


def _want(read, ref, chain, cfg, top1, margin):
    if cfg.exact_first and O.exact_match_exists(read, ref, chain):
        n = len(read)
        return ("exact", "accept", None, O.identical_nm(read), str(n), [(n, "M")],
                (0, chain[0], cfg.match_score * n))
    r = O.prefilter(read, ref, chain, _ocfg(cfg), top1, margin)
    span = None
    if r.result == "accept":
        span = (r.metrics[5], r.metrics[6], r.metrics[4])
    return (r.result, r.reason, r.metrics, r.nm, r.md, r.cigar, span)


def _got(res, ops, md, i):
    from kira_ls_aligner_b200 import decode_cigar
    r = res[i]
    kinds = ("accept", "reject", "fallback", "exact")
    reason = O.PREFILTER_REASONS[r["reason"]]
    if r["reason"] == 9:
        reason = O.PREFILTER_OTHER[r["other"]]
    met = None
    if r["has_metrics"]:
        met = (int(r["len"]), int(r["mism"]), int(r["matches"]), int(r["identity_x10000"]),
               int(r["score"]), int(r["read_start"]), int(r["ref_start"]))
    kind = kinds[r["result"]]
    if kind in ("accept", "exact"):
        cig = decode_cigar(ops[int(r["cigar_off"]):int(r["cigar_off"]) + int(r["n_cigar"])])
        text = md[int(r["md_off"]):int(r["md_off"]) + int(r["md_len"])].tobytes().decode()
        return (kind, reason, met, int(r["nm"]), text, [(a, b) for a, b in cig],
                (int(r["read_start"]), int(r["ref_start"]), int(r["score"])))
    return (kind, reason, met, 0, "", None, None)


def _run(ctx, reads, refs, chains, cfg, top1=None, margin=None):
    from kira_ls_aligner_b200 import PairBatch, _abi
    b = PairBatch.from_pairs(reads, refs)
    ch = np.array([tuple(c) for c in chains], _abi.CHAIN_DTYPE)
    res, ops, md = ctx.prefilter_batch(b, ch, cfg, is_top1=top1, score_margin=margin)
    for i in range(len(reads)):
        t = 1 if top1 is None else int(top1[i])
        m = 2**31 - 1 if margin is None else int(margin[i])
        want = _want(bytes(reads[i]), bytes(refs[i]), tuple(chains[i]), cfg, t, m)
        assert _got(res, ops, md, i) == want, (i, chains[i])
    return res


def test_reference_cases(ctx):
    from kira_ls_aligner_b200 import PrefilterConfig
    cfg = PrefilterConfig(xdrop=50, accept_span_slack=5, accept_min_identity=98.0,
                          accept_max_mismatches=2, long_read_threshold=300, exact_first=False)
    one = bytearray(READ150)
    one[10] = ord("T")
    reads = [READ150, b"A" * 400, b"A" * 400, b"A" * 150, b"A" * 400]
    refs = [bytes(one), b"T" * 400, b"T" * 400, b"T" * 150, b"T" * 400]
    chains = [(0, 150, 0, 150), (0, 44, 0, 44), (0, 400, 0, 400), (0, 150, 0, 150),
              (0, 400, 0, 400)]
    res = _run(ctx, reads, refs, chains, cfg, top1=np.array([1, 1, 0, 1, 1], np.uint8))
    assert list(res["result"]) == [0, 1, 2, 2, 2]
    assert list(res["reason"]) == [0, 5, 3, 6, 2]
    # tests/md_format.rs: canonical MD of accepted spans, ambiguity codes, exact match
    md_cfg = PrefilterConfig(xdrop=50, accept_span_slack=15, accept_min_identity=98.0,
                             accept_max_mismatches=5, long_read_threshold=300, exact_first=False)
    variants = []
    for edits in ([], [10], [5, 99], [149], [0]):
        ref = bytearray(READ150)
        for e in edits:
            ref[e] = ord("T") if ref[e] != ord("T") else ord("A")
        variants.append(bytes(ref))
    longer = bytearray(b"ACGT" * 38)
    longer[70] = ord("N")
    reads = [READ150] * 5 + [bytes(longer)]
    refs = variants + [bytes(longer)]
    res = _run(ctx, reads, refs, [(0, len(r), 0, len(r)) for r in reads], md_cfg)
    assert (res["result"] == 0).all() and list(res["nm"]) == [0, 1, 2, 1, 1, 1]
    bases = b"ACGTNRYACGT"
    ex = PrefilterConfig(exact_first=True)
    res = _run(ctx, [bases], [bases], [(0, 11, 0, 11)], ex)
    assert (int(res["result"][0]), int(res["nm"][0])) == (3, 3)


@pytest.mark.parametrize("variant", ["default", "no_exact", "tight_xdrop", "no_tail",
                                     "strict", "margin", "disabled", "minid"])
def test_stage4_corpus(ctx, variant):
    from kira_ls_aligner_b200 import PairBatch, PrefilterConfig, synth
    w = synth.prefilter_chains(4000, seed=0x77 + len(variant), err_hi=0.03, ref_len=600_000)
    cfg = {"default": PrefilterConfig(),
           "no_exact": PrefilterConfig(exact_first=False),
           "tight_xdrop": PrefilterConfig(xdrop=12),
           "no_tail": PrefilterConfig(tail=False, xdrop=30),
           "strict": PrefilterConfig(accept_span_slack=0, accept_max_mismatches=1,
                                     accept_min_identity=99.5, long_read_threshold=149),
           "margin": PrefilterConfig(accept_require_score_margin=10, accept_only_top1=False),
           "disabled": PrefilterConfig(accept_enable=False, multi_alignments_enabled=True),
           "minid": PrefilterConfig(min_identity_x10000=9700)}[variant]
    ctx.ref_upload(w.reference)
    n = w.n_pairs
    b = PairBatch(w.reads, w.read_off, w.read_len, None, np.zeros(n, np.uint64),
                  np.full(n, len(w.reference), np.uint32))
    res, ops, md = ctx.prefilter_batch(b, w.chains, cfg, is_top1=w.is_top1,
                                       score_margin=w.score_margin)
    ref = w.reference.tobytes()
    kinds = np.bincount(res["result"], minlength=4)
    for i in range(n):
        read = w.reads[i * 150:(i + 1) * 150].tobytes()
        want = _want(read, ref, tuple(int(x) for x in w.chains[i]), cfg, int(w.is_top1[i]),
                     int(w.score_margin[i]))
        assert _got(res, ops, md, i) == want, (i, w.chains[i])
    if variant == "default":
        assert kinds[0] > 0 and kinds[2] > 0 and kinds[3] > 0
    exact = ctx.exact_match_batch(b, w.chains)
    want = [O.exact_match_exists(w.reads[i * 150:(i + 1) * 150].tobytes(), ref,
                                 tuple(int(x) for x in w.chains[i])) for i in range(n)]
    assert list(exact) == [int(x) for x in want]


def test_edge_cases(ctx):
    from kira_ls_aligner_b200 import PrefilterConfig
    rng = np.random.default_rng(11)
    alpha = b"ACGTNacgt="
    reads, refs, chains = [b"", b"ACGT", b"ACGT", b"ACGTACGT"], [b"ACGT", b"ACGT", b"ACGT",
                                                                     b"ACGTACGT"], \
        [(0, 0, 0, 0), (0, 4, 3, 1), (0, 2, 2, 2), (0, 8, 0, 8)]
    for _ in range(400):
        m = int(rng.integers(1, 120))
        read = bytes(alpha[int(i)] for i in rng.integers(0, len(alpha), m))
        pad = int(rng.integers(0, 50))
        ref = bytearray(bytes(b"ACGT"[int(i)] for i in rng.integers(0, 4, pad)) + read +
                        bytes(b"ACGT"[int(i)] for i in rng.integers(0, 4, 30)))
        for _ in range(int(rng.integers(0, 4))):
            ref[int(rng.integers(0, len(ref)))] = ord("G")
        s = int(rng.integers(0, m))
        e = int(rng.integers(s, m + 1))
        reads.append(read)
        refs.append(bytes(ref))
        chains.append((pad + s, min(pad + e + int(rng.integers(-1, 2)), len(ref)), s, e))
    for cfg in (PrefilterConfig(long_read_threshold=100), PrefilterConfig(exact_first=False,
                                                                          xdrop=5)):
        _run(ctx, reads, refs, chains, cfg)


def test_invalid_and_capacity(ctx):
    from kira_ls_aligner_b200 import (CapacityError, InvalidArgument, PairBatch, PrefilterConfig,
                                      _abi)
    b = PairBatch.from_pairs([READ150], [READ150])
    bad = np.array([(0, 150, 0, 151)], _abi.CHAIN_DTYPE)
    with pytest.raises(InvalidArgument):
        ctx.prefilter_batch(b, bad, PrefilterConfig())
    ok = np.array([(0, 150, 0, 150)], _abi.CHAIN_DTYPE)
    with pytest.raises(CapacityError):
        ctx.prefilter_batch(b, ok, PrefilterConfig(), md_cap=2)
    res, ops, md = ctx.prefilter_batch(b, ok, PrefilterConfig())
    assert int(res["result"][0]) == 3 and md.tobytes() == b"150"


def test_chunked_host_path(ctx):
    # Several chunks (overlapped uploads / kernels / downloads, CIGAR and MD offsets
    # through running totals, no host round trip between the passes) equal the
    # one-shot call; a too-small MD buffer still reports the bytes needed.
    from kira_ls_aligner_b200 import CapacityError, PairBatch, PrefilterConfig, _abi, synth
    w = synth.prefilter_chains(90_000, seed=0xC4A1, err_hi=0.03, ref_len=2_000_000)
    n = w.n_pairs
    ctx.ref_upload(w.reference)
    b = PairBatch(w.reads, w.read_off, w.read_len, None, np.zeros(n, np.uint64),
                  np.full(n, len(w.reference), np.uint32))
    cfg = PrefilterConfig()
    L = _abi.lib()
    try:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 0))
        one = ctx.prefilter_batch(b, w.chains, cfg, is_top1=w.is_top1, score_margin=w.score_margin)
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, 32768))
        many = ctx.prefilter_batch(b, w.chains, cfg, is_top1=w.is_top1,
                                   score_margin=w.score_margin)
        with pytest.raises(CapacityError):
            ctx.prefilter_batch(b, w.chains, cfg, is_top1=w.is_top1, score_margin=w.score_margin,
                                md_cap=1000)
    finally:
        ctx.check(L.kira_gpu_set_chunk_pairs(ctx.handle, -1))
    for a, c in zip(one, many):
        assert np.array_equal(a, c)
    ref = w.reference.tobytes()
    res, ops, md = many
    for i in range(0, n, 89):
        read = w.reads[i * 150:(i + 1) * 150].tobytes()
        want = _want(read, ref, tuple(int(x) for x in w.chains[i]), cfg, int(w.is_top1[i]),
                     int(w.score_margin[i]))
        assert _got(res, ops, md, i) == want, i
