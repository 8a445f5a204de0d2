"""The oracle's ungapped prefilter and exact-match restatement (orc_prefilter,
orc_exact_match_exists: src/alignment/prefilter.rs:93-517, mod.rs:779-832)
pinned by the reference's tests: tests/prefilter_accept.rs (accept, short-span
reject, not-top1, mismatches, not-short-preset), tests/md_format.rs (canonical
MD / NM of accepted alignments, ambiguity codes, exact_match_alignment's NM),
plus direct checks of the x-drop block walk and the decision cascade."""
import numpy as np
import pytest

import pyoracle as O

READ150 = b"ACGT" * 37 + b"AC"


def _cfg(**kw):
    base = dict(match_score=1, mismatch=4, xdrop=50, accept_span_slack=5,
                accept_min_identity=98.0, accept_max_mismatches=2, long_read_threshold=300)
    base.update(kw)
    return O.prefilter_cfg(**base)


def _full(n):
    return (0, n, 0, n)


def test_prefilter_accept_rs():
    ref = bytearray(READ150)
    ref[10] = ord("T")
    r = O.prefilter(READ150, bytes(ref), _full(150), _cfg())
    assert (r.result, r.reason) == ("accept", "accept")
    r = O.prefilter(b"A" * 400, b"T" * 400, (0, 44, 0, 44), _cfg())
    assert (r.result, r.reason) == ("reject", "span_too_small")
    r = O.prefilter(b"A" * 400, b"T" * 400, _full(400), _cfg(), is_top1=False)
    assert (r.result, r.reason) == ("fallback", "not_top1")
    r = O.prefilter(b"A" * 150, b"T" * 150, _full(150), _cfg())
    assert (r.result, r.reason) == ("fallback", "mism_too_high")
    r = O.prefilter(b"A" * 400, b"T" * 400, _full(400), _cfg())
    assert (r.result, r.reason) == ("fallback", "not_short_preset")


def _canon(read, ref):
    """tests/md_format.rs:27-43 (canonical SAM MD / NM of an ungapped span)."""
    md, run, nm = "", 0, 0
    for q, r in zip(read, ref):
        if q == r:
            run += 1
        else:
            nm += 1
            md += f"{run}{chr(r)}"
            run = 0
    return md + str(run), nm


def _accept_md(read, ref):
    r = O.prefilter(read, ref, _full(len(read)), _cfg(accept_span_slack=15,
                                                       accept_max_mismatches=5))
    assert r.result == "accept", r
    return r.md, r.nm


@pytest.mark.parametrize("edits", [[], [10], [5, 99], [149], [0]])
def test_md_format_rs(edits):
    ref = bytearray(READ150)
    for e in edits:
        ref[e] = ord("T") if ref[e] != ord("T") else ord("A")
    assert _accept_md(READ150, bytes(ref)) == _canon(READ150, ref)
    if not edits:
        assert _accept_md(READ150, bytes(ref)) == ("150", 0)


def test_ambiguity_and_exact_match():
    # tests/md_format.rs:162-186
    bases = b"ACGTNRYACGT"
    assert O.exact_match_exists(bases, bases, _full(len(bases)))
    assert O.identical_nm(bases) == 3
    longer = bytearray(b"ACGT" * 38)
    longer[70] = ord("N")
    assert _accept_md(bytes(longer), bytes(longer)) == ("152", 1)


def test_exact_match_exists_rules():
    # mod.rs:819-832: whole read, co-linear span of the read length, inside the reference
    ref = b"TT" + READ150 + b"GG"
    assert O.exact_match_exists(READ150, ref, (2, 152, 0, 150))
    assert not O.exact_match_exists(READ150, ref, (3, 153, 0, 150))
    assert not O.exact_match_exists(READ150, ref, (2, 152, 1, 150))
    assert not O.exact_match_exists(READ150, ref, (2, 151, 0, 150))
    assert not O.exact_match_exists(READ150, ref[:151], (2, 152, 0, 150))
    assert not O.exact_match_exists(READ150.lower(), ref, (2, 152, 0, 150))


def test_xdrop_block_walk():
    # Right of the anchor: a clean block (+32), then a block with 12 mismatches
    # (20 - 48 = -28). xdrop 20 stops the walk there (right extension 32); xdrop 50
    # walks on and the clean blocks after it and the 8-byte tail win back the lead
    # (right extension 136, the whole read).
    rng = np.random.default_rng(3)
    ref = bytes(b"ACGT"[i] for i in rng.integers(0, 4, 400))
    read = bytearray(ref[100:300])
    for i in range(96, 128, 8):
        for j in (i, i + 3, i + 5):
            read[j] = ord("A") if read[j] != ord("A") else ord("C")
    chain = (100 + 32, 100 + 64, 32, 64)
    tight = O.prefilter(bytes(read), ref, chain, _cfg(xdrop=20, long_read_threshold=1000))
    wide = O.prefilter(bytes(read), ref, chain, _cfg(xdrop=50, long_read_threshold=1000))
    assert tight.metrics[0] == 32 + 32 + 32 and tight.result == "reject"
    assert wide.metrics[0] == 200 and wide.metrics[1] == 12
    assert (wide.result, wide.reason) == ("fallback", "mism_too_high")
    no_tail = O.prefilter(bytes(read), ref, chain, _cfg(xdrop=50, long_read_threshold=1000,
                                                        tail=False))
    assert no_tail.metrics[0] == 32 + 32 + 128


def test_cascade_order_and_other_reasons():
    ref = bytes(READ150)
    c = _cfg()
    assert O.prefilter(b"", ref, (0, 0, 0, 0), c).reason == "read_len0"
    assert O.prefilter(READ150, ref, (0, 150, 10, 5), c).reason == "non_monotonic"
    assert O.prefilter(READ150, ref, (0, 10, 7, 7), c).reason == "anchor0"
    assert O.prefilter(READ150, ref, _full(150), _cfg(accept_enable=False)).reason == "disabled"
    assert O.prefilter(READ150, ref, _full(150),
                       _cfg(multi_alignments_enabled=True)).reason == "max_alignments_not_one"
    assert O.prefilter(READ150, ref, _full(150), _cfg(accept_require_score_margin=5),
                       score_margin=4).reason == "margin_fail"
    assert O.prefilter(READ150, ref, (0, 149, 0, 150), c).reason == "indel_suspect"
    r = O.prefilter(READ150, ref, (0, 150, 0, 150), _cfg(min_id_override=10001))
    assert r.reason == "id_too_low"
    with pytest.raises(ValueError):
        O.prefilter(READ150, ref, (0, 150, 0, 151), c)
