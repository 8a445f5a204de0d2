"""The oracle's WFA restatement (oracle/kira_oracle.cpp: orc_wfa, following
src/alignment/wfa.rs) pinned by the reference's own WFA tests, restated with
the same generators and seeds:

* tests/wfa_semi_global.rs -- known answers (8M / score 0, single mismatch,
  single indel, cutoff, two mismatches) and the random replay corpus (0xC0FFEE);
* tests/wfa2_modes.rs -- adaptive drop 50 equals exact (0xBADC0FFE), tight drop
  self-consistent (0x13579bdf), score-only equals full (0x9e3779b9), ends-free
  leading text;
* src/alignment/wfa.rs:965-1129 -- the 134M16I traceback regression and the
  end-divergence replay sweep (LCG 0x1234_5678_9abc_def0);
* tests/scored_wfa.rs -- scored WFA against an independent affine DP over 1800
  trials (0x6a09e667f3bcc909), score-only agreement, budget loss-1 -> None, and
  match rewards changing the optimal path (0xbb67ae8584caa73b).
"""
import pyoracle as O

M64 = (1 << 64) - 1
BASES = b"ACGT"


def xorshift(state):
    s = state[0]
    s ^= (s << 13) & M64
    s ^= s >> 7
    s ^= (s << 17) & M64
    state[0] = s
    return s


class Lcg:  # src/alignment/wfa.rs:1040-1052
    def __init__(self, seed):
        self.s = seed

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & M64
        return self.s >> 33

    def base(self):
        return BASES[self.next() % 4]


def pen_cfg(max_score, adaptive_drop=None, text_begin_free=0, traceback=True):
    return O.wfa_cfg(4, 6, 1, max_score, adaptive_drop, text_begin_free, traceback=traceback)


def apply_cigar(pattern, text, text_start, cigar, x=4, o=6, e=1):
    """tests/wfa2_modes.rs:24-52: replay -> (cost, text end); the pattern is consumed whole."""
    score, qi, ti = 0, 0, text_start
    for n, op in cigar:
        if op == "M":
            for _ in range(n):
                score += x if pattern[qi] != text[ti] else 0
                qi += 1
                ti += 1
        elif op == "I":
            score += o + e * n
            qi += n
        elif op == "D":
            score += o + e * n
            ti += n
        else:
            raise AssertionError(op)
    assert qi == len(pattern)
    return score, ti


def _mutate(rng, pattern, n_err, kinds=3):
    text = bytearray(pattern)
    for _ in range(n_err):
        pos = xorshift(rng) % len(text)
        kind = xorshift(rng) % kinds
        if kind == 0:
            text[pos] = BASES[xorshift(rng) % 4]
        elif kind == 1:
            text.insert(pos, BASES[xorshift(rng) % 4])
        elif len(text) > 1:
            del text[pos]
    return text


def test_semi_global_known_answers():
    # tests/wfa_semi_global.rs:66-136
    a = O.wfa(b"ACGTACGT", b"ACGTACGTAA", pen_cfg(20))
    assert (a.score, a.cigar_str(), a.text_end) == (0, "8M", 8)
    for pat, txt, want in ((b"ACGTACGT", b"ACATACGT", 4), (b"ACGTACGT", b"ACGACGT", 7),
                           (b"ACGACGT", b"ACGTACGT", 7)):
        a = O.wfa(pat, txt, pen_cfg(20))
        assert a.score == want
        assert apply_cigar(pat, txt, 0, a.cigar) == (a.score, a.text_end)
    assert O.wfa(b"AAAAAAAA", b"TTTTTTTT", pen_cfg(5)) is None
    a = O.wfa(b"AAAAAAAA", b"TTTTTTTT", pen_cfg(14))
    assert a.score == 14 and apply_cigar(b"AAAAAAAA", b"TTTTTTTT", 0, a.cigar)[0] == 14
    pat = b"ACGT" * 20
    txt = bytearray(pat)
    txt[15] = ord("C") if txt[15] == ord("A") else ord("A")
    txt[60] = ord("A") if txt[60] == ord("C") else ord("C")
    a = O.wfa(pat, bytes(txt), pen_cfg(20))
    assert a.score == 8 and apply_cigar(pat, txt, 0, a.cigar)[0] == 8


def test_semi_global_replay_random():
    # tests/wfa_semi_global.rs:138-178
    rng = [0xC0FFEE]
    for _ in range(50):
        m = 20 + xorshift(rng) % 80
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = _mutate(rng, pattern, xorshift(rng) % 4)
        for _ in range(5):
            text.append(BASES[xorshift(rng) % 4])
        a = O.wfa(pattern, bytes(text), pen_cfg(80))
        assert a is not None
        assert apply_cigar(pattern, text, 0, a.cigar) == (a.score, a.text_end)


def test_traceback_regression_134m16i():
    # src/alignment/wfa.rs:982-1030 (read captured from an E. coli run)
    read = (b"ATAGTCGAGCAGGTAATAACGCCCTTCGTGGCGGAACACCAGGTCGATAAAGCCTTTTAACATGCCACGTACCTGC"
            b"ATGAACTCCAGCGGCGGGCAGCCTGCGGATAGCGGGGCAAAATGGCGGATTAAAGTATAAAACCGCCTGGGGGT")
    text = (b"ATAGTCGAGCAGGTAATAACGCCCTTCGTGGCGGAACACCAGGTCGATAAAGCCTTTTAACATGCCACGTACCTGC"
            b"ATGAACTCCAGCGGCGGGCAGCCTGCGGATAGCGGGTCAAACTGGCGGATTAACGTATCAAGCTGACTGGCGATAA"
            b"GCGGTTCACTAATCGGCAGATAAAACTCCATCTCCACCTGTTTATTGC")
    assert len(read) == 150
    a = O.wfa(read, text, pen_cfg(150))
    assert a.cigar == [(134, "M"), (16, "I")]
    assert (a.score, a.text_start, a.text_end) == (34, 0, 134)


def test_traceback_end_divergence():
    # src/alignment/wfa.rs:1087-1127
    rng = Lcg(0x1234_5678_9ABC_DEF0)
    text = bytes(rng.base() for _ in range(260))
    cases = 0
    for prefix in (110, 120, 130, 134, 140, 145, 148, 149, 150):
        for tail in (1, 2, 3, 4, 6, 8, 12, 16, 20):
            read = bytearray(text[:prefix])
            for _ in range(tail):
                read.append(rng.base())
            a = O.wfa(bytes(read), text, pen_cfg(400))
            if a is None:
                continue
            cases += 1
            assert sum(n for n, op in a.cigar if op in "MI") == len(read)
            assert apply_cigar(read, text, a.text_start, a.cigar) == (a.score, a.text_end)
    assert cases >= 60


def test_adaptive_wide_drop_equals_exact():
    # tests/wfa2_modes.rs:63-124
    rng = [0xBADC0FFE]
    for _ in range(60):
        m = 40 + xorshift(rng) % 100
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = bytearray(pattern)
        for _ in range(xorshift(rng) % 4):
            pos = xorshift(rng) % len(text)
            kind = xorshift(rng) % 3
            if kind == 0:
                text[pos] = BASES[xorshift(rng) % 4]
            elif kind == 1:
                text.insert(pos, BASES[xorshift(rng) % 4])
            elif len(text) > 1:
                del text[pos]
        for _ in range(6):
            text.append(BASES[xorshift(rng) % 4])
        text = bytes(text)
        exact = O.wfa(pattern, text, pen_cfg(200))
        adaptive = O.wfa(pattern, text, pen_cfg(200, adaptive_drop=50))
        assert apply_cigar(pattern, text, adaptive.text_start, adaptive.cigar) == \
            (adaptive.score, adaptive.text_end)
        assert adaptive.score == exact.score


def test_adaptive_tight_drop_self_consistent():
    # tests/wfa2_modes.rs:128-167
    rng = [0x1357_9BDF]
    for _ in range(40):
        m = 50 + xorshift(rng) % 80
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = bytearray(pattern)
        for _ in range(xorshift(rng) % 5):
            pos = xorshift(rng) % len(text)
            text[pos] = BASES[xorshift(rng) % 4]
        for _ in range(6):
            text.append(BASES[xorshift(rng) % 4])
        text = bytes(text)
        exact = O.wfa(pattern, text, pen_cfg(400))
        adaptive = O.wfa(pattern, text, pen_cfg(400, adaptive_drop=3))
        if adaptive is not None:
            assert apply_cigar(pattern, text, adaptive.text_start, adaptive.cigar) == \
                (adaptive.score, adaptive.text_end)
            assert adaptive.score >= exact.score


def test_score_only_equals_full():
    # tests/wfa2_modes.rs:171-213
    rng = [0x9E37_79B9]
    for _ in range(200):
        m = 20 + xorshift(rng) % 120
        pattern = bytes(BASES[xorshift(rng) % 4] for _ in range(m))
        text = _mutate(rng, pattern, xorshift(rng) % 6)
        for _ in range(5):
            text.append(BASES[xorshift(rng) % 4])
        text = bytes(text)
        for budget in (8, 30, 200):
            full = O.wfa(pattern, text, pen_cfg(budget))
            so = O.wfa(pattern, text, pen_cfg(budget, traceback=False))
            assert (full and full.score) == (so and so.score)
            if full:
                assert full.text_end == so.text_end


def test_ends_free_leading_text():
    # tests/wfa2_modes.rs:218-257
    pattern = b"ACGTACGTACGTACGT"
    text = b"TTTTT" + pattern + b"GG"
    pinned = O.wfa(pattern, text, pen_cfg(200))
    assert (pinned.text_start, pinned.score) == (0, 11)
    assert apply_cigar(pattern, text, 0, pinned.cigar) == (pinned.score, pinned.text_end)
    free = O.wfa(pattern, text, pen_cfg(200, text_begin_free=5))
    assert (free.score, free.text_start, free.cigar_str(), free.text_end) == (0, 5, "16M", 21)


# --- tests/scored_wfa.rs -------------------------------------------------------

def _next32(state):
    return xorshift(state) >> 32


def affine_dp(q, r, a, b, o, e, lead):
    """tests/scored_wfa.rs:17-44: query-global, reference ends-free DP (best score)."""
    width = len(r) + 1
    neg = -(2**31) // 8
    lead = min(lead, max(len(r) - 1, 0))
    h = [0 if j <= lead else -o - e * (j - lead) for j in range(width)]
    ins = [neg] * width
    for i in range(1, len(q) + 1):
        nh = [neg] * width
        nins = [neg] * width
        nh[0] = -o - e * i
        nins[0] = nh[0]
        dl = neg
        for j in range(1, width):
            nins[j] = max(h[j] - o - e, ins[j] - e)
            dl = max(nh[j - 1] - o - e, dl - e)
            sub = a if q[i - 1] == r[j - 1] else -b
            nh[j] = max(h[j - 1] + sub, nins[j], dl)
        h, ins = nh, nins
    return max(h)


def replay_scored(q, r, res, a, b, o, e):
    """tests/scored_wfa.rs:46-78."""
    qi, ri, score = 0, res.text_start, 0
    for n, op in res.cigar:
        if op == "M":
            for _ in range(n):
                score += a if q[qi] == r[ri] else -b
                qi += 1
                ri += 1
        elif op == "I":
            qi += n
            score -= o + e * n
        elif op == "D":
            ri += n
            score -= o + e * n
        else:
            raise AssertionError(op)
    assert qi == len(q) and ri == res.text_end
    assert a * len(q) - score == res.score
    return score


def test_scored_matches_affine_dp():
    rng = [0x6A09E667F3BCC909]
    for trial in range(1800):
        a, b, o, e = ((1, 4, 6, 1), (2, 3, 2, 1), (3, 2, 0, 2))[trial % 3]
        qlen = 1 + _next32(rng) % 28
        rlen = 1 + _next32(rng) % 35
        q = bytes(BASES[_next32(rng) % 4] for _ in range(qlen))
        r = bytes(BASES[_next32(rng) % 4] for _ in range(rlen))
        lead = _next32(rng) % 5
        want = affine_dp(q, r, a, b, o, e, lead)
        res = O.wfa_scored(q, r, a, b, o, e, 300, text_begin_free=lead)
        assert replay_scored(q, r, res, a, b, o, e) == want, trial
        assert O.wfa_scored(q, r, a, b, o, e, 300, text_begin_free=lead, traceback=False) == want
        loss = qlen * a - want
        if loss > 0:
            assert O.wfa_scored(q, r, a, b, o, e, loss - 1, text_begin_free=lead) is None
            assert O.wfa_scored(q, r, a, b, o, e, loss - 1, text_begin_free=lead,
                                traceback=False) is None


def test_match_rewards_change_the_optimal_path():
    a, b, o, e = 2, 3, 2, 1
    rng = [0xBB67AE8584CAA73B]
    improved = 0
    for _ in range(300):
        q = bytes(BASES[_next32(rng) % 4] for _ in range(18))
        r = bytes(BASES[_next32(rng) % 4] for _ in range(24))
        old = O.wfa(q, r, O.wfa_cfg(b, o, e, 200))
        new = O.wfa_scored(q, r, a, b, o, e, 200)
        old_score, qi, ri = 0, 0, old.text_start
        for n, op in old.cigar:
            if op == "M":
                for _ in range(n):
                    old_score += a if q[qi] == r[ri] else -b
                    qi += 1
                    ri += 1
            else:
                old_score -= o + e * n
                qi += n if op == "I" else 0
                ri += n if op == "D" else 0
        new_score = replay_scored(q, r, new, a, b, o, e)
        assert new_score >= old_score
        improved += new_score > old_score
    assert improved > 0
