"""Seeded generators and naive checkers restated from the reference test suite.

* ``xorshift`` -- the 13/7/17 xorshift64 of tests/bitpacked_scan.rs:36-41,
  tests/myers_bounded_edit.rs:33-38, tests/cuda_spectral.rs:13-18.
* ``Lcg`` -- the MMIX LCG of tests/common/mod.rs:25-52.
* ``naive_*`` -- the brute-force references of tests/bitpacked_scan.rs:13-34,
  tests/spectral_scan.rs:7-28, tests/myers_bounded_edit.rs:9-31 and
  tests/unit/alignment_sw_int8_vnni.rs:44-76.
"""
M64 = (1 << 64) - 1
BASES = b"ACGT"


class XorShift:
    def __init__(self, seed: int):
        self.s = seed & M64

    def next(self) -> int:
        s = self.s
        s ^= (s << 13) & M64
        s ^= s >> 7
        s ^= (s << 17) & M64
        self.s = s
        return s


class Lcg:
    def __init__(self, seed: int):
        self.s = seed & M64

    def next_u64(self) -> int:
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & M64
        return self.s

    def below(self, n: int) -> int:
        return (self.next_u64() >> 33) % n

    def base(self) -> int:
        return BASES[(self.next_u64() >> 33) & 3]


def rand_dna_lcg(length: int, state: int) -> bytes:
    """rand_dna of tests/unit/alignment_sw_int8_vnni.rs:28-38 (bases from bits 60..61)."""
    out = bytearray()
    for _ in range(length):
        state = (state * 6364136223846793005 + 1442695040888963407) & M64
        out.append(BASES[(state >> 60) & 3])
    return bytes(out)


def gen_ref(length: int) -> bytes:
    """gen_ref of src/alignment/mod.rs:2344-2355 (xorshift seed 0x1234_5678_9abc_def0)."""
    s = 0x123456789ABCDEF0
    out = bytearray()
    for _ in range(length):
        s ^= (s << 13) & M64
        s ^= s >> 7
        s ^= (s << 17) & M64
        out.append(BASES[s & 3])
    return bytes(out)


def naive_mismatches(read: bytes, win: bytes, shift: int) -> int:
    return sum(1 for a, b in zip(read, win[shift:shift + len(read)]) if a != b)


def naive_best_shift(read: bytes, win: bytes):
    r = len(read)
    best, best_t = r + 1, 0
    for t in range(len(win) - r + 1):
        m = naive_mismatches(read, win, t)
        if m < best:
            best, best_t = m, t
    return best_t, best


def naive_semi_global(pattern: bytes, text: bytes):
    m, n = len(pattern), len(text)
    prev = [0] * (n + 1)
    for i in range(1, m + 1):
        cur = [i] + [0] * n
        pi = pattern[i - 1]
        for j in range(1, n + 1):
            cost = 0 if pi == text[j - 1] else 1
            cur[j] = min(prev[j - 1] + cost, prev[j] + 1, cur[j - 1] + 1)
        prev = cur
    best, pos = prev[0], 0
    for j, v in enumerate(prev):
        if v < best:
            best, pos = v, j
    return best, pos


def truth_sw(read: bytes, ref: bytes, match: int, mismatch: int, gap_open: int, gap_extend: int):
    """Full O(q*r) local SW score (tests/unit/alignment_sw_int8_vnni.rs:44-76)."""
    q, r = len(read), len(ref)
    neg = -(2**31) // 4
    prev_h = [0] * (r + 1)
    prev_e = [neg] * (r + 1)
    best = 0
    for i in range(1, q + 1):
        cur_h = [0] * (r + 1)
        cur_e = [neg] * (r + 1)
        cur_f = neg
        for j in range(1, r + 1):
            s = match if read[i - 1] == ref[j - 1] else -mismatch
            hm = prev_h[j - 1] + s
            e = max(prev_h[j] - gap_open, prev_e[j] - gap_extend)
            f = max(cur_h[j - 1] - gap_open, cur_f - gap_extend)
            h = max(hm, e, f, 0)
            cur_h[j] = h
            cur_e[j] = e
            cur_f = f
            best = max(best, h)
        prev_h, prev_e = cur_h, cur_e
    return best


def replay_score(read: bytes, ref: bytes, read_start: int, ref_start: int, cigar, c) -> int:
    """Score of a CIGAR replayed over the sequences (mod.rs:2591-2635)."""
    qi, ri, s = read_start, ref_start, 0
    for n, op in cigar:
        if op == "M":
            for _ in range(n):
                s += c.match_score if read[qi] == ref[ri] else -c.mismatch
                qi += 1
                ri += 1
        elif op == "I":
            s -= c.gap_open + c.gap_extend * n
            qi += n
        elif op == "D":
            s -= c.gap_open + c.gap_extend * n
            ri += n
        elif op == "S":
            qi += n
        elif op == "N":
            ri += n
    return s


def flip(b: int) -> int:
    return ord("T") if b == ord("A") else ord("A")
