"""Pins the sieve restatement (oracle) to the reference's known-answer tests:
tests/bitpacked_scan.rs, tests/unit/alignment_bitpacked.rs, tests/spectral_scan.rs
and the corpus of tests/cuda_spectral.rs."""
import pyoracle as O
from refgen import BASES, XorShift, naive_best_shift, naive_mismatches


def test_pack_roundtrip_short():  # tests/bitpacked_scan.rs:43-50
    bits, _, _ = O.pack(b"ACGTACGT")
    assert bits == bytes([0xE4, 0xE4])


def test_pack_handles_padding():  # tests/bitpacked_scan.rs:52-59
    bits, _, _ = O.pack(b"ACGTA")
    assert len(bits) == 2 and bits[1] & 0b11 == 0 and bits[1] >> 2 == 0


def test_scan_exact_match_at_zero():  # :61-69
    read = b"ACGTACGTACGT"
    assert O.scan(read, read, 0) == (0, 0)


def test_scan_exact_match_in_middle():  # :71-80
    assert O.scan(b"ACGTACGT", b"AAAAACGTACGTAAAA", 0) == (4, 0)


def test_scan_rejects_when_too_many_mismatches():  # :82-91
    assert O.scan(b"AAAAAAAA", b"TTTTTTTTTTTT", 3) is None
    assert O.scan(b"AAAAAAAA", b"TTTTTTTTTTTT", 8)[1] == 8


def test_scan_long_read_avx_path():  # :93-108
    read = bytes(BASES[i % 4] for i in range(150))
    text = bytearray(BASES[(i + 1) % 4] for i in range(200))
    text[25:175] = read
    text[25 + 7] = ord("T") if read[7] == ord("A") else ord("A")
    text[25 + 100] = ord("G") if read[100] == ord("C") else ord("C")
    hit = O.scan(read, bytes(text), 5)
    assert hit is not None and naive_mismatches(read, bytes(text), hit[0]) == hit[1] <= 5


def test_random_corpus_self_consistent():  # :110-149 (seed 0xC0FFEEBAD)
    rng = XorShift(0xC0FFEEBAD)
    for _ in range(200):
        r = 16 + rng.next() % 180
        w = r + rng.next() % 100
        read = bytes(BASES[rng.next() % 4] for _ in range(r))
        text = bytearray(BASES[rng.next() % 4] for _ in range(w))
        if rng.next() % 2 == 0 and w >= r:
            start = rng.next() % (w - r + 1)
            text[start:start + r] = read
        text = bytes(text)
        _, naive_m = naive_best_shift(read, text)
        hit = O.scan(read, text, r)
        assert naive_mismatches(read, text, hit[0]) == hit[1]
        tight = O.scan(read, text, naive_m)
        assert tight[1] <= naive_m
        if naive_m > 0:
            assert O.scan(read, text, naive_m - 1) is None


def test_shift_aligns_one_nucleotide():  # tests/unit/alignment_bitpacked.rs:3-9
    bits, _, _ = O.pack(b"ACGT")
    assert O.shift_bits_right(bits, 2)[0] == 0x39


def test_pre_shift_phases():  # :11-25 (owned vs reused buffers agree by construction)
    bits, _, _ = O.pack(b"ACGTTGCAAGGCTTAC")
    ph = O.pre_shift(bits)
    for p in range(4):
        assert ph[p] == O.shift_bits_right(bits, 2 * p)


def test_pack_into_validity():  # :27-35, :52-56
    assert O.pack(b"ACGTACGTA")[2]
    assert not O.pack(b"ACNT")[2]
    assert not O.pack(b"acgu")[2]
    assert O.pack(b"acgt")[2]


def test_scan_returns_global_best():  # :58-66
    assert O.scan(b"ACGT", b"TTTTACGT", 4) == (4, 0)


def test_scan_reports_tied_second_best():  # :68-76
    best = O.scan_best_with_second(b"ACGT", b"ACGTACGT")
    assert best[1] == 0 and best[2] == 0


def test_scan_second_best_semantics():
    # Second best is the minimum count over every other shift (ties with the best count).
    rng = XorShift(0xA11CE)
    for _ in range(100):
        r = 4 + rng.next() % 40
        w = r + rng.next() % 30
        read = bytes(BASES[rng.next() % 4] for _ in range(r))
        text = bytes(BASES[rng.next() % 4] for _ in range(w))
        counts = [naive_mismatches(read, text, t) for t in range(w - r + 1)]
        got = O.scan_best_with_second(read, text)
        best = min(counts)
        assert got[0] == counts.index(best) and got[1] == best
        rest = counts[: got[0]] + counts[got[0] + 1:]
        assert got[2] == (min(rest) if rest else None)


# ---- tests/spectral_scan.rs (byte sieve) ----
def naive_byte(read, win):
    r = len(read)
    bm, bs = 0, 0
    for t in range(len(win) - r + 1):
        m = sum(1 for a, b in zip(read, win[t:t + r]) if a == b)
        if m > bm:
            bm, bs = m, t
    return bs, r - bm


def test_byte_scan_known_answers():
    assert O.byte_scan(b"ACGT", b"ACG", 5) is None
    assert O.byte_scan(b"ACGTACGT", b"ACGTACGT", 0) == (0, 0)
    assert O.byte_scan(b"ACGTACGT", b"NNNNACGTACGTNNNN", 0) == (4, 0)
    hit = O.byte_scan(b"ACGTACGT", b"NNACGTAXGTNN", 5)
    assert hit == naive_byte(b"ACGTACGT", b"NNACGTAXGTNN") and hit[1] == 1
    assert O.byte_scan(b"AAAAAAAAAA", b"TTTTTTTTTTTT", 3) is None
    assert O.byte_scan(b"AAAAAAAAAA", b"TTTTTTTTTTTT", 10)[1] == 10


def test_byte_scan_random_corpus():  # tests/spectral_scan.rs:94-125 (seed 0xFEEDFACE)
    rng = XorShift(0xFEEDFACE)
    for _ in range(200):
        r = 16 + rng.next() % 200
        w = r + rng.next() % 100
        read = bytes(BASES[rng.next() % 4] for _ in range(r))
        text = bytearray(BASES[rng.next() % 4] for _ in range(w))
        if rng.next() % 2 == 0 and w >= r:
            start = rng.next() % (w - r + 1)
            text[start:start + r] = read
        text = bytes(text)
        hit = O.byte_scan(read, text, r)
        assert hit[1] == naive_mismatches(read, text, hit[0])
        assert hit[1] == naive_byte(read, text)[1]


def cuda_corpus(n=64):
    """make_corpus of tests/cuda_spectral.rs:20-47 (seed 0xCAFE_F00D)."""
    rng = XorShift(0xCAFEF00D)
    out = []
    for _ in range(n):
        r = 16 + rng.next() % 200
        w = r + rng.next() % 80
        read = bytes(BASES[rng.next() % 4] for _ in range(r))
        text = bytearray(BASES[rng.next() % 4] for _ in range(w))
        if rng.next() % 2 == 0 and w >= r:
            start = rng.next() % (w - r + 1)
            text[start:start + r] = read
            for _ in range(rng.next() % 4):
                pos = start + rng.next() % r
                text[pos] = ord("T") if text[pos] == ord("A") else ord("A")
        out.append((read, bytes(text), max(r * 8 // 100, 5)))
    return out


def test_gpu_semantics_consistent_with_cpu():  # tests/cuda_spectral.rs:74-137 on the oracle
    for read, text, max_m in cuda_corpus():
        rb, _, _ = O.pack(read)
        tb, _, _ = O.pack(text)
        shift, mism, second = O.gpu_sieve_semantics(rb, len(read), tb, len(text), max_m)
        cpu = O.scan_best_with_second(read, text)
        assert (None if second == 2**31 - 1 else second) == cpu[2]
        if cpu[1] <= max_m:
            assert (shift, mism) == (cpu[0], cpu[1])
            assert naive_mismatches(read, text, shift) == mism
        else:
            assert shift == -1 and mism == 2**31 - 1
