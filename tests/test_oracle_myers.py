"""Pins the Myers restatement to tests/myers_bounded_edit.rs and the storage
equivalence test of src/alignment/myers.rs:326-367."""
import pyoracle as O
from refgen import BASES, XorShift, naive_semi_global


def bed(p, t, k, path=0):
    return O.bounded_edit_distance(p, t, k, path)


def test_hand_cases():  # tests/myers_bounded_edit.rs:40-132
    assert bed(b"", b"ACGT", 0) == (0, 0)
    assert bed(b"ACGT", b"", 4) == (4, 0)
    for pat, text, k in [(b"ACGTACGTACGT", b"NNACGTACGTACGTNN", 5),
                         (b"ACGTACGTACGT", b"NNACGTAXGTACGTNN", 3),
                         (b"ACGTACGT", b"NNACGTAAACGTNN", 3),
                         (b"ACGTACGT", b"NNACGACGTNN", 3)]:
        assert bed(pat, text, k) == naive_semi_global(pat, text)
    assert bed(b"ACGTACGTACGT", b"NNACGTACGTACGTNN", 5)[0] == 0
    assert bed(b"AAAAAAAA", b"TTTTTTTT", 3) is None
    assert bed(b"AAAAAAAA", b"TTTTTTTT", 8)[0] == 8


def test_multi_block_boundaries():  # :102-132
    p64 = bytes(BASES[i % 4] for i in range(64))
    t = bytearray(p64)
    t[20] = ord("A")
    assert bed(p64, bytes(t), 5)[0] == naive_semi_global(p64, bytes(t))[0]
    p65 = bytes(BASES[i % 4] for i in range(65))
    t = bytearray(p65)
    t[64] = ord("C") if p65[64] == ord("A") else ord("A")
    assert bed(p65, bytes(t), 5)[0] == naive_semi_global(p65, bytes(t))[0]
    p150 = bytes(BASES[(i * 7 + 3) % 4] for i in range(150))
    t = bytearray(p150)
    t[10] = ord("T") if t[10] == ord("A") else ord("A")
    t[77] = ord("G") if t[77] == ord("C") else ord("C")
    t[140] = ord("A") if t[140] == ord("G") else ord("G")
    assert bed(p150, bytes(t), 10)[0] == naive_semi_global(p150, bytes(t))[0]


def test_early_exit_preserves_accept_boundary():  # :137-171 (seed 0x5EED_1234)
    rng = XorShift(0x5EED1234)
    for _ in range(120):
        m = 1 + rng.next() % 160
        n = m + rng.next() % 80
        pat = bytes(BASES[rng.next() % 4] for _ in range(m))
        text = bytearray(BASES[rng.next() % 4] for _ in range(n))
        if rng.next() % 2 == 0 and n >= m:
            s = rng.next() % (n - m + 1)
            text[s:s + m] = pat
        text = bytes(text)
        truth, _ = naive_semi_global(pat, text)
        for k in range(m + 1):
            got = bed(pat, text, k)
            if k >= truth:
                assert got is not None and got[0] == truth
            else:
                assert got is None


def test_storage_paths_across_256():  # :176-212 (seed 0x0BAD_C0DE)
    rng = XorShift(0x0BADC0DE)
    for m in (200, 255, 256, 257, 300, 400):
        for trial in range(6):
            n = m + rng.next() % 60
            pat = bytes(BASES[rng.next() % 4] for _ in range(m))
            text = bytearray(BASES[rng.next() % 4] for _ in range(n))
            if trial % 2 == 0 and n >= m:
                s = rng.next() % (n - m + 1)
                text[s:s + m] = pat
                p = s + rng.next() % m
                text[p] = ord("T") if text[p] == ord("A") else ord("A")
            text = bytes(text)
            truth, _ = naive_semi_global(pat, text)
            assert bed(pat, text, m)[0] == truth
            if truth > 0:
                assert bed(pat, text, truth - 1) is None


def test_random_corpus_end_reaches_min():  # :214-249 (seed 0xDEADBEEF)
    rng = XorShift(0xDEADBEEF)
    for _ in range(100):
        m = 1 + rng.next() % 192
        n = m + rng.next() % 64
        pat = bytes(BASES[rng.next() % 4] for _ in range(m))
        text = bytearray(BASES[rng.next() % 4] for _ in range(n))
        if rng.next() % 2 == 0 and n >= m:
            s = rng.next() % (n - m + 1)
            text[s:s + m] = pat
        text = bytes(text)
        nd, _ = naive_semi_global(pat, text)
        d, end = bed(pat, text, m)
        assert d == nd
        assert naive_semi_global(pat, text[:end])[0] == nd


def test_fixed_and_heap_paths_agree_exactly():  # src/alignment/myers.rs:341-366
    rng = XorShift(0xFACE135724680BAD)
    alpha = b"ACGTN"
    for _ in range(4000):
        m = 1 + rng.next() % 256
        n = 1 + rng.next() % 300
        pat = bytes(alpha[rng.next() % 5] for _ in range(m))
        text = bytes(alpha[rng.next() % 5] for _ in range(n))
        for k in (0, 1, 3, m // 8, m // 4, m // 2, m):
            assert bed(pat, text, k, 1) == bed(pat, text, k, 2)


def test_last_column_tie_rule():
    # `err <= best` keeps the LAST column reaching the minimum (myers.rs:189-192).
    assert bed(b"AC", b"ACAC", 0) == (0, 4)
