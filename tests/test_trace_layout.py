"""Packed banded-SW trace layout, restated on the CPU: a 4-bit code per cell, four
words (eight cells) per 4-byte slab, rows interleaved in blocks of 32 / G (8 for G = 1)
([row block][slab][row in block][lane] of 4-byte slabs, csrc/bsw16.cuh). For every
packed launch shape and read length: each (row, lane, slab) slab is unique and lies
inside the item's slot (shape_slot_bytes, csrc/internal.h), and each cell's code
the traceback decoder reads (Bsw16Code) lies in the slab its lane stored for that
cell, at the byte and nibble the DP kernel packed it into."""
import pytest

PACKED_SHAPES = [(2, 9), (4, 5), (4, 9), (8, 5), (8, 9), (16, 9), (32, 9), (2, 17),
                 (2, 18), (1, 34), (2, 34), (4, 34)]  # (G, K words)


def geometry(g, k):
    slabs = (k + 3) // 4              # 4-byte code slabs per lane per row
    stride = g * 4 * slabs            # bytes per row
    inter = 8 if g == 1 else 1 if g >= 32 else 32 // g
    return slabs, stride, inter


def slot_bytes(g, k, max_q):
    _, stride, inter = geometry(g, k)
    rows = (max_q + 1 + inter - 1) // inter * inter
    return (rows * stride + 15) // 16 * 16


def store_word(g, k, i, lane, slab):
    """Byte address of lane `lane`'s slab `slab` of row i (the DP kernel's store)."""
    _, stride, r = geometry(g, k)
    return (i & ~(r - 1)) * stride + (i & (r - 1)) * g * 4 + lane * 4 + slab * r * g * 4


def packed_position(kk, hi):
    """(byte in the slab, nibble) of word kk's cell in half hi, as the DP packs it:
    prmt of words (0, 1) and (2, 3) to the halves' high bytes, low nibbles from
    words 0-1, high nibbles from words 2-3."""
    w = kk & 3
    return (w & 1) * 2 + hi, w >> 1


def decode_byte(g, k, i, idx):
    """Byte address and nibble the traceback reads for band cell idx of row i."""
    _, stride, r = geometry(g, k)
    half = g * k
    hi = 1 if idx >= half else 0
    c = idx - hi * half
    gi, kk = divmod(c, k)
    ib = i & (r - 1)
    addr = (i - ib) * stride + ((kk >> 2) * r + ib) * g * 4 + gi * 4 + (kk & 1) * 2 + hi
    return addr, (kk & 2) >> 1, gi, kk >> 2, packed_position(kk, hi)


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
@pytest.mark.parametrize("max_q", [1, 3, 5, 150, 511])
def test_words_unique_and_inside_the_slot(g, k, max_q):
    slabs, _, _ = geometry(g, k)
    slot = slot_bytes(g, k, max_q)
    seen = set()
    for i in range(1, max_q + 1):
        for lane in range(g):
            for slab in range(slabs):
                a = store_word(g, k, i, lane, slab)
                assert a % 4 == 0 and 0 <= a and a + 4 <= slot, (i, lane, slab, a, slot)
                assert a not in seen
                seen.add(a)


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_decoder_reads_the_stored_code(g, k):
    for i in (1, 2, 3, 4, 5, 17, 150):
        seen = set()
        for idx in range(2 * g * k):
            a, nib, lane, slab, (byte, pnib) = decode_byte(g, k, i, idx)
            w = store_word(g, k, i, lane, slab)
            assert a == w + byte and nib == pnib, (g, k, i, idx, a, w, byte)
            assert (a, nib) not in seen  # one cell per nibble
            seen.add((a, nib))


def test_every_packed_shape_of_the_library_is_covered():
    from kira_ls_aligner_b200 import autotune
    lib = {(g, cells // 2) for (g, cells), p in zip(autotune.shapes(), autotune.packed()) if p}
    assert lib == set(PACKED_SHAPES)
