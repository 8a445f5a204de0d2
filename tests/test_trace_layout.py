"""Packed banded-SW trace layout, restated on the CPU: rows interleave in blocks of
16 / G ([row block][slab][row in block][lane] of 8-byte words, csrc/bsw16.cuh). For
every packed launch shape and read length: each (row, lane, slab) word is unique
and lies inside the item's slot (shape_slot_bytes, csrc/internal.h), and each cell
byte the traceback decoder reads (Bsw16Code) lies in the word its lane stored for
that cell's slab."""
import pytest

PACKED_SHAPES = [(2, 9), (4, 5), (4, 9), (8, 5), (8, 9), (16, 9), (32, 9)]  # (G, K)


def geometry(g, k):
    words = (k + 1) // 2              # code words per lane per row
    slabs = (words + 1) // 2          # 8-byte stores per lane per row
    stride = g * 8 * slabs            # bytes per row
    inter = 1 if g >= 16 else 16 // g
    return slabs, stride, inter


def slot_bytes(g, k, max_q):
    _, stride, inter = geometry(g, k)
    rows = (max_q + 1 + inter - 1) // inter * inter
    return (rows * stride + 15) // 16 * 16


def store_word(g, k, i, lane, slab):
    """Byte address of lane `lane`'s slab-`slab` word of row i (the DP kernel's store)."""
    _, stride, r = geometry(g, k)
    return (i & ~(r - 1)) * stride + (i & (r - 1)) * g * 8 + lane * 8 + slab * r * g * 8


def decode_byte(g, k, i, idx):
    """Byte address the traceback reads for band cell idx of row i (Bsw16Code)."""
    _, stride, r = geometry(g, k)
    half = g * k
    hi = 1 if idx >= half else 0
    c = idx - hi * half
    gi, kk = divmod(c, k)
    ib = i & (r - 1)
    return ((i - ib) * stride + ((kk >> 2) * r + ib) * g * 8 + gi * 8 +
            ((kk >> 1) & 1) * 4 + (kk & 1) * 2 + hi), gi, kk >> 2


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
                assert a % 8 == 0 and 0 <= a and a + 8 <= slot, (i, lane, slab, a, slot)
                assert a not in seen
                seen.add(a)


@pytest.mark.parametrize("g,k", PACKED_SHAPES)
def test_decoder_reads_the_stored_word(g, k):
    for i in (1, 2, 3, 4, 5, 17, 150):
        for idx in range(2 * g * k):
            a, lane, slab = decode_byte(g, k, i, idx)
            w = store_word(g, k, i, lane, slab)
            assert w <= a < w + 8, (g, k, i, idx, a, w)
