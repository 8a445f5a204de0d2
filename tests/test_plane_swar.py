"""The SWAR byte arithmetic of pack_planes_kernel (csrc/kernels.cu: plane_nibbles),
restated on the CPU: for every byte of a 4-byte word it must give base_code's three
plane bits (code bit 0, code bit 1, ACGT-valid; encode_base / is_acgt of
src/alignment/bitpacked.rs:12-20,89-91) in nibbles 0..3."""
import random

M = 0xFFFFFFFF


def base_code(b):
    valid = (b & 0xDF) in (0x41, 0x43, 0x47, 0x54)
    return ((((b >> 1) ^ (b >> 2)) & 3) | 4) if valid else 0


def prmt(a, b, sel):
    both = (a & M) | ((b & M) << 32)
    out = 0
    for k in range(4):
        n = (sel >> (4 * k)) & 0xF
        byte = (both >> (8 * (n & 7))) & 0xFF
        if n & 8:
            byte = 0xFF if byte & 0x80 else 0
        out |= byte << (8 * k)
    return out


def plane_nibbles(w):
    x = ((w >> 1) ^ (w >> 2)) & M
    y = x & 0x03030303
    z = y | (y >> 4)
    letter = prmt(0x54474341, 0, prmt(z, 0, 0x4420))
    t = (w & 0xDFDFDFDF) ^ letter
    v = ((~((((t & 0x7F7F7F7F) + 0x7F7F7F7F) & M) | t)) & 0x80808080 & M) >> 7
    g = lambda m: ((m * 0x01020408) & M) >> 24  # noqa: E731
    return g(x & v), g((x >> 1) & v), g(v)


def test_every_byte_value_in_every_position():
    rng = random.Random(7)
    for b in range(256):
        for pos in range(4):
            fill = [rng.choice(b"ACGTacgtNn-*") for _ in range(4)]
            fill[pos] = b
            w = sum(c << (8 * k) for k, c in enumerate(fill))
            n0, n1, nv = plane_nibbles(w)
            assert max(n0, n1, nv) < 16
            for k, c in enumerate(fill):
                code = base_code(c)
                assert ((n0 >> k) & 1, (n1 >> k) & 1, (nv >> k) & 1) == \
                    (code & 1, (code >> 1) & 1, code >> 2), (fill, k)
