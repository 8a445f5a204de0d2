"""GPU Myers bounded edit distance vs the oracle (tests/myers_bounded_edit.rs corpora)."""
import pytest

import pyoracle as O
from gpu_cases import mutate
from refgen import BASES, XorShift

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from kira_ls_aligner_b200 import GpuContext
    c = GpuContext(0)
    yield c
    c.close()


def _run(ctx, pats, texts, k):
    from kira_ls_aligner_b200 import PairBatch
    b = PairBatch.from_pairs(pats, texts)
    d, e = ctx.myers_batch(b, k)
    for p, t, dd, ee in zip(pats, texts, d, e):
        want = O.bounded_edit_distance(p, t, k)
        got = None if dd < 0 else (int(dd), int(ee))
        assert got == want, (p, t, k)


def test_hand_cases(ctx):
    pats = [b"ACGTACGTACGT", b"ACGTACGTACGT", b"ACGTACGT", b"ACGTACGT", b"AAAAAAAA", b"ACGT",
            b""]
    texts = [b"NNACGTACGTACGTNN", b"NNACGTAXGTACGTNN", b"NNACGTAAACGTNN", b"NNACGACGTNN",
             b"TTTTTTTT", b"", b"ACGT"]
    for k in (0, 1, 3, 5, 8):
        _run(ctx, pats, texts, k)


@pytest.mark.parametrize("seed", [0x5EED1234, 0xDEADBEEF, 0xFACE1357])
def test_random_corpus_all_k(ctx, seed):
    rng = XorShift(seed)
    alpha = b"ACGTN"
    pats, texts = [], []
    for _ in range(600):
        m = 1 + rng.next() % 512
        n = rng.next() % (m + 80)
        pat = bytes(alpha[rng.next() % (5 if rng.next() % 8 == 0 else 4)] for _ in range(m))
        text = bytearray(alpha[rng.next() % 4] for _ in range(n))
        if rng.next() % 2 and n >= m:
            s = rng.next() % (n - m + 1)
            text[s:s + m] = mutate(rng, pat, rng.next() % 5, rng.next() % 3)[: n - s]
        pats.append(pat)
        texts.append(bytes(text))
    for k in (0, 2, 8, 26, 64):
        _run(ctx, pats, texts, k)
