"""Pins the banded SW and full-window batch SW restatements to the reference
tests: src/alignment/mod.rs:2326-2677, tests/alignment.rs,
tests/unit/alignment_sw_int8_vnni.rs."""
import pytest

import pyoracle as O
from refgen import XorShift, BASES, gen_ref, rand_dna_lcg, replay_score, truth_sw


def cfgb(bw):  # mod.rs:2330-2340
    return O.cfg(1, 4, 6, 1, bw, 1000, 5)


def del_len(res):
    return sum(n for n, op in res.cigar if op == "D")


def test_adaptive_recovers_drifted_indels_fixed_band_clips():  # mod.rs:2368-2417
    ref = gen_ref(120)
    read = ref[0:30] + ref[33:60] + ref[63:120]
    assert len(read) == 114
    a = O.banded_sw(read, ref, 0, cfgb(4), adaptive=True)
    f = O.banded_sw(read, ref, 0, cfgb(4), adaptive=False)
    aligned = lambda r: r.read_end - r.read_start
    assert del_len(a) == 6 and aligned(a) >= 113
    assert del_len(f) < 6
    assert a.score > f.score + 15 and aligned(a) > aligned(f) + 15


def test_gapless_adaptive_equals_fixed():  # mod.rs:2421-2439
    ref = gen_ref(120)
    read = ref[10:90]
    a = O.banded_sw(read, ref, 10, cfgb(6), adaptive=True)
    f = O.banded_sw(read, ref, 10, cfgb(6), adaptive=False)
    assert (a.score, a.cigar, a.read_start, a.read_end) == (f.score, f.cigar, f.read_start,
                                                            f.read_end)
    assert del_len(a) == 0 and a.read_end - a.read_start >= 79


def test_first_base_match_is_not_softclipped():  # mod.rs:2483-2500
    ref = gen_ref(80)
    read = ref[0:60]
    for adaptive in (False, True):
        r = O.banded_sw(read, ref, 0, cfgb(8), adaptive=adaptive)
        assert (r.read_start, r.read_end, r.score, del_len(r)) == (0, 60, 60, 0)


def test_affine_traceback_score_matches_replayed_cigar():  # mod.rs:2591-2635
    ref = gen_ref(90)
    read = ref[:40] + b"TTGCA" + ref[40:]
    c = cfgb(20)
    r = O.banded_sw(read, ref, 0, c, adaptive=True)
    assert replay_score(read, ref, r.read_start, r.ref_start, r.cigar, c) == r.score
    assert any(op == "I" and n >= 5 for n, op in r.cigar)


def test_replayed_cigar_random_corpus():
    # Property: every traceback replays to its score, for both band modes.
    rng = XorShift(0x5CA1AB1E)
    c = O.cfg(1, 4, 6, 1, 12, 100, 5)
    for _ in range(300):
        n = 40 + rng.next() % 120
        ref = bytes(BASES[rng.next() % 4] for _ in range(n + 40))
        read = bytearray(ref[20:20 + n])
        for _ in range(rng.next() % 6):
            p = rng.next() % len(read)
            kind = rng.next() % 3
            if kind == 0:
                read[p] = BASES[rng.next() % 4]
            elif kind == 1:
                read.insert(p, BASES[rng.next() % 4])
            elif len(read) > 10:
                del read[p]
        read = bytes(read)
        for adaptive in (True, False):
            r = O.banded_sw(read, ref, 20, c, adaptive=adaptive)
            assert replay_score(read, ref, r.read_start, r.ref_start, r.cigar, c) == r.score


# ---- tests/alignment.rs (align_chain / align_batch_simd surface) ----
def clamp_window(ref_len, ref_start, ref_end, bw):  # mod.rs:1766-1771
    flank = max(max(bw, 1) * 2, 50)
    start = max(ref_start - flank, 0)
    end = min(ref_end + flank, ref_len)
    return start, max(end, start + 1)


def align_chain(read, ref, span, c):
    """align_oriented_chain_with_meta (mod.rs:851-877) without the exact-match shortcut."""
    ref_start, ref_end, read_start, read_end = span
    ws, we = clamp_window(len(ref), ref_start, ref_end, c.bandwidth)
    win = ref[ws:we]
    off = ref_start - ws - read_start
    sw = O.banded_sw(read, win, off, c)
    cig = list(sw.cigar)
    if sw.read_start > 0:
        cig.insert(0, (sw.read_start, "S"))
    if sw.read_end < len(read):
        cig.append((len(read) - sw.read_end, "S"))
    return sw, cig, ws


def end_indel_fixture():  # tests/alignment.rs:35-45
    base = bytes(b"CGTA"[i % 4] for i in range(150))
    ref = b"TT" + base + b"TT"
    read = base[:145] + b"G" + base[145:149]
    assert len(read) == 150
    return ref, read


def test_alignment_finds_full_match():  # tests/alignment.rs:4-33
    c = O.cfg(2, 4, 6, 1, 50, 40, 5)
    sw, cig, ws = align_chain(b"ACGTACGT", b"TTACGTACGTGG", (2, 10, 0, 8), c)
    assert (8, "M") in cig


def test_end_of_read_insertion_emits_i_op():  # :47-92
    ref, read = end_indel_fixture()
    c = O.cfg(1, 4, 6, 1, 50, 50, 5)
    sw, cig, _ = align_chain(read, ref, (2, 147, 0, 145), c)
    assert any(op == "I" for _, op in cig)
    trailing = cig[-1][0] if cig[-1][1] == "S" else 0
    assert trailing <= 1


def test_end_of_read_insertion_softclips_without_penalty():  # :94-122
    ref, read = end_indel_fixture()
    c = O.cfg(1, 4, 6, 1, 50, 50, 0)
    sw, cig, _ = align_chain(read, ref, (2, 147, 0, 145), c)
    assert not any(op == "I" for _, op in cig)


def test_batch_cardinality_and_order():  # :124-171
    bases = b"ACGTTGCTAATCGTGCATGACCTG"
    c = O.cfg(2, 4, 6, 1, 50, 40, 5)
    for mode in (O.SIMD_AVX2, O.SIMD_NEON, O.SIMD_VNNI):
        for count in (0, 1, 4, 5, 16, 17, 33):
            res = O.align_batch_simd([bases] * count, [bases] * count, c, mode, O.SIMD_VNNI,
                                     aborts=[0] * count, offsets=[0] * count)
            assert len(res) == count
            for r in res:
                assert (r.ref_start, r.ref_end) == (0, len(bases)) and r.cigar == [(24, "M")]


def test_scalar_and_mixed_batches_follow_seed_diagonal():  # :173-224
    read = b"GATTACAGCTTGAGTCCACG"
    window = b"C" * 100 + read
    c = O.cfg(2, 4, 6, 1, 8, 40, 5)
    off = 303 - 200 - 3
    for reads in ([read], [read, read[:19]]):
        for mode in (O.SIMD_SCALAR, O.SIMD_AVX2, O.SIMD_NEON):
            res = O.align_batch_simd(reads, [window] * len(reads), c, mode, O.SIMD_VNNI,
                                     offsets=[off] * len(reads))
            r = res[0]
            assert (200 + r.ref_start, 200 + r.ref_end, r.score) == (300, 320, 40)
            assert r.cigar_str() == "20M"


@pytest.mark.parametrize("length,reward,offset", [(7, 4681, 0), (8, 4096, 0), (150, 300, 0),
                                                  (8, 1, 32768)])
def test_i16_boundary(length, reward, offset):  # :226-274
    read = b"G" * length
    ref = b"C" * offset + read
    c = O.cfg(reward, 4, 6, 1, 8, 40, 5)
    for mode in (O.SIMD_AVX2, O.SIMD_VNNI):
        r = O.align_batch_simd([read], [ref], c, mode, O.SIMD_VNNI, offsets=[offset])[0]
        assert r.score == reward * length
        assert (r.ref_start, r.ref_end) == (offset, offset + length)
        assert r.cigar == [(length, "M")]


# ---- int8 kernel (tests/unit/alignment_sw_int8_vnni.rs) ----
def test_int8_matches_truth_on_clean_reads():  # :78-124
    c = O.cfg(1, 4, 6, 1, 50, 50, 5)
    reads, refs = [], []
    for k in range(32):
        r = rand_dna_lcg(130, 0xCAFEBABEDEAD ^ k)
        refs.append(r)
        reads.append(r[15:115])
    _, res = O.sw_batch("int8", reads, refs, c)
    for k in range(32):
        assert res[k].score == truth_sw(reads[k], refs[k], 1, 4, 6, 1) == 100


def test_int8_matches_truth_with_mismatches():  # :126-183
    c = O.cfg(1, 4, 6, 1, 50, 50, 0)
    nxt = {ord("A"): ord("C"), ord("C"): ord("G"), ord("G"): ord("T")}
    reads, refs = [], []
    for k in range(32):
        r = rand_dna_lcg(100, 0x12345678 ^ k)
        q = bytearray(r[10:90])
        for pos in ((k * 7) % 80, (k * 11 + 23) % 80):
            q[pos] = nxt.get(q[pos], ord("A"))
        reads.append(bytes(q))
        refs.append(r)
    _, res = O.sw_batch("int8", reads, refs, c)
    for k in range(32):
        assert res[k].score == truth_sw(reads[k], refs[k], 1, 4, 6, 1)


def test_int8_path_viable_thresholds():  # :185-199
    c = O.cfg(1, 4, 6, 1, 50, 50, 5)
    assert O.int8_path_viable(100, c) and O.int8_path_viable(119, c)
    assert not O.int8_path_viable(120, c) and not O.int8_path_viable(150, c)
    c2 = O.cfg(2, 4, 6, 1, 50, 50, 5)
    assert not O.int8_path_viable(100, c2) and O.int8_path_viable(50, c2)


def _random_batch(rng, lanes, q, r):
    reads, wins = [], []
    for _ in range(lanes):
        win = bytes(BASES[rng.next() % 4] for _ in range(r))
        s = rng.next() % (r - q + 1)
        read = bytearray(win[s:s + q])
        for _ in range(rng.next() % 8):
            p = rng.next() % q
            read[p] = BASES[rng.next() % 4]
        if rng.next() % 3 == 0:
            p = rng.next() % (q - 5)
            read[p:p + 3] = b""
            read += bytes(BASES[rng.next() % 4] for _ in range(3))
        wins.append(win)
        reads.append(bytes(read))
    return reads, wins


def test_avx2_kernel_equals_scalar_model():
    # The portable i16 model (the CUDA full-window spec) reproduces the AVX2 kernel,
    # including per-lane abort bounds and the all-lanes-done break.
    rng = XorShift(0xB16B00B5)
    c = O.cfg(1, 4, 6, 1, 33, 100, 5)
    for trial in range(40):
        q = 20 + rng.next() % 60
        r = q + rng.next() % 40
        lanes = 1 + rng.next() % 16
        reads, wins = _random_batch(rng, lanes, q, r)
        aborts = [O.ABORT_DISABLED if rng.next() % 2 else int(rng.next() % (q + 10))
                  for _ in range(lanes)]
        rc, a = O.sw_batch("avx2", reads, wins, c, aborts=aborts)
        assert rc == 1
        _, m = O.sw_batch("model16", reads, wins, c, aborts=aborts)
        assert [x.key() for x in a] == [x.key() for x in m]


def test_int8_kernel_equals_i16_within_viability():
    rng = XorShift(0x1F2E3D4C)
    c = O.cfg(1, 4, 6, 1, 33, 100, 5)
    for trial in range(20):
        q = 20 + rng.next() % 90
        r = q + rng.next() % 30
        reads, wins = _random_batch(rng, 32, q, r)
        _, a = O.sw_batch("int8", reads, wins, c)
        _, m8 = O.sw_batch("model8", reads, wins, c)
        _, m16 = O.sw_batch("model16", reads, wins, c)
        assert [x.key() for x in a] == [x.key() for x in m8] == [x.key() for x in m16]
