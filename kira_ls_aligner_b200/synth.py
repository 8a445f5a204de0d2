"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: references, reads and candidate windows are
generated from fixed seeds (numpy PCG64), with the sizes and error profiles of
the verification workloads:

* ``small``   -- 1 Mbp uniform reference, 10k reads of 150 bp (1 % substitutions,
  0.1 % indels of length 1-3, geometric), 4 windows of 250 bp per read
  (1 true + 3 random): 40k pairs.
* ``batched`` -- 100 Mbp reference (uniform + 5 % of 300 bp repeat families at
  2-10 % divergence), 250k reads x 8 candidates (1 true) = 2M pairs,
  150 / 250 bp, per-read substitution rate U[0.5 %, 2 %], 0.1 % indels.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BASES = np.frombuffer(b"ACGT", np.uint8)


@dataclass
class Workload:
    name: str
    reference: np.ndarray      # uint8 ASCII
    reads: np.ndarray          # uint8 ASCII arena (all reads)
    read_off: np.ndarray       # per pair (uint64)
    read_len: np.ndarray       # per pair (uint32)
    win_off: np.ndarray        # per pair, reference coordinate (uint64)
    win_len: np.ndarray        # per pair (uint32)
    is_true: np.ndarray        # per pair: window holds the read's origin

    @property
    def n_pairs(self) -> int:
        return int(len(self.read_off))

    def windows_arena(self):
        """Materialise windows into their own arena (host-window mode)."""
        offs = np.zeros(self.n_pairs, np.uint64)
        if self.n_pairs:
            offs[1:] = np.cumsum(self.win_len[:-1].astype(np.uint64))
        total = int(self.win_len.astype(np.uint64).sum())
        arena = np.empty(total + 16, np.uint8)
        idx = np.repeat(self.win_off.astype(np.int64), self.win_len) + (
            np.arange(total) - np.repeat(offs.astype(np.int64), self.win_len))
        arena[:total] = self.reference[idx]
        arena[total:] = 0
        return arena, offs


def random_reference(rng, length: int, repeat_frac: float = 0.0, family_len: int = 300,
                     div_lo: float = 0.02, div_hi: float = 0.10, n_families: int = 200):
    ref = BASES[rng.integers(0, 4, length)]
    if repeat_frac > 0:
        copies = int(length * repeat_frac) // family_len
        fams = BASES[rng.integers(0, 4, (n_families, family_len))]
        starts = rng.integers(0, length - family_len, copies)
        which = rng.integers(0, n_families, copies)
        div = rng.uniform(div_lo, div_hi, copies)
        for s, f, d in zip(starts, which, div):
            seq = fams[f].copy()
            m = rng.random(family_len) < d
            seq[m] = BASES[(np.searchsorted(BASES, seq[m]) + rng.integers(1, 4, m.sum())) % 4]
            ref[s:s + family_len] = seq
    return ref


def _mutate(rng, frag: np.ndarray, read_len: int, sub_rate: float, indel_rate: float):
    """Substitutions + indels (length 1-3, geometric p=0.5) on a reference fragment
    that is longer than the read; returns exactly read_len bases."""
    out = []
    i = 0
    n = len(frag)
    while len(out) < read_len and i < n:
        if rng.random() < indel_rate:
            ln = min(int(rng.geometric(0.5)), 3)
            if rng.random() < 0.5:  # insertion
                out.extend(BASES[rng.integers(0, 4, ln)].tolist())
            else:  # deletion
                i += ln
            continue
        out.append(int(frag[i]))
        i += 1
    while len(out) < read_len:
        out.append(int(BASES[rng.integers(0, 4)]))
    r = np.asarray(out[:read_len], np.uint8)
    m = rng.random(read_len) < sub_rate
    if m.any():
        r[m] = BASES[(np.searchsorted(BASES, r[m]) + rng.integers(1, 4, m.sum())) % 4]
    return r


def make_workload(name: str, n_reads: int, ref_len: int, read_len: int = 150,
                  win_len: int = 250, cands: int = 4, sub_lo: float = 0.01,
                  sub_hi: float = 0.01, indel_rate: float = 0.001, repeat_frac: float = 0.0,
                  seed: int = 0x5EED, block: int = 0, ref: np.ndarray | None = None) -> Workload:
    """Reference from `seed`, then reads and candidate windows. Block 0 continues the
    reference's random stream; block b > 0 draws its reads from the stream (seed, b),
    so a job of several blocks shares one reference and block 0 is the one-block
    workload itself. `ref` (the same seed's reference) skips regenerating it."""
    rng = np.random.default_rng(seed)
    if ref is None:
        ref = random_reference(rng, ref_len, repeat_frac)
    elif block == 0:
        raise ValueError("block 0 continues the reference's stream: pass ref=None")
    if block:
        rng = np.random.default_rng([seed, block])
    slack = win_len - read_len
    origins = rng.integers(slack, ref_len - win_len - 8, n_reads)
    sub = rng.uniform(sub_lo, sub_hi, n_reads)
    has_indel = rng.random(n_reads) < 1.0 - (1.0 - indel_rate) ** read_len
    reads = ref[origins[:, None] + np.arange(read_len)[None, :]]
    m = rng.random((n_reads, read_len)) < sub[:, None]
    reads[m] = BASES[(np.searchsorted(BASES, reads[m]) + rng.integers(1, 4, int(m.sum()))) % 4]
    for r in np.nonzero(has_indel)[0]:
        o = int(origins[r])
        reads[r] = _mutate(rng, ref[o:o + read_len + 16], read_len, sub[r], indel_rate)
    n_pairs = n_reads * cands
    read_off = np.repeat(np.arange(n_reads, dtype=np.uint64) * read_len, cands)
    true_slot = rng.integers(0, cands, n_reads)
    win_off = rng.integers(0, ref_len - win_len, n_pairs).astype(np.uint64)
    lead = rng.integers(0, slack + 1, n_reads)
    true_idx = np.arange(n_reads) * cands + true_slot
    win_off[true_idx] = (origins - lead).astype(np.uint64)
    is_true = np.zeros(n_pairs, bool)
    is_true[true_idx] = True
    return Workload(name, ref, reads.reshape(-1), read_off,
                    np.full(n_pairs, read_len, np.uint32), win_off,
                    np.full(n_pairs, win_len, np.uint32), is_true)


def small(seed: int = 0x5EED) -> Workload:
    """1 Mbp, 10k x 150 bp reads, 4 windows of 250 bp each: 40k pairs."""
    return make_workload("small_40k_150x250", 10_000, 1_000_000, cands=4, sub_lo=0.01,
                         sub_hi=0.01, seed=seed)


def batched(seed: int = 0xB200, n_reads: int = 250_000, ref_len: int = 100_000_000,
            block: int = 0, ref: np.ndarray | None = None) -> Workload:
    """100 Mbp + 5 % repeats, 250k reads x 8 candidates = 2M pairs of 150 / 250 bp.
    Block b of a multi-block job (same reference, reads from the stream (seed, b))."""
    return make_workload("batched_2M_150x250", n_reads, ref_len, cands=8, sub_lo=0.005,
                         sub_hi=0.02, repeat_frac=0.05, seed=seed, block=block, ref=ref)


def batched_reference(seed: int = 0xB200, ref_len: int = 100_000_000) -> np.ndarray:
    """The reference of `batched` (the first draws of its seed's stream)."""
    return random_reference(np.random.default_rng(seed), ref_len, 0.05)


def batched_range(lo: int, hi: int, block_pairs: int = 2_000_000, seed: int = 0xB200,
                  ref_len: int = 100_000_000) -> Workload:
    """Pairs [lo, hi) of the job made of consecutive `batched` blocks of block_pairs
    pairs each (8 candidates per read): the blocks that overlap the range are
    generated and sliced, read arena compacted to the reads the range uses."""
    cands = 8
    if block_pairs % cands:
        raise ValueError("block_pairs must be a multiple of 8")
    n_reads = block_pairs // cands
    first, last = lo // block_pairs, max(lo, hi - 1) // block_pairs
    ref = None
    parts = []
    for b in range(first, last + 1):
        w = batched(seed, n_reads, ref_len, block=b, ref=ref if b else None)
        ref = w.reference if ref is None else ref
        a, e = max(lo - b * block_pairs, 0), min(hi - b * block_pairs, block_pairs)
        parts.append((w, a, e))
    reads, roff, rlen, woff, wlen, tru = [], [], [], [], [], []
    base = 0
    for w, a, e in parts:
        r0 = int(w.read_off[a]) if e > a else 0
        r1 = int(w.read_off[e - 1]) + int(w.read_len[e - 1]) if e > a else 0
        reads.append(w.reads[r0:r1])
        roff.append(w.read_off[a:e] - np.uint64(r0) + np.uint64(base))
        base += r1 - r0
        rlen.append(w.read_len[a:e])
        woff.append(w.win_off[a:e])
        wlen.append(w.win_len[a:e])
        tru.append(w.is_true[a:e])
    cat = np.concatenate
    return Workload(f"batched_pairs_{lo}_{hi}", ref if ref is not None else parts[0][0].reference,
                    cat(reads), cat(roff).astype(np.uint64), cat(rlen), cat(woff), cat(wlen),
                    cat(tru))


def _mutate_matrix(rng, frag: np.ndarray, q: np.ndarray, rate: np.ndarray,
                   split=(8, 1, 1)):
    """Vectorised read simulation: frag is (n, L) source bases (L >= 2 * max q);
    per output position an op M/S/I/D is drawn (error `rate` per read split
    subs:ins:del); D skips one source base. Returns (n, max q) reads."""
    n, L = frag.shape
    qm = int(q.max())
    tot = float(sum(split))
    u = rng.random((n, qm))
    r = rate[:, None]
    sub = u < r * split[0] / tot
    ins = (u >= r * split[0] / tot) & (u < r * (split[0] + split[1]) / tot)
    dele = (u >= r * (split[0] + split[1]) / tot) & (u < r)
    adv = np.where(ins, 0, np.where(dele, 2, 1)).astype(np.int32)
    src = np.cumsum(adv, axis=1) - adv + dele  # index of the base emitted at each position
    src = np.minimum(src, L - 1)
    out = np.take_along_axis(frag, src, axis=1)
    if sub.any():
        out[sub] = BASES[(np.searchsorted(BASES, out[sub]) + rng.integers(1, 4, int(sub.sum())))
                         % 4]
    if ins.any():
        out[ins] = BASES[rng.integers(0, 4, int(ins.sum()))]
    return out


@dataclass
class SwWorkload:
    """Independent (read, window, band offset, band) pairs for the banded SW."""
    name: str
    reads: np.ndarray
    read_off: np.ndarray
    read_len: np.ndarray
    wins: np.ndarray
    win_off: np.ndarray
    win_len: np.ndarray
    band_offset: np.ndarray
    bandwidth: np.ndarray
    reference: np.ndarray | None = None  # set when win_off are reference coordinates

    @property
    def n_pairs(self) -> int:
        return int(len(self.read_off))


def uneven(n_pairs: int = 500_000, seed: int = 0x3E3E, q_lo: int = 50, q_hi: int = 300,
           bands=(16, 32, 64, 128), err_hi: float = 0.03, ref_len: int = 20_000_000,
           resident: bool = False) -> SwWorkload:
    """Reads U[50, 300] bp, band uniform in {16, 32, 64, 128}, window = read + 2 x band
    with the read's origin at window offset band, errors U[0, 3 %] at 8:1:1. With
    `resident` the windows stay reference coordinates (wins None, reference set: the
    reference is device-resident), else they are copied into their own arena."""
    rng = np.random.default_rng(seed)
    ref = BASES[rng.integers(0, 4, ref_len)]
    q = rng.integers(q_lo, q_hi + 1, n_pairs).astype(np.int64)
    b = np.asarray(bands, np.int64)[rng.integers(0, len(bands), n_pairs)]
    w = q + 2 * b
    start = rng.integers(0, ref_len - int(w.max()) - q_hi - 64, n_pairs)
    L = q_hi + 48  # deletions beyond 48 per read clamp at the fragment end
    frag = ref[(start + b).astype(np.int32)[:, None] + np.arange(L, dtype=np.int32)[None, :]]
    rate = rng.uniform(0.0, err_hi, n_pairs)
    reads = _mutate_matrix(rng, frag, q, rate)
    mask = np.arange(reads.shape[1])[None, :] < q[:, None]
    read_arena = reads[mask]
    read_off = np.zeros(n_pairs, np.uint64)
    read_off[1:] = np.cumsum(q[:-1])
    if resident:
        return SwWorkload("uneven_500k_q50-300_band16-128",
                          np.concatenate([read_arena, np.zeros(16, np.uint8)]), read_off,
                          q.astype(np.uint32), None, start.astype(np.uint64), w.astype(np.uint32),
                          b.astype(np.int32), b.astype(np.int32), ref)
    win_off = np.zeros(n_pairs, np.uint64)
    win_off[1:] = np.cumsum(w[:-1])
    idx = np.repeat(start, w) + (np.arange(int(w.sum())) - np.repeat(win_off.astype(np.int64), w))
    wins = ref[idx]
    return SwWorkload("uneven_500k_q50-300_band16-128", np.concatenate([read_arena, np.zeros(16, np.uint8)]),
                      read_off, q.astype(np.uint32), np.concatenate([wins, np.zeros(16, np.uint8)]),
                      win_off, w.astype(np.uint32), b.astype(np.int32), b.astype(np.int32))


def random_genome(rng, ref_len: int, repeat_frac: float = 0.10) -> np.ndarray:
    """Uniform ACGT with `repeat_frac` of the bases in 300 bp repeat families
    (copies at 2-10 % divergence) -- the long-read reference of the gap-fill runs."""
    return random_reference(rng, ref_len, repeat_frac)


def gapfill(n_segments: int = 20_000, seed: int = 0x6A9F, seg_lo: int = 200, seg_hi: int = 2000,
            band: int = 256, err_lo: float = 0.05, err_hi: float = 0.12,
            reference: np.ndarray | None = None, ref_len: int = 50_000_000) -> SwWorkload:
    """Long-read gap-fill segments: U[200, 2000] bp of a long read between two exact
    anchors, error U[5 %, 12 %] at 2:1:1 (subs:ins:del), aligned with band 256 in a
    window of segment + 2 x band taken straight from the (device-resident) reference:
    win_off are reference coordinates and the segment starts at window offset band."""
    rng = np.random.default_rng(seed)
    ref = reference if reference is not None else random_genome(rng, ref_len)
    q = rng.integers(seg_lo, seg_hi + 1, n_segments).astype(np.int64)
    w = q + 2 * band
    start = rng.integers(0, len(ref) - int(w.max()) - seg_hi - 512, n_segments)
    L = seg_hi + 400  # room for deletions
    reads = np.empty((n_segments, seg_hi), np.uint8)
    for a in range(0, n_segments, 4096):  # bounded temporaries
        b = min(a + 4096, n_segments)
        frag = ref[(start[a:b] + band)[:, None] + np.arange(L)[None, :]]
        m = _mutate_matrix(rng, frag, q[a:b], rng.uniform(err_lo, err_hi, b - a),
                           split=(2, 1, 1))
        reads[a:b, :m.shape[1]] = m
    mask = np.arange(seg_hi)[None, :] < q[:, None]
    read_off = np.zeros(n_segments, np.uint64)
    read_off[1:] = np.cumsum(q[:-1])
    return SwWorkload(f"gapfill_{n_segments}_{seg_lo}-{seg_hi}_band{band}",
                      np.concatenate([reads[mask], np.zeros(16, np.uint8)]), read_off,
                      q.astype(np.uint32), None, start.astype(np.uint64), w.astype(np.uint32),
                      np.full(n_segments, band, np.int32), np.full(n_segments, band, np.int32),
                      ref)


@dataclass
class LongReadSegments(SwWorkload):
    """Gap-fill segments of simulated long reads (SwWorkload fields) plus, per
    segment, the read it came from; `read_bases` = bases of the simulated reads."""
    read_of: np.ndarray | None = None
    n_reads: int = 0
    read_bases: int = 0


def simulate_long_read(rng, ref: np.ndarray, length: int, err: float, split=(2, 1, 1)):
    """One long read drawn from `ref` at a random origin with error rate `err` split
    subs:ins:del. Returns (bases, origin, src, exact): src[p] = reference offset (from
    origin) of the base read position p copies or replaces, exact[p] = position p is
    an error-free base on the alignment's diagonal (a match with no gap before it)."""
    tot = float(sum(split))
    u = rng.random(length)
    sub = u < err * split[0] / tot
    ins = (u >= err * split[0] / tot) & (u < err * (split[0] + split[1]) / tot)
    dele = (u >= err * (split[0] + split[1]) / tot) & (u < err)
    adv = np.where(ins, 0, np.where(dele, 2, 1)).astype(np.int64)
    src = np.cumsum(adv) - adv + dele
    span = int(src[-1]) + 2
    origin = int(rng.integers(0, len(ref) - span - 1))
    out = ref[origin + src].copy()
    if sub.any():
        out[sub] = BASES[(np.searchsorted(BASES, out[sub]) + rng.integers(1, 4, int(sub.sum())))
                         % 4]
    if ins.any():
        out[ins] = BASES[rng.integers(0, 4, int(ins.sum()))]
    return out, origin, src, ~(sub | ins | dele)


def gapfill_reads(n_reads: int = 20_000, seed: int = 0x10C4, ref_len: int = 1_000_000_000,
                  repeat_frac: float = 0.10, mean: float = 10_000.0, sd: float = 6_000.0,
                  len_lo: int = 1_000, len_hi: int = 50_000, err_lo: float = 0.05,
                  err_hi: float = 0.12, split=(2, 1, 1), k: int = 15, seg_lo: int = 200,
                  seg_hi: int = 2_000, band: int = 256,
                  reference: np.ndarray | None = None) -> LongReadSegments:
    """Long-read gap-fill: reads of lognormal length (mean 10 kbp, sd 6 kbp, clipped to
    1-50 kbp) at error U[5 %, 12 %] (subs:ins:del 2:1:1) from a genome with 10 % repeat
    families, each split at exact k-mer anchors (k = 15 bases that match the reference
    on the read's diagonal) into the segments between consecutive anchors. Walking
    along a read, the next anchor is the first one that starts at least U[seg_lo,
    seg_hi - 150] bases after the previous anchor's end, so segments run 200-2000
    bases. Each segment is aligned with band `band` in a window of the reference gap
    between the anchors plus `band` bases on either side (win_off: reference
    coordinates; the segment starts at window offset `band`)."""
    rng = np.random.default_rng(seed)
    ref = reference if reference is not None else random_genome(rng, ref_len, repeat_frac)
    sig2 = np.log(1.0 + (sd / mean) ** 2)
    lengths = np.clip(rng.lognormal(np.log(mean) - sig2 / 2, np.sqrt(sig2), n_reads),
                      len_lo, len_hi).astype(np.int64)
    errs = rng.uniform(err_lo, err_hi, n_reads)
    seg_bases, q, wstart, wlen, read_of = [], [], [], [], []
    total = 0
    kernel = np.ones(k, np.int64)
    for r in range(n_reads):
        bases, origin, src, exact = simulate_long_read(rng, ref, int(lengths[r]), float(errs[r]),
                                                       split)
        total += len(bases)
        # run[p] = k: positions p-k+1..p are all exact (an anchor ends at p)
        run = np.convolve(exact.astype(np.int64), kernel, mode="full")[:len(bases)]
        ends = np.nonzero(run == k)[0]
        if len(ends) < 2:
            continue
        a_end = int(ends[0])  # the first anchor
        while True:
            target = a_end + 1 + int(rng.integers(seg_lo, seg_hi - 150 + 1))
            nxt = np.searchsorted(ends, target + k - 1)  # anchor starting at >= target
            if nxt >= len(ends):
                break
            b_end = int(ends[nxt])
            b_start = b_end - k + 1
            s0, s1 = a_end + 1, b_start  # segment = read[s0:s1]
            r0 = origin + int(src[a_end]) + 1  # reference gap [r0, r1)
            r1 = origin + int(src[b_start])
            if s1 > s0 and r1 > r0 and r0 - band >= 0 and r1 + band <= len(ref):
                seg_bases.append(bases[s0:s1])
                q.append(s1 - s0)
                wstart.append(r0 - band)
                wlen.append(r1 - r0 + 2 * band)
                read_of.append(r)
            a_end = b_end
    q = np.asarray(q, np.int64)
    read_off = np.zeros(len(q), np.uint64)
    read_off[1:] = np.cumsum(q[:-1])
    n = len(q)
    return LongReadSegments(
        f"gapfill_reads_{n_reads}_lognormal10k_band{band}",
        np.concatenate(seg_bases + [np.zeros(16, np.uint8)]), read_off, q.astype(np.uint32), None,
        np.asarray(wstart, np.uint64), np.asarray(wlen, np.uint32), np.full(n, band, np.int32),
        np.full(n, band, np.int32), ref, np.asarray(read_of, np.int32), n_reads, int(total))


def wfa_cascade(n_pairs: int = 2_000_000, seed: int = 0x3FA0, read_len: int = 150,
                band: int = 33, err_hi: float = 0.04, split=(4, 1, 1),
                reference: np.ndarray | None = None, ref_len: int = 50_000_000) -> SwWorkload:
    """Pairs of the WFA step of the cascade (try_fast_dp_alignment): a read of
    read_len bases against the text at its seed-implied start, read_len + band bases
    long (mod.rs:344-371: the window begins at the read's origin and carries band
    bases of trailing slack). Errors U[0, err_hi] per read at subs:ins:del = 4:1:1,
    the indel-bearing reads that reach WFA after the ungapped paths decline.
    win_off are reference coordinates (a device-resident reference)."""
    rng = np.random.default_rng(seed)
    ref = reference if reference is not None else random_genome(rng, ref_len)
    q = np.full(n_pairs, read_len, np.int64)
    w = q + band
    start = rng.integers(0, len(ref) - int(w.max()) - read_len - 64, n_pairs)
    L = read_len + 48
    reads = np.empty((n_pairs, read_len), np.uint8)
    for a in range(0, n_pairs, 1 << 18):  # bounded temporaries
        b = min(a + (1 << 18), n_pairs)
        frag = ref[start[a:b, None] + np.arange(L)[None, :]]
        reads[a:b] = _mutate_matrix(rng, frag, q[a:b], rng.uniform(0.0, err_hi, b - a),
                                    split=split)[:, :read_len]
    read_off = np.arange(n_pairs, dtype=np.uint64) * np.uint64(read_len)
    return SwWorkload(f"wfa_{n_pairs}_{read_len}_pad{band}",
                      np.concatenate([reads.reshape(-1), np.zeros(16, np.uint8)]), read_off,
                      q.astype(np.uint32), None, start.astype(np.uint64), w.astype(np.uint32),
                      np.zeros(n_pairs, np.int32), np.full(n_pairs, band, np.int32), ref)


@dataclass
class ChainWorkload:
    """Reads with one chain each over one contig (window = the whole contig)."""
    name: str
    reads: np.ndarray
    read_off: np.ndarray
    read_len: np.ndarray
    reference: np.ndarray
    chains: np.ndarray        # (ref_start, ref_end, read_start, read_end) per read, uint32
    is_top1: np.ndarray       # uint8
    score_margin: np.ndarray  # int32

    @property
    def n_pairs(self) -> int:
        return int(len(self.read_off))


def prefilter_chains(n_chains: int = 2_000_000, seed: int = 0x9F17, read_len: int = 150,
                     err_hi: float = 0.02, exact_frac: float = 0.3, indel_frac: float = 0.1,
                     ref_len: int = 50_000_000, reference: np.ndarray | None = None) -> ChainWorkload:
    """Stage-4 prefilter input: a read_len read per chain, errors U[0, err_hi] per
    read (8:1:1) except an exact_frac of error-free reads, and one chain per read
    over the contig. The chain is the read's co-linear anchor: read [s, e) with s
    in [0, 40) and e in (read_len - 40, read_len] (the whole read for error-free
    reads), ref_start = origin + s, and a ref span 1-3 bases off the read span for
    an indel_frac of chains (the indel-suspect case)."""
    rng = np.random.default_rng(seed)
    ref = reference if reference is not None else random_genome(rng, ref_len)
    n = n_chains
    origin = rng.integers(64, len(ref) - read_len - 128, n)
    L = read_len + 48
    rate = np.where(rng.random(n) < exact_frac, 0.0, rng.uniform(0.0, err_hi, n))
    reads = np.empty((n, read_len), np.uint8)
    for a in range(0, n, 1 << 18):
        b = min(a + (1 << 18), n)
        frag = ref[origin[a:b, None] + np.arange(L)[None, :]]
        reads[a:b] = _mutate_matrix(rng, frag, np.full(b - a, read_len), rate[a:b])[:, :read_len]
    exact = rate == 0.0
    s = np.where(exact, 0, rng.integers(0, 40, n))
    e = np.where(exact, read_len, read_len - rng.integers(0, 40, n))
    delta = np.where(rng.random(n) < indel_frac, rng.integers(1, 4, n) * rng.choice([-1, 1], n), 0)
    rs = origin + s
    chains = np.stack([rs, rs + (e - s) + delta, s, e], axis=1).astype(np.uint32)
    return ChainWorkload(f"prefilter_{n}_{read_len}",
                         np.concatenate([reads.reshape(-1), np.zeros(16, np.uint8)]),
                         np.arange(n, dtype=np.uint64) * np.uint64(read_len),
                         np.full(n, read_len, np.uint32), ref, chains,
                         (rng.random(n) < 0.9).astype(np.uint8),
                         rng.integers(-5, 40, n).astype(np.int32))


@dataclass
class ServingPool:
    """Pools the serving requests are cut from, over one shared reference."""
    reference: np.ndarray
    short: Workload     # reads U[100, 250] bp x 4 candidate windows (1 true)
    long: SwWorkload    # gap-fill segments, band 256


def short_reads(rng, ref: np.ndarray, n_reads: int, cands: int = 4, q_lo: int = 100,
                q_hi: int = 250, pad: int = 100, sub: float = 0.01,
                indel: float = 0.001) -> Workload:
    """Variable-length short reads (U[q_lo, q_hi]) with `cands` windows of read + pad
    each, one of them the read's origin; win_off are reference coordinates."""
    q = rng.integers(q_lo, q_hi + 1, n_reads).astype(np.int64)
    L = q_hi + 32
    origins = rng.integers(pad, len(ref) - q_hi - pad - 64, n_reads)
    frag = ref[origins[:, None] + np.arange(L)[None, :]]
    rate = np.full(n_reads, sub + 2 * indel)
    reads = _mutate_matrix(rng, frag, q, rate, split=(int(sub * 1000), int(indel * 1000),
                                                      int(indel * 1000)))[:, :q_hi]
    mask = np.arange(q_hi)[None, :] < q[:, None]
    roff = np.zeros(n_reads, np.uint64)
    roff[1:] = np.cumsum(q[:-1])
    n_pairs = n_reads * cands
    wl = np.repeat(q + pad, cands)
    win_off = rng.integers(0, len(ref) - q_hi - pad - 1, n_pairs).astype(np.uint64)
    true_slot = rng.integers(0, cands, n_reads)
    true_idx = np.arange(n_reads) * cands + true_slot
    win_off[true_idx] = (origins - rng.integers(0, pad + 1, n_reads)).astype(np.uint64)
    is_true = np.zeros(n_pairs, bool)
    is_true[true_idx] = True
    return Workload("short_reads", ref, np.concatenate([reads[mask], np.zeros(16, np.uint8)]),
                    np.repeat(roff, cands), np.repeat(q, cands).astype(np.uint32), win_off,
                    wl.astype(np.uint32), is_true)


def serving_pool(seed: int = 0x5E7E, ref_len: int = 1_000_000_000, short_reads_n: int = 400_000,
                 long_segments: int = 40_000) -> ServingPool:
    """1 Gbp reference (10 % repeats), a pool of short reads (x 4 windows) and a pool of
    gap-fill segments; requests are contiguous slices of the pools."""
    rng = np.random.default_rng(seed)
    ref = random_genome(rng, ref_len)
    sr = short_reads(rng, ref, short_reads_n)
    lg = gapfill(long_segments, seed=seed + 1, reference=ref)
    return ServingPool(ref, sr, lg)


def arrivals(seed: int, rate: float, duration_s: float, long_frac: float = 0.3,
             short_reads=(1_000, 64_000), long_reads=(50, 2_000)):
    """Seeded Poisson arrivals: (time_s, kind 'short'|'long', reads) per request."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration_s:
            return out
        if rng.random() < long_frac:
            out.append((t, "long", int(rng.integers(long_reads[0], long_reads[1] + 1))))
        else:
            out.append((t, "short", int(rng.integers(short_reads[0], short_reads[1] + 1))))
