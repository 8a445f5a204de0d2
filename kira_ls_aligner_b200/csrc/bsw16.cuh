// bsw16.cuh -- banded affine Smith-Waterman on packed int16 lanes (two cells per
// 32-bit register), bit-exact with the int32 sweep of bsw.cuh / banded_sw_with
// (src/alignment/mod.rs:1370-1650) whenever the host-side range check passes.
//
// Layout
//   A group of G lanes owns one pair. The row (capacity 2H cells, H = G*K) is cut
//   in two halves: word k of lane g holds cell c = g*K + k in its low 16 bits and
//   cell H + c in its high 16 bits, so every per-row quantity (band start, shift,
//   argmax, x-drop) stays one scalar per pair while the DP arithmetic runs two
//   cells per instruction with the DPX 16x2 forms (__viaddmax_s16x2,
//   __vimax_s16x2_relu, and the three-input __vimax3_s16x2_relu / __vimax3_u16x2
//   for the scan operand's lane maximum and the row-max keys).
//
// Biased values
//   Every DP value v is kept as v + B (B = bias >= gof + 2H*ge + mismatch + 1), so
//   all stored halves are non-negative and below 2^13 (checked on the host). That
//   makes plain 32-bit IADD/IADD3 exact on packed words (no carry crosses the
//   half boundary when each half's result stays in [0, 2^16)), and turns every
//   comparison into the sign of a biased difference: 2^p + a - b has bit p set iff
//   a >= b when |a - b| < 2^p. The four trace flags of a cell are produced that way
//   at distinct bit positions and merged with bit-select LOP3s: diag >= E, max(diag,
//   E) >= F, E extended, F not extended (bits 14..11 of words 0-1 of each group of
//   four, 15..12 of words 2-3, so one PRMT per word pair and one shift and one LOP3
//   per group pack them as 4-bit codes). Whether H > 0 is not stored: the traceback
//   carries the exact H, E or F value of the cell it stands on (from the end score,
//   the match / mismatch scores of its diagonal steps and the gap costs), and an H
//   of 0 is the stop.
//
// Band edges
//   Cells outside the previous row's band read as "neutral" (H = 0, E = the
//   biased floor 0): a diagonal predecessor out of band then contributes 0 + s
//   (the reference's scored-restart quirk, mod.rs:1464-1480) and an upper
//   predecessor out of band yields E = -gof instead of i32::MIN/4, which never
//   wins a cell, never ties a nonzero H and never sets an extend flag, so H,
//   directions and flags equal the reference's. The invariant is kept by masking
//   the cells at and beyond the row length after each row.
#pragma once

#include "common.cuh"

namespace kira {

template <int G, int K>
struct Bsw16Shape {
  static constexpr int kHalf = G * K;                  // cells per half row
  static constexpr int kCap = 2 * kHalf;               // cells per row
  static constexpr int kWords = (K + 1) / 2;           // window-byte words per lane
  static constexpr int kSlabs = (K + 3) / 4;           // 4-byte code stores per lane per row
  static constexpr int kLaneBytes = 4 * kSlabs;        // a 4-bit code per cell
  static constexpr int kRowStride = G * kLaneBytes;
  // Rows interleave in blocks of kInterleave: a block stores slab by slab, and in
  // each slab row by row, so one 128-byte line holds one slab of kInterleave
  // consecutive rows (the cells a diagonal traceback run reads next). One lane per
  // pair interleaves 8 rows (a 32-byte sector per slab), which keeps its
  // shared-memory staging strip (one block) small.
  static constexpr int kInterleave = G == 1 ? 8 : G >= 32 ? 1 : 32 / G;
  // Bytes of one interleave block of a group (its shared-memory staging strip).
  static constexpr int kStripBytes = kSlabs * kInterleave * G * 4;
  // Bits of the word index in a row-max key ((h << kKeyBits) | (max - k) per half).
  static constexpr int kKeyBits =
      K <= 2 ? 1 : K <= 4 ? 2 : K <= 8 ? 3 : K <= 16 ? 4 : K <= 32 ? 5 : 6;
  static_assert(K <= 64, "a row-max key holds 6 bits of word index");
};

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
  return r;
}

// Bits of `y` where m is set, bits of `x` elsewhere (one LOP3).
__device__ __forceinline__ uint32_t bsel(uint32_t x, uint32_t y, uint32_t m) {
  return (x & ~m) | (y & m);
}

// Both halves of a packed word as the same 16-bit value (two's complement).
__host__ __device__ __forceinline__ uint32_t pk2(int32_t v) {
  return ((uint32_t)v & 0xFFFFu) * 0x10001u;
}

// (lo, hi) as an integer sum hi * 2^16 + lo: the form that 32-bit IADD adds per
// half when both halves' results stay inside [0, 2^16).
__host__ __device__ __forceinline__ uint32_t isum(int32_t lo, int32_t hi) {
  return (uint32_t)hi * 65536u + (uint32_t)lo;
}

// __shfl_sync within a group of G lanes (a group of one lane reads itself).
template <int G>
__device__ __forceinline__ uint32_t gshfl(uint32_t gmask, uint32_t v, int src) {
  if constexpr (G == 1) return v;
  else return __shfl_sync(gmask, v, src, G);
}

// Window bytes of a lane's cells as the sweep keeps them (word j: bytes of cells 2j
// and 2j + 1 of the low half and of the high half, in the order lo 2j, hi 2j,
// lo 2j+1, hi 2j+1), from the two runs of bytes starting at `a` (low-half cells) and
// `b` (high-half cells). Aligned 4-byte loads and funnel shifts: no word loaded
// lies past the one holding the window's last byte `last`, so bytes past the window
// end are whatever that word holds (those cells are never active).
template <int K>
__device__ __forceinline__ void bsw16_window_words(uint32_t (&wb)[(K + 1) / 2],
                                                   const uint8_t* a, const uint8_t* b,
                                                   const uint8_t* last) {
  constexpr int NW = (K + 1) / 2;
  constexpr int NU = (K + 3) / 4;  // 4-byte runs per half: words 2m and 2m + 1
  const uintptr_t la = reinterpret_cast<uintptr_t>(last) & ~static_cast<uintptr_t>(3);
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a) & ~static_cast<uintptr_t>(3);
  const uintptr_t b0 = reinterpret_cast<uintptr_t>(b) & ~static_cast<uintptr_t>(3);
  const uint32_t sa = (static_cast<uint32_t>(reinterpret_cast<uintptr_t>(a)) & 3u) * 8u;
  const uint32_t sb = (static_cast<uint32_t>(reinterpret_cast<uintptr_t>(b)) & 3u) * 8u;
  auto at = [la](uintptr_t x) {
    return __ldg(reinterpret_cast<const uint32_t*>(x < la ? x : la));
  };
  uint32_t wa = at(a0), wv = at(b0);
#pragma unroll
  for (int m = 0; m < NU; ++m) {
    const uint32_t na = at(a0 + 4u * (m + 1)), nb = at(b0 + 4u * (m + 1));
    const uint32_t ua = __funnelshift_r(wa, na, sa), ub = __funnelshift_r(wv, nb, sb);
    wb[2 * m] = prmt(ua, ub, 0x5140u);
    if (2 * m + 1 < NW) wb[2 * m + 1 < NW ? 2 * m + 1 : 0] = prmt(ua, ub, 0x7362u);
    wa = na;
    wv = nb;
  }
}

// Realign the packed previous row by `s` cells (cell c <- old cell c + s); old
// cells outside [0, prev_len) become neutral. Each group stages the row as
// 16-bit halves in its own shared-memory strip [h: 2H][e: 2H].
template <int G, int K>
__device__ __forceinline__ void bsw16_realign(uint32_t (&ph)[K], uint32_t (&pe)[K], int32_t s,
                                              int32_t prev_len, uint16_t* buf, int32_t c0,
                                              uint32_t b2, uint32_t gmask) {
  constexpr int H = G * K;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    buf[c0 + k] = (uint16_t)(ph[k] & 0xFFFFu);
    buf[H + c0 + k] = (uint16_t)(ph[k] >> 16);
    buf[2 * H + c0 + k] = (uint16_t)(pe[k] & 0xFFFFu);
    buf[3 * H + c0 + k] = (uint16_t)(pe[k] >> 16);
  }
  __syncwarp(gmask);
  const uint32_t bias = b2 & 0xFFFFu;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int32_t a = c0 + k + s, b = H + c0 + k + s;
    const bool va = a >= 0 && a < prev_len, vb = b >= 0 && b < prev_len;
    const uint32_t hl = va ? (uint32_t)buf[a] : bias, hh = vb ? (uint32_t)buf[b] : bias;
    const uint32_t el = va ? (uint32_t)buf[2 * H + a] : 0u, eh = vb ? (uint32_t)buf[2 * H + b] : 0u;
    ph[k] = hl | (hh << 16);
    pe[k] = el | (eh << 16);
  }
  __syncwarp(gmask);
}

// Realignment by one cell in registers (the band stayed, or moved two columns):
// cell c <- old cell c - 1 (DOWN) or old cell c + 1 (up). The cells of the previous
// row at and beyond its length are already neutral, so only the cells shifted in
// from outside the row capacity (cell -1, cell 2H) need the neutral value: H = the
// bias, E = 0. Word k's halves hold cells g*K + k and H + g*K + k, so the cell
// before a lane's word 0 is the previous lane's word K - 1 (for lane 0: none in
// the low half, cell H - 1 = the last lane's low half in the high half), and the
// cell after its word K - 1 the next lane's word 0 (for the last lane: cell H =
// lane 0's high half in the low half, none in the high half).
template <int G, int K, bool DOWN>
__device__ __forceinline__ void bsw16_shift1(uint32_t (&ph)[K], uint32_t (&pe)[K], uint32_t b2,
                                             int32_t gi, uint32_t gmask) {
  if constexpr (DOWN) {
    uint32_t h = gshfl<G>(gmask, ph[K - 1], (gi + G - 1) & (G - 1));
    uint32_t e = gshfl<G>(gmask, pe[K - 1], (gi + G - 1) & (G - 1));
    if (gi == 0) {
      h = prmt(b2, h, 0x5410u);
      e = prmt(0u, e, 0x5410u);
    }
#pragma unroll
    for (int k = K - 1; k > 0; --k) {
      ph[k] = ph[k - 1];
      pe[k] = pe[k - 1];
    }
    ph[0] = h;
    pe[0] = e;
  } else {
    uint32_t h = gshfl<G>(gmask, ph[0], (gi + 1) & (G - 1));
    uint32_t e = gshfl<G>(gmask, pe[0], (gi + 1) & (G - 1));
    if (gi == G - 1) {
      h = prmt(h, b2, 0x5432u);
      e = prmt(e, 0u, 0x5432u);
    }
#pragma unroll
    for (int k = 0; k + 1 < K; ++k) {
      ph[k] = ph[k + 1];
      pe[k] = pe[k + 1];
    }
    ph[K - 1] = h;
    pe[K - 1] = e;
  }
}

// Activity mask of word k (0xFFFF per active half) from d0 = (2^15 + row_len - 1 -
// cell) per half of word 0: bit 15 of a half is set while its cell is inside the
// row, and PRMT replicates it over the half.
__device__ __forceinline__ uint32_t bsw16_act(uint32_t d0, int k) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBB99;" : "=r"(r) : "r"(d0 - (uint32_t)k * 0x10001u));
  return r;
}

// Trace rows go to global memory in whole interleave blocks. A group stages the
// slabs of its current block (kInterleave rows, kStripBytes, laid out exactly
// as in global memory) in its own shared-memory strip and, once the block is complete
// (or the sweep ends), one lane copies the strip out with one bulk asynchronous copy
// (cp.async.bulk shared -> global): every DRAM sector is written whole, once, and the
// per-row stores stay in shared memory. The strip is reused after the copy has read
// it (wait_group.read before the next block's first store).
struct TraceStage {
  uint32_t* strip;    // this group's shared-memory strip (16-byte aligned)
  uint8_t* gtrace;    // the item's trace slot in global memory
  uint32_t bytes;     // kStripBytes: one interleave block
  bool dirty = false;     // rows staged since the last copy
  bool inflight = false;  // a copy of the strip may still be reading it
  int32_t blk = 0;        // block the staged rows belong to

  // Before a store into the strip: the previous copy has finished reading it.
  __device__ __forceinline__ void ready(uint32_t g, uint32_t gmask) {
    if (inflight) {
      if (g == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      __syncwarp(gmask);
      inflight = false;
    }
  }
  // Copies the staged block out (the group's stores are made visible to the async
  // proxy first; lane 0 issues the copy).
  __device__ __forceinline__ void flush(uint32_t g, uint32_t gmask) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp(gmask);
    if (g == 0) {
      const uint32_t src = (uint32_t)__cvta_generic_to_shared(strip);
      const uint8_t* dst = gtrace + (size_t)blk * bytes;
      asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                   :: "l"(dst), "r"(src), "r"(bytes) : "memory");
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    inflight = true;
    dirty = false;
  }
};

// Waits until every bulk copy this thread issued has completed (end of a kernel).
__device__ __forceinline__ void bulk_copies_done() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

template <int G, int K>
__device__ __forceinline__ void bsw16_group_sweep(
    const uint8_t* __restrict__ rd, uint32_t q, const uint8_t* __restrict__ wn, uint32_t w,
    int32_t band, int32_t offset, int32_t abort_score, const SwParams& sp, int32_t bias,
    uint16_t* rowbuf, uint32_t* strip, uint8_t* __restrict__ trace, uint32_t* __restrict__ meta,
    uint32_t g, uint32_t gmask, DpEnd& out, uint64_t& cells_out) {
  constexpr int H = G * K;
  constexpr int NW = Bsw16Shape<G, K>::kWords;
  constexpr int NS = Bsw16Shape<G, K>::kSlabs;
  constexpr int R = Bsw16Shape<G, K>::kInterleave;
  TraceStage ts{strip, trace, (uint32_t)Bsw16Shape<G, K>::kStripBytes};
  const int32_t gi = (int32_t)g;
  const int32_t c0 = gi * K;
  const int32_t match = sp.match, mism = sp.mismatch, gof = sp.gof, ge = sp.gap_extend;
  // Packed constants (per-half two's complement for DPX, integer sums for IADD).
  const uint32_t B2 = pk2(bias);
  const uint32_t MAT2 = pk2(match), MIS2 = pk2(-mism), NGE2 = pk2(-ge);
  const uint32_t GOFS = isum(gof, gof);
  const uint32_t FOFS = isum(ge - gof, ge - gof);              // f = run - C_k + (ge - gof)
  const uint32_t C0 = isum(c0 * ge - gof, (H + c0) * ge - gof);  // C_k = idx*ge - gof
  const uint32_t GE2S = isum(ge, ge);
  // Per-half cell index of word 0 under 2^15 (the activity masks' d0 less row_len - 1).
  const uint32_t D0B = isum(0x8000 - 1 - c0, 0x8000 - 1 - H - c0);

  int32_t prev_start = 1, prev_len = 0;
  int32_t best = 0, bi = 0, bj = 0, bq = 0, bqj = 0;
  uint32_t early = 0;
  uint32_t cells = 0;  // < 2^32: read_len * row length
  const int32_t drift = sp.adaptive ? sp.max_drift : 0;
  int32_t acenter = 1 + offset;
  const int32_t wl = (int32_t)w;
  uint32_t ph[K], pe[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    ph[k] = B2;
    pe[k] = 0u;
  }
  // Window bytes of this lane's cells, four per word: word j holds cells 2j (low
  // half, high half) and 2j+1 (low, high) as bytes 0..3.
  uint32_t wb[NW];
#pragma unroll
  for (int j = 0; j < NW; ++j) wb[j] = 0u;

  // The read base of the next row is loaded a row ahead (its latency hides behind
  // the current row's work).
  uint32_t qb_next = q ? ldb(rd, 0) : 0u;
  uint32_t wnext = 0u;
  for (uint32_t iu = 1; iu <= q; ++iu) {
    const int32_t i = (int32_t)iu;
    const uint32_t qb = qb_next;
    if (iu < q) qb_next = ldb(rd, (uint64_t)iu);
    const int32_t sc = i + offset;
    const int32_t center = sp.adaptive ? min(max(acenter, sc - drift), sc + drift) : sc;
    const int32_t js = max(center - band, 1);
    const int32_t je = min(center + band, wl);
    if (js > je) {  // mod.rs:1437-1444: row skipped, no centre / x-drop update
      if (g == 0) meta[i] = (1u << 11);
      if (ts.dirty && (i & (R - 1)) == R - 1) ts.flush(g, gmask);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        ph[k] = B2;
        pe[k] = 0u;
      }
      prev_len = 0;
      prev_start = 1;
      continue;
    }
    const int32_t row_len = je - js + 1;
    cells += (uint32_t)row_len;
    const int32_t sft = js - prev_start - 1;
    if (sft != 0 && prev_len > 0) {
      if (sft == -1)
        bsw16_shift1<G, K, true>(ph, pe, B2, gi, gmask);
      else if (sft == 1)
        bsw16_shift1<G, K, false>(ph, pe, B2, gi, gmask);
      else
        bsw16_realign<G, K>(ph, pe, sft, prev_len, rowbuf, c0, B2, gmask);
    }
    // Upper neighbours of the last word: the next lane's first word; for the last
    // lane the low half continues into cell H (lane 0's high half) and the high
    // half runs past the capacity (neutral).
    uint32_t nh = gshfl<G>(gmask, ph[0], (gi + 1) & (G - 1));
    uint32_t ne = gshfl<G>(gmask, pe[0], (gi + 1) & (G - 1));
    if (gi == G - 1) {
      nh = prmt(nh, B2, 0x5432u);
      ne = prmt(ne, 0u, 0x5432u);
    }
    const uint8_t* wrow = wn + (js - 1);
    // The next row's new window byte if its band moves one column (index in
    // [js - 1, wl - 1]); used only by the group's last lane.
    const uint32_t wcur = wnext;
    if (gi == G - 1) wnext = __ldg(wn + js + min(2 * H - 1, wl - js - 1));
    // Window bytes: cells past the window end hold any byte (they are never active
    // in this or a later row); cells past the row end hold real window bytes, so
    // a row whose band moved one column takes the previous row's bytes shifted by
    // one cell (the group's last lane fetches the one new byte), and a row whose
    // band stayed keeps them.
    if (sft == 0 && prev_len > 0) {
      const uint32_t n0 = gshfl<G>(gmask, wb[0], (gi + 1) & (G - 1));
#pragma unroll
      for (int j = 0; j + 1 < NW; ++j) wb[j] = prmt(wb[j], wb[j + 1], 0x5432u);
      // The cell after this lane's last: the next lane's first (for the last lane,
      // cell H in the low half and wcur in the high half). wcur: this row's new
      // byte, loaded during the previous row on the guess that the band moves one
      // column (wrow + min(2H - 1, wl - js) for js = prev_start + 1).
      const uint32_t nx = gi == G - 1 ? prmt(n0, wcur, 0x0041u) : n0;
      // Odd K: the last word holds cell K - 1 alone; even K: cells K - 2 and K - 1.
      wb[NW - 1] = (K & 1) ? nx : prmt(wb[NW - 1], nx, 0x5432u);
    } else if (sft != -1 || prev_len == 0) {  // (the band stayed: same window bytes)
      bsw16_window_words<K>(wb, wrow + c0, wrow + H + c0, wn + (wl - 1));
    }
    // Activity: every word is masked in every row. (Groups of a warp sweep
    // different pairs; a separate unmasked form for full rows made the warp run
    // both forms whenever any of its groups had a short row at a band edge.)
    const uint32_t d0 = D0B + isum(row_len, row_len);
    uint32_t m1[K], code[K];
    {
      // Pass 1: E (+ extend flag), H_diag + s, the diag-vs-E flag, max(Hdiag+s, E)
      // and the F-scan operand G = max(Hdiag+s, E, 0) - gof + idx*ge (its lane
      // maximum). E is final here, so the previous row's E of word k is replaced at
      // once (word k reads only words k and k + 1 of the previous row).
      // Bit 7 of each byte of z: that cell's window base differs from the read base.
      const uint32_t qb4 = qb * 0x01010101u;
      // Two running maxima (alternate word pairs) halve the dependent chain.
      uint32_t z = 0u, lmax = 0u, lmax1 = 0u, gprev = 0u, glast = 0u;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if ((k & 1) == 0) {
          const uint32_t x = wb[k >> 1] ^ qb4;
          z = x | ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu);
        }
        const uint32_t uh = k + 1 < K ? ph[k + 1 < K ? k + 1 : 0] : nh;
        const uint32_t ue = k + 1 < K ? pe[k + 1 < K ? k + 1 : 0] : ne;
        // Flag bits: 14..11 for words 0-1 of each group of four, 15..12 for words 2-3.
        const uint32_t up = (k & 2) ? 1u : 0u;
        const uint32_t t = uh - GOFS;                      // H_up - gof
        const uint32_t e = __viaddmax_s16x2(ue, NGE2, t);  // max(E_up - ge, H_up - gof)
        const uint32_t yee = e + (0x0FFF0FFFu << up | (up ? 0x00010001u : 0u)) - t;  // e > t
        // 0xFFFF per mismatching half (sign of the cell's byte replicated).
        const uint32_t ms = prmt(z, 0u, (k & 1) ? 0xBBAAu : 0x9988u);
        const uint32_t s2 = bsel(MAT2, MIS2, ms);
        const uint32_t hm = __viaddmax_s16x2(ph[k], s2, B2);     // max(Hdiag + s, 0)
        const uint32_t y1 = hm + (0x40004000u << up) - e;  // hm >= e
        const uint32_t mm = __vimax_s16x2_relu(hm, e);
        code[k] = bsel(y1, yee, 0x10001000u << up);
        m1[k] = mm;
        const uint32_t gv = mm + C0 + (uint32_t)k * GE2S;
        if ((k & 1) && (k & 2))
          lmax1 = __vimax3_s16x2_relu(lmax1, gprev, gv);
        else if (k & 1)
          lmax = __vimax3_s16x2_relu(lmax, gprev, gv);
        else if (k == K - 1)
          lmax = __vimax3_s16x2_relu(lmax, lmax1, gv);
        if (k == K - 1 && (k & 1)) lmax = __vimax_s16x2_relu(lmax, lmax1);
        gprev = gv;
        if (k == K - 1) glast = gv;
        pe[k] = e & bsw16_act(d0, k);
      }
      // Cross-lane inclusive max-scan of G per half; exclusive value per lane, then
      // the high half also sees every low-half cell (they precede it in the row).
      uint32_t excl, tot, gp;
      if constexpr (G == 1) {  // one lane: nothing before it, the total is its own
        excl = 0u;
        tot = lmax;
        gp = glast;
      } else if constexpr (G == 2) {  // two lanes: one exchange gives both the prefix and the total
        const uint32_t other = __shfl_xor_sync(gmask, lmax, 1, G);
        gp = __shfl_xor_sync(gmask, glast, 1, G);
        tot = __vimax_s16x2_relu(lmax, other);
        excl = gi == 0 ? 0u : other;
      } else {
        uint32_t v = lmax;
#pragma unroll
        for (int off = 1; off < G; off <<= 1) {
          const uint32_t tt = __shfl_up_sync(gmask, v, off, G);
          if (gi >= off) v = __vimax_s16x2_relu(v, tt);
        }
        excl = __shfl_up_sync(gmask, v, 1, G);
        if (gi == 0) excl = 0u;
        tot = __shfl_sync(gmask, v, G - 1, G);
        gp = __shfl_sync(gmask, glast, (gi + G - 1) & (G - 1), G);
      }
      excl = __vimax_s16x2_relu(excl, prmt(tot, 0u, 0x1054u));
      if (gi == 0) gp = prmt(gp, 0u, 0x1054u);

      // Pass 2: F word by word (F' = max(F - ge, max(Hdiag+s, E) - gof), from the
      // scan's value for word 0), H, the remaining flags; neutralise inactive cells.
      uint32_t f = excl - C0 + FOFS;  // max over the row's earlier G - (idx - 1)*ge
      uint32_t tprev = 0u;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const uint32_t up = (k & 2) ? 1u : 0u;
        const uint32_t h = __vimax_s16x2_relu(m1[k], f);
        const uint32_t y2 = m1[k] + (0x20002000u << up) - f;  // max(hm, e) >= f
        // F not extended: word 0 by the scan (the previous cell's operand reaches
        // the running maximum), later words by F == max(hm, e)_prev - gof (F is
        // never below it).
        const uint32_t yfe = k == 0 ? gp + (0x08000800u << up) - excl
                                    : tprev + (0x08000800u << up) - f;
        code[k] = bsel(bsel(code[k], y2, 0x20002000u << up), yfe, 0x08000800u << up);
        const uint32_t t = m1[k] - GOFS;
        f = __viaddmax_s16x2(f, NGE2, t);
        tprev = t;
        ph[k] = bsel(B2, h, bsw16_act(d0, k));
      }
    }
    // 4-bit codes of words 4x .. 4x+3 in one 32-bit slab: byte (w & 1) * 2 + half
    // holds word w's cell in its low nibble for w < 2, its high nibble for w >= 2.
    // Layout [row block][slab][row in block][lane] of 4-byte slabs: a group's lanes
    // fill one contiguous G x 4-byte run per slab and row. The block is staged in
    // the group's strip and copied out whole (TraceStage).
    ts.ready(g, gmask);
    ts.blk = i / R;
    uint32_t* trow = ts.strip + (i & (R - 1)) * G + g;
#pragma unroll
    for (int x = 0; x < NS; ++x) {
      constexpr int kLast = K - 1;
      const int a = 4 * x, b = a + 1 <= kLast ? a + 1 : kLast, c = a + 2 <= kLast ? a + 2 : kLast,
                d = a + 3 <= kLast ? a + 3 : kLast;
      const uint32_t lo = prmt(code[a], code[b], 0x7531u);  // flags at bits 6..3 of each byte
      const uint32_t hi = a + 2 <= kLast ? prmt(code[c], code[d], 0x7531u) : 0u;  // bits 7..4
      trow[x * R * G] = bsel(hi, lo >> 3, 0x0F0F0F0Fu);
    }
    ts.dirty = true;
    if ((i & (R - 1)) == R - 1) ts.flush(g, gmask);
    if (g == 0) meta[i] = ((uint32_t)js << 11) | (uint32_t)row_len;

    // Row max and its first cell: per half the key (h << KB) | (KM - k), whose
    // unsigned maximum carries the lowest k holding the max; then one 32-bit key per
    // lane (low-half cells precede high-half cells on ties).
    constexpr int KB = Bsw16Shape<G, K>::kKeyBits;
    constexpr uint32_t KM = (1u << KB) - 1u;
    uint32_t mx = 0u, mx1 = 0u;  // two running maxima (alternate word pairs)
#pragma unroll
    for (int k = 0; k < K; k += 2) {
      const uint32_t ka = ph[k] * (1u << KB) + (KM - (uint32_t)k) * 0x10001u;
      const uint32_t kb = k + 1 < K ? ph[k + 1 < K ? k + 1 : 0] * (1u << KB) +
                                          (KM - (uint32_t)(k + 1)) * 0x10001u
                                    : 0u;
      if (k & 2)
        mx1 = __vimax3_u16x2(mx1, ka, kb);
      else
        mx = __vimax3_u16x2(mx, ka, kb);
    }
    mx = __vimax3_u16x2(mx, mx1, 0u);
    const uint32_t vlo = (mx & 0xFFFFu) >> KB, vhi = mx >> (16 + KB);
    const bool lo_first = vlo >= vhi;
    const uint32_t idx = lo_first ? (uint32_t)c0 + (KM - (mx & KM))
                                  : (uint32_t)(H + c0) + (KM - ((mx >> 16) & KM));
    uint32_t key = ((lo_first ? vlo : vhi) << 11) | (2047u - idx);
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) key = max(key, __shfl_xor_sync(gmask, key, off, G));
    const int32_t row_best = (int32_t)(key >> 11) - bias;
    const int32_t row_best_j = row_best > 0 ? js + (2047 - (int32_t)(key & 2047u)) : -1;
    if (row_best > best) {
      best = row_best;
      bi = i;
      bj = row_best_j;
    }
    if (iu == q && row_best > bq) {
      bq = row_best;
      bqj = row_best_j;
    }
    prev_start = js;
    prev_len = row_len;
    if (sp.adaptive) {  // mod.rs:1546-1559
      const int32_t raw = row_best_j >= 0 ? row_best_j + 1 : acenter + 1;
      const int32_t sn = i + 1 + offset;
      acenter = min(max(raw, sn - drift), sn + drift);
    }
    if (sp.dp_xdrop > 0 && best - row_best > sp.dp_xdrop) {  // mod.rs:1561-1564
      early = 1;
      break;
    }
    if (abort_score > kAbortOff) {  // mod.rs:1565-1572
      const int32_t remaining = (int32_t)(q - iu);
      if (best + remaining * match < abort_score) {
        early = 1;
        break;
      }
    }
  }
  // The last (partial) block, then the strip is free for the group's next item.
  if (ts.dirty) ts.flush(g, gmask);
  ts.ready(g, gmask);
  if (bq > 0 && sat_add(bq, sp.clip) > best) {  // mod.rs:1575-1579
    best = bq;
    bi = (int32_t)q;
    bj = bqj;
  }
  out.score = best;
  out.end_i = bi;
  out.end_j = bj;
  out.early_abort = early;
  cells_out = cells;
}

// Trace codes of the packed sweep. The 4-bit code of a cell: bit 3 diag >= E, bit
// 2 max(diag, E) >= F, bit 1 E extended, bit 0 F NOT extended (F always closes after
// one cell when the gap open is 0). The row holds two halves of G*K band cells; in
// each, lane gi keeps cells gi*K .. +K-1, word kk of lane gi in slab kk/4, stored as
// [row block][slab][row in block][lane] of 4-byte slabs (Bsw16Shape::kInterleave
// rows per block). Decoded into warp_walk's code layout; the H move is never "stop"
// here (the walk stops where its carried H is 0).
template <int G, int K, bool STAGED_META = false>
struct Bsw16Code {
  const uint8_t* __restrict__ trace;
  const uint32_t* __restrict__ meta;  // global, or the walk's shared-memory copy
  int32_t go;
  __device__ __forceinline__ uint32_t operator()(int32_t i, int32_t j) const {
    constexpr uint32_t H = Bsw16Shape<G, K>::kHalf, S = Bsw16Shape<G, K>::kRowStride;
    constexpr uint32_t R = Bsw16Shape<G, K>::kInterleave;
    const uint32_t m = STAGED_META ? meta[i] : __ldg(meta + i);
    const int32_t rs = (int32_t)(m >> 11), rl = (int32_t)(m & 2047u);
    const int32_t idx = j - rs;
    if (idx < 0 || idx >= rl) return 0xFFu;
    const uint32_t hi = (uint32_t)idx >= H ? 1u : 0u;
    const uint32_t c = (uint32_t)idx - hi * H;
    const uint32_t gi = c / (uint32_t)K, kk = c - gi * (uint32_t)K;
    const uint32_t ib = (uint32_t)i & (R - 1u);
    const uint32_t b = __ldg(trace + (size_t)((uint32_t)i - ib) * S +
                             ((kk >> 2) * R + ib) * (G * 4u) + gi * 4u + (kk & 1u) * 2u + hi);
    const uint32_t nib = (b >> ((kk & 2u) * 2u)) & 15u;
    const uint32_t h = !(nib & 4u) ? 3u : (nib & 8u) ? 1u : 2u;
    return h | ((nib & 2u) << 1) | ((go > 0 && !(nib & 1u)) ? 8u : 0u);
  }
};

// warp_walk (bsw.cuh) for codes without a stop move (rd / wn: the pair's read and
// window, in global or shared memory): the walk carries the exact
// value of the cell it stands on -- H in the H state, E or F in a gap -- starting
// from the end cell's score. A diagonal step from (i, j) lands on H(i, j) - s(i, j),
// s the match / mismatch score of read[i - 1] against window[j - 1] (raw bytes); a
// gap cell that extends adds gap_extend, the cell that opens it adds gap_open +
// gap_extend on the way back to H. An H state on a cell whose value is 0 stops the
// walk, as the reference's STOP move does (mod.rs:1587-1627). In a diagonal run the
// 32 lanes take one cell each: a ballot of the matching cells and the popcount of
// the lower lanes' bits give each lane's H, and a ballot finds the first cell that
// ends the run.
template <class Code>
__device__ __forceinline__ uint32_t warp_walk_scored(const Code& code, int32_t& i, int32_t& j,
                                                     int32_t v, const uint8_t* __restrict__ rd,
                                                     const uint8_t* __restrict__ wn,
                                                     const SwParams& sp, uint32_t* __restrict__ ops,
                                                     uint32_t cap, uint32_t& overflow) {
  const int32_t lane = (int32_t)(threadIdx.x & 31u);
  uint32_t state = 0;  // 0 H, 1 E, 2 F; also the CIGAR op the state emits (M, I, D)
  uint32_t n = 0, cur_op = 0xFFu, cur_len = 0;
  auto push = [&](uint32_t op, uint32_t cnt) {
    if (!cnt) return;
    if (op == cur_op) {
      cur_len += cnt;
      return;
    }
    if (cur_len) {
      if (n < cap) {
        if (lane == 0) ops[n] = (cur_len << 4) | cur_op;
      } else {
        overflow = 1;
      }
      ++n;
    }
    cur_op = op;
    cur_len = cnt;
  };
  while (i > 0 && j > 0) {
    const int32_t di = state != 2u ? 1 : 0, dj = state != 1u ? 1 : 0;
    const int32_t ci = i - lane * di, cj = j - lane * dj;
    const bool inside = ci > 0 && cj > 0;
    // A cell past row or column 0 ends the walk like the loop test does.
    const uint32_t c = inside ? code(ci, cj) : 0xFFu;
    bool cont;
    int32_t vt = v, step = 0;  // this lane's value; its diagonal step's score
    if (state == 0u) {
      // Steps before this lane: a ballot of the matching cells and a popcount of the
      // lower lanes' bits (no scan): sum = matches * match - mismatches * mismatch.
      const bool eq = inside && rd[ci - 1] == wn[cj - 1];
      step = eq ? sp.match : -sp.mismatch;
      const uint32_t eqm = __ballot_sync(0xffffffffu, eq);
      const int32_t before = __popc(eqm & ((1u << lane) - 1u));
      vt = v - before * (sp.match + sp.mismatch) + lane * sp.mismatch;
      cont = c != 0xFFu && vt != 0 && (c & 3u) == 1u;
    } else {
      cont = c != 0xFFu && (state == 1u ? (c & 4u) != 0u : (c & 8u) != 0u);
    }
    const uint32_t stop = __ballot_sync(0xffffffffu, !cont);
    const uint32_t t = stop ? (uint32_t)(__ffs(stop) - 1) : 32u;
    push(state, t);
    i -= (int32_t)t * di;
    j -= (int32_t)t * dj;
    if (state == 0u) {
      v = __shfl_sync(0xffffffffu, t < 32u ? vt : vt - step, t < 32u ? (int)t : 31);
    } else {
      v += (int32_t)t * sp.gap_extend;
    }
    if (t == 32u) continue;
    const uint32_t ct = __shfl_sync(0xffffffffu, c, (int)t);
    if (ct == 0xFFu) break;
    if (state == 0u) {
      if (v == 0) break;           // H == 0: the reference's STOP
      state = (ct & 3u) - 1u;      // E or F at the same cell (the same value)
    } else {                       // the gap's last cell, then back to H
      push(state, 1u);
      v += sp.gof;
      if (state == 1u) --i;
      else --j;
      state = 0u;
    }
  }
  if (cur_len) {
    if (n < cap) {
      if (lane == 0) ops[n] = (cur_len << 4) | cur_op;
    } else {
      overflow = 1;
    }
    ++n;
  }
  return n;
}

}  // namespace kira
