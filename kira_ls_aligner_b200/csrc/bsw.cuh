// bsw.cuh -- banded affine Smith-Waterman with adaptive band, x-drop, abort,
// clip-penalty end preference and 4-bit traceback (src/alignment/mod.rs:1370-1650).
//
// B200 mapping
//   A group of G lanes (G | 32) owns one pair and sweeps its rows in order; lane
//   g holds K consecutive cells idx = g*K .. g*K+K-1 of the row (G*K >= 2*band+1).
//   Row i+1's band depends on row i's argmax, so rows stay sequential (exactly as
//   the reference) and the parallelism is across the band and across pairs.
//   Per row:
//     1. H_diag / E from the previous row, read from a shared-memory row buffer at
//        the band shift d = j_start(i) - j_start(i-1) (any d, so the adaptive
//        re-centring costs nothing extra);
//     2. F exactly, without the serial left-to-right chain: with go >= 0,
//          F[idx] = max_{k<idx} (Hstar[k] - gof - (idx-1-k)*ge),  Hstar = max(Hdiag+s, E, 0)
//        i.e. an exclusive prefix max of Hstar[k] - gof + k*ge, done in-lane over K
//        cells and across lanes with log2(G) __shfl_up_sync steps;
//     3. H, the direction with the reference priority diag >= E >= F, and the E/F
//        extend flags; f_from_f > f_from_h reduces to "the prefix max of G before
//        cell idx-1 exceeds G[idx-1]" (and never holds when go == 0), so one
//        in-lane running max serves F, H and the flag;
//     4. row max and FIRST argmax with one packed key (h << 10 | 1023 - idx)
//        reduced by __shfl_xor_sync; best / x-drop / abort / adaptive centre are
//        then warp-uniform scalar updates.
//   The 4-bit trace (dir | E-ext << 2 | F-ext << 3, the reference's u8 trace code)
//   is written to a per-item slot of an HBM trace arena, two cells per byte, and
//   a separate kernel walks it with one thread per pair (thousands of
//   independent walks hide the dependent-load latency).
#pragma once

#include "common.cuh"

namespace kira {

template <int G, int K>
struct BswShape {
  static_assert(K <= 32, "the E-extend flags of a lane's cells are one 32-bit mask");
  static constexpr int kCap = G * K;                    // cells per row
  static constexpr int kWords = (K + 7) / 8;            // trace words per lane per row
  static constexpr int kLaneBytes = 4 * kWords;         // nibble k at byte k/2, half k&1
  static constexpr int kRowStride = G * kLaneBytes;
};

// The previous row stays in registers: ph[k] / pe[k] hold H / E of cell
// g*K + k + sh of the previous row, where `sh` is the realignment applied so far.
// With the band moving one column per row (d = j_start(i) - j_start(i-1) = 1,
// the common case for a read following its diagonal) the diagonal predecessor of
// cell idx is previous cell idx (same register) and the upper one is idx + 1 (next
// register, or lane g+1's first register via one shuffle). Rows with d != 1
// realign the registers through a transposed shared-memory buffer
// ([k][warp lane]: bank-conflict-free for every shift).
template <int G, int K>
__device__ __forceinline__ void bsw_realign(int32_t (&ph)[K], int32_t (&pe)[K], int32_t s,
                                            int32_t* buf, uint32_t lb, int32_t gi,
                                            uint32_t gmask) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
    buf[k * 32 + (int32_t)lb + gi] = ph[k];
    buf[(K + k) * 32 + (int32_t)lb + gi] = pe[k];
  }
  __syncwarp(gmask);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int32_t t = k + s;
    const int32_t tq = t >= 0 ? t / K : -((K - 1 - t) / K);  // floor(t / K)
    const int32_t tr = t - tq * K;
    const int32_t src = gi + tq;
    const bool ok = src >= 0 && src < G;  // outside: never read (masked by the bounds)
    const int32_t a = tr * 32 + (int32_t)lb + (ok ? src : gi);
    ph[k] = buf[a];
    pe[k] = buf[K * 32 + a];
  }
  __syncwarp(gmask);
}

// FULL = the full-window kernel of align_batch_simd (sw_batch_avx2_inner,
// src/alignment/mod.rs:1914-2135): every row covers columns 1..w, row 0 has H = 0
// and E = -16384, column 0 has H = 0 and F = -16384, no band, no x-drop. Within the
// i16 fit check of sw_batch_avx2 (mod.rs:1854-1868) the saturating i16 lanes never
// change an observable value, so exact int32 arithmetic reproduces them. The
// per-group "every lane done" abort break is resolved afterwards from the per-row
// keys written to `rowkeys` (bsw_full_resolve_kernel).
template <int G, int K, bool FULL>
__device__ __forceinline__ void bsw_group_sweep(
    const uint8_t* __restrict__ rd, uint32_t q, const uint8_t* __restrict__ wn, uint32_t w,
    int32_t band, int32_t offset, int32_t abort_score, const SwParams& sp, int32_t* rowbuf,
    uint32_t lb, uint8_t* __restrict__ trace, uint32_t* __restrict__ meta, uint32_t g,
    uint32_t gmask, DpEnd& out, uint64_t& cells_out, uint32_t* __restrict__ rowkeys) {
  constexpr int NW = BswShape<G, K>::kWords;
  constexpr int LB = BswShape<G, K>::kLaneBytes;
  constexpr int S = BswShape<G, K>::kRowStride;
  constexpr int32_t NEGBIG = INT32_MIN / 2;

  int32_t prev_start = 1, prev_len = 0;
  int32_t best = 0, bi = 0, bj = 0, bq = 0, bqj = 0;
  uint32_t early = 0;
  uint64_t cells = 0;
  const int32_t drift = sp.adaptive ? sp.max_drift : 0;
  int32_t acenter = 1 + offset;
  const int32_t match = sp.match, mism = sp.mismatch, gof = sp.gof, ge = sp.gap_extend;
  const int32_t go = sp.gap_open;
  const int32_t wl = (int32_t)w;
  const int32_t gi = (int32_t)g;
  const int32_t base_idx = gi * K;
  constexpr int32_t kNeg16 = -16384;  // row-0 E / column-0 F of the full-window kernel
  int32_t ph[K], pe[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    ph[k] = 0;
    pe[k] = FULL ? kNeg16 : kNeg4;
  }

  for (uint32_t iu = 1; iu <= q; ++iu) {
    const int32_t i = (int32_t)iu;
    const int32_t sc = i + offset;
    const int32_t center = sp.adaptive ? min(max(acenter, sc - drift), sc + drift) : sc;
    const int32_t js = FULL ? 1 : max(center - band, 1);
    const int32_t je = FULL ? wl : min(center + band, wl);
    if (js > je) {  // mod.rs:1437-1444: row skipped, no centre / x-drop update
      if (g == 0) meta[i] = (1u << 11);
      if (FULL && rowkeys && g == 0) rowkeys[i] = 0;
      prev_len = 0;
      prev_start = 1;
      continue;
    }
    const int32_t row_len = je - js + 1;
    cells += (uint64_t)row_len;
    const uint32_t qb = ldb(rd, (uint64_t)(i - 1));
    // Previous cell of diag = idx + s with s = d - 1; realign registers unless s == 0.
    // (Full window: the band never moves, diag = previous cell idx - 1, up = idx.)
    const int32_t sft = FULL ? -1 : js - prev_start - 1;
    if (!FULL && sft != 0 && prev_len > 0) bsw_realign<G, K>(ph, pe, sft, rowbuf, lb, gi, gmask);
    const int32_t lo = -sft, hi = prev_len - sft;  // valid previous cells: lo <= idx < hi
    const int32_t up_h1 = __shfl_down_sync(gmask, ph[0], 1, G);
    const int32_t up_e1 = __shfl_down_sync(gmask, pe[0], 1, G);
    const int32_t diag_left = FULL ? __shfl_up_sync(gmask, ph[K - 1], 1, G) : 0;
    const uint8_t* wrow = wn + (js - 1);

    // Pass 1: H_diag + s, E (with its extend flag) and the F-scan operand
    // G[idx] = max(Hdiag+s, E, 0) - gof + idx*ge.
    int32_t hm[K], e[K], gv[K];
    uint32_t eext = 0;
    int32_t lane_max = NEGBIG;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int32_t idx = base_idx + k;
      const bool act = idx < row_len;
      const uint32_t rb = act ? __ldg(wrow + idx) : 0x100u;
      const int32_t s = (qb == rb) ? match : -mism;
      int32_t uh, ue;
      bool uv;
      if (FULL) {
        const int32_t hd = k ? ph[k ? k - 1 : 0] : (g == 0 ? 0 : diag_left);
        hm[k] = hd + s;
        uv = true;
        uh = ph[k];
        ue = pe[k];
      } else {
        hm[k] = ((idx >= lo && idx < hi) ? ph[k] : 0) + s;
        uv = idx + 1 >= lo && idx + 1 < hi;
        uh = k + 1 < K ? ph[k + 1 < K ? k + 1 : 0] : up_h1;
        ue = k + 1 < K ? pe[k + 1 < K ? k + 1 : 0] : up_e1;
      }
      // max(uh - gof, ue - ge) and e_from_e > e_from_h, with gof = go + ge.
      e[k] = uv ? __viaddmax_s32(uh, -go, ue) - ge : kNeg4;
      eext |= (uv && ue + go > uh ? 1u : 0u) << k;
      gv[k] = __vimax_s32_relu(hm[k], e[k]) + ((FULL ? idx + 1 : idx) * ge - gof);
      lane_max = max(lane_max, gv[k]);
    }
    // Cross-lane scan: excl = max of G over all cells left of this lane.
    int32_t v = lane_max;
#pragma unroll
    for (int off = 1; off < G; off <<= 1) {
      const int32_t t = __shfl_up_sync(gmask, v, off, G);
      if ((int)g >= off) v = max(v, t);
    }
    int32_t excl = __shfl_up_sync(gmask, v, 1, G);
    const int32_t left_g = __shfl_up_sync(gmask, gv[K - 1], 1, G);
    // Full window: column 0 contributes G(0) = H(0) - gof = -gof and the F chain
    // seeded by F(0) = -16384 folds in as the constant -16384 - ge.
    if (g == 0) excl = FULL ? max(-gof, kNeg16 - ge) : NEGBIG;
    // Pass 2 (in-lane running max): F[idx] = max_{k<idx} G[k] - (idx-1)*ge,
    // H = max(Hdiag+s, E, F, 0) with the diag >= E >= F priority (mod.rs:1504-1516),
    // F-extend = f_from_f > f_from_h = go > 0 && max_{k<idx-1} G[k] > G[idx-1].
    uint32_t key = 0;
    uint32_t tw[NW];
#pragma unroll
    for (int x = 0; x < NW; ++x) tw[x] = 0;
    int32_t run = excl;  // max of G over the cells before idx
    int32_t g_prev = g == 0 ? (FULL ? -gof : NEGBIG) : left_g;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int32_t idx = base_idx + k;
      const bool act = idx < row_len;
      const int32_t f = FULL ? run - idx * ge : (idx >= 1 ? run - (idx - 1) * ge : kNeg4);
      const int32_t h = __vimax3_s32_relu(hm[k], e[k], f);
      const uint32_t dir = h == 0 ? 0u : (h == hm[k] ? 1u : (h == e[k] ? 2u : 3u));
      // F-extend of cell idx: max of G strictly before idx-1 exceeds G[idx-1];
      // run = max(that, G[idx-1]), so the test is run > G[idx-1]. With go == 0
      // f_from_f > f_from_h would need F[idx-1] > H[idx-1] >= F[idx-1]: never.
      const bool fext = go > 0 && (FULL || idx >= 1) && run > g_prev;
      const uint32_t nib = dir | (((eext >> k) & 1u) << 2) | (fext ? 8u : 0u);
      tw[k / 8] |= (act ? nib : 0u) << (4 * (k % 8));
      const uint32_t kk = ((uint32_t)h << kKeyIdxBits) | (uint32_t)(1023 - idx);
      key = act ? max(key, kk) : key;
      ph[k] = h;
      pe[k] = e[k];
      g_prev = gv[k];
      run = max(run, gv[k]);
    }
    uint32_t* trow = reinterpret_cast<uint32_t*>(trace + (size_t)i * S + (size_t)g * LB);
#pragma unroll
    for (int x = 0; x < NW; ++x) trow[x] = tw[x];
    if (g == 0) meta[i] = ((uint32_t)js << 11) | (uint32_t)row_len;
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) key = max(key, __shfl_xor_sync(gmask, key, off, G));
    if (FULL && rowkeys && g == 0) rowkeys[i] = key;
    const int32_t row_best = (int32_t)(key >> kKeyIdxBits);
    const int32_t row_best_j = row_best > 0 ? js + (1023 - (int32_t)(key & 1023u)) : -1;
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
    if (FULL) continue;  // no centre, x-drop or abort inside the full-window sweep
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
  // Clip-penalty end preference (mod.rs:1575-1579).
  if (bq > 0 && sat_add(bq, sp.clip) > best) {
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

// Traceback state machine of mod.rs:1581-1627, one warp per item. The 32 lanes
// read the next 32 cells of the current run at once (diagonal in H, up in E, left
// in F) and a ballot finds the first cell that ends it, so a run costs one memory
// round trip per 32 cells instead of one per cell; the moves, their tie order and
// the CIGAR are those of the one-cell-at-a-time walk. `code(i, j)` gives a cell's
// trace code: bits 0-1 the H move (0 stop, 1 diagonal, 2 E, 3 F), bit 2 E
// extended, bit 3 F extended, 0xFF outside the row's band. CIGAR runs are written
// in reverse order into `ops` by lane 0 (the compaction kernel reverses them).
template <class Code>
__device__ __forceinline__ uint32_t warp_walk(const Code& code, int32_t& i, int32_t& j,
                                              uint32_t* __restrict__ ops, uint32_t cap,
                                              uint32_t& overflow) {
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
    // A cell past row or column 0 ends the walk like the loop test does.
    const uint32_t c = (ci > 0 && cj > 0) ? code(ci, cj) : 0xFFu;
    const bool cont = c != 0xFFu && (state == 0u   ? (c & 3u) == 1u
                                     : state == 1u ? (c & 4u) != 0u
                                                   : (c & 8u) != 0u);
    const uint32_t stop = __ballot_sync(0xffffffffu, !cont);
    const uint32_t t = stop ? (uint32_t)(__ffs(stop) - 1) : 32u;
    push(state, t);
    i -= (int32_t)t * di;
    j -= (int32_t)t * dj;
    if (t == 32u) continue;
    const uint32_t ct = __shfl_sync(0xffffffffu, c, (int)t);
    if (ct == 0xFFu) break;
    if (state == 0u) {
      if ((ct & 3u) == 0u) break;  // H == 0
      state = (ct & 3u) - 1u;      // E or F at the same cell
    } else {                       // the gap's last cell, then back to H
      push(state, 1u);
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

// Trace codes of the int32 sweep of shape <G, K>: one nibble per cell, already in
// warp_walk's code layout; lane gi of the row holds band cells gi*K .. +K-1.
template <int G, int K>
struct BswCode {
  const uint8_t* __restrict__ trace;
  const uint32_t* __restrict__ meta;
  __device__ __forceinline__ uint32_t operator()(int32_t i, int32_t j) const {
    constexpr uint32_t LB = BswShape<G, K>::kLaneBytes, S = BswShape<G, K>::kRowStride;
    const uint32_t m = __ldg(meta + i);
    const int32_t rs = (int32_t)(m >> 11), rl = (int32_t)(m & 2047u);
    const int32_t idx = j - rs;
    if (idx < 0 || idx >= rl) return 0xFFu;
    const uint32_t gi = (uint32_t)idx / (uint32_t)K, kk = (uint32_t)idx - gi * (uint32_t)K;
    const uint32_t byte = __ldg(trace + (size_t)i * S + gi * LB + (kk >> 1));
    return (byte >> ((kk & 1u) * 4u)) & 15u;
  }
};

}  // namespace kira
