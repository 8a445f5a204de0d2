// wfa.cu -- the WFA batch kernel (wfa.cuh) and its CIGAR compaction.
#include <cuda_runtime.h>

#include "internal.h"
#include "wfa.cuh"

namespace kira {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

// router::wfa_score_budget (src/alignment/router.rs:160-165).
__device__ __forceinline__ int32_t wfa_budget(int read_len, const WfaLaunch& L) {
  const int64_t mism = (int64_t)read_len * L.budget_pct / 100 * L.budget_x;
  const int64_t indel = ((int64_t)L.budget_o + (int64_t)L.budget_e * 4) * 3;
  const int64_t b = mism > indel ? mism : indel;
  return b > INT32_MAX ? INT32_MAX : (int32_t)b;
}

__device__ __forceinline__ int wfa_low_bit(unsigned b) { return __ffs(b) - 1; }
__device__ __forceinline__ int wfa_high_bit(unsigned b) { return 31 - __clz(b); }

// Traceback in one lane (build_cigar, wfa.rs:762-952). Ops are pushed in reverse
// order into the pair's slot with push_cigar's merging (wfa.rs:954-962); returns
// the diagonal at termination (the alignment's text start). get(layer, score, k)
// returns the stored offset or kWfaNone.
template <class Get>
__device__ int wfa_traceback_t(const WfaLaunch& L, Get get, const uint32_t* pw,
                               const uint32_t* tw, int m, int n, int s, int k,
                               uint32_t* __restrict__ slot, uint32_t& nops, bool& overflow) {
  uint32_t last = 0xFFFFFFFFu;  // op of the newest entry
  auto push = [&](uint32_t op, uint32_t len) {
    if (last == op) {
      if (nops <= L.slot_cap) slot[nops - 1] += len << 4;
      return;
    }
    if (nops < L.slot_cap) slot[nops] = (len << 4) | op;
    else overflow = true;
    ++nops;
    last = op;
  };
  const int x = L.x, oi = L.o + L.ei, od = L.o + L.ed;
  int off = m, layer = 0;
  for (uint32_t guard = 0; guard < (uint32_t)(2 * (m + n) + 8); ++guard) {
    if (s == 0 && layer == 0 && off == 0) break;
    if (layer == 0) {
      const int iv = get(1, s, k), dv = get(2, s, k);
      const int pv = s >= x ? get(0, s - x, k) : kWfaNone;
      // The walk stops at the first landing point of an edge at or below off.
      int low = max(0, -k);
      if (iv != kWfaNone && iv <= off) low = max(low, iv);
      if (dv != kWfaNone && dv <= off) low = max(low, dv);
      if (pv != kWfaNone && pv + 1 <= off) low = max(low, pv + 1);
      const int run = (off > low && off - 1 < m && off - 1 + k < n) ? wfa_back_run(pw, tw, k, off, low)
                                                                    : 0;
      if (run > 0) push(0u, (uint32_t)run);
      off -= run;
      if (s == 0 && off == 0) break;
      if (pv != kWfaNone && pv + 1 == off) {
        push(0u, 1u);
        off -= 1;
        s -= x;
      } else if (iv == off) {
        layer = 1;
      } else if (dv == off) {
        layer = 2;
      } else {
        break;
      }
    } else if (layer == 1) {
      const int a = s >= oi ? get(0, s - oi, k + 1) : kWfaNone;
      if (a != kWfaNone && a + 1 == off) {
        push(1u, 1u);
        off -= 1, k += 1, s -= oi, layer = 0;
        continue;
      }
      const int b = s >= L.ei ? get(1, s - L.ei, k + 1) : kWfaNone;
      if (b != kWfaNone && b + 1 == off) {
        push(1u, 1u);
        off -= 1, k += 1, s -= L.ei;
        continue;
      }
      break;
    } else {
      const int a = s >= od ? get(0, s - od, k - 1) : kWfaNone;
      if (a != kWfaNone && a == off) {
        push(2u, 1u);
        k -= 1, s -= od, layer = 0;
        continue;
      }
      const int b = s >= L.ed ? get(2, s - L.ed, k - 1) : kWfaNone;
      if (b != kWfaNone && b == off) {
        push(2u, 1u);
        k -= 1, s -= L.ed;
        continue;
      }
      break;
    }
  }
  return k;
}

__device__ int wfa_traceback(const WfaLaunch& L, const int2* __restrict__ meta,
                             const int16_t* __restrict__ H, const uint32_t* pw,
                             const uint32_t* tw, int m, int n, int s, int k,
                             uint32_t* __restrict__ slot, uint32_t& nops, bool& overflow) {
  auto get = [&](int layer, int sc, int kk) -> int {
    if (sc < 0) return kWfaNone;
    return wfa_get(H, wfa_unpack(meta[(uint32_t)sc * 3u + layer]), kk);
  };
  return wfa_traceback_t(L, get, pw, tw, m, n, s, k, slot, nops, overflow);
}

// G lanes align one pair; the 32 / G groups of a warp step in lockstep through
// an outer loop of three phases so that their warp instructions are shared:
//   fetch   -- groups without a pair take the next one and stage its bytes;
//   step    -- every group in the forward search computes its next score;
//   finish  -- groups whose search ended write the result (traceback in the
//              group's first lane).
// Sync primitives run on the full warp outside divergent code; each group reads
// its own bits of the ballots and shuffles from its own lanes.
template <int G, bool TB>
__global__ void __launch_bounds__(128) wfa_kernel(DevPairs P, WfaLaunch L) {
  constexpr int NG = 32 / G;
  constexpr unsigned kGroupBits = G == 32 ? kFull : ((1u << G) - 1u);
  extern __shared__ __align__(16) uint8_t wfa_smem[];
  const int lane = threadIdx.x & 31;
  const int g = lane / G, gl = lane % G, gbase = g * G;
  const unsigned gmask = kGroupBits << gbase;
  const uint32_t wib = threadIdx.x >> 5;
  const uint32_t grp = (blockIdx.x * (blockDim.x >> 5) + wib) * NG + (uint32_t)g;
  uint8_t* my = wfa_smem + (size_t)(wib * NG + (uint32_t)g) * L.smem_group;
  uint8_t* scr = L.scratch + (size_t)grp * L.group_bytes;
  int2* ring = L.ring_bytes ? (int2*)my : (int2*)(scr + L.ring_goff);
  uint32_t* pw = (uint32_t*)(my + L.ring_bytes + 16);
  uint32_t* tw = (uint32_t*)(my + L.ring_bytes + L.pat_region + 16);
  uint8_t* pb = (uint8_t*)pw;
  uint8_t* tb = (uint8_t*)tw;
  int2* meta = (int2*)scr;  // traceback: every score
  int16_t* H = (int16_t*)(scr + L.hist_off);
  const int x = L.x, oi = L.o + L.ei, od = L.o + L.ed;
  const uint32_t R = L.ring_len;

  int phase = 0;  // 0: needs a pair, 1: forward search, 2: no pairs left
  uint32_t p = 0, top = 0;
  int m = 0, n = 0, S_loop = 0, tbf = 0, s = 0, last_live = 0;
  for (;;) {
    // ---- fetch
    if (phase == 0) {
      uint32_t q = 0;
      if (gl == 0) q = atomicAdd(L.work, 1u);
      q = __shfl_sync(gmask, q, gbase);
      if (q >= (L.list ? min(*L.list_count, L.n) : L.n)) {
        phase = 2;
      } else {
        p = L.list ? L.list[q] : q;
        m = (int)P.read_len[p];
        n = (int)P.win_len[p];
        if (!L.valid || m == 0) {  // WfaCosts::scored refused: None; empty read: wfa.rs:555-563
          if (gl == 0) {
            kira_wfa_result res{};
            res.cost = L.valid ? 0 : -1;
            res.found = L.valid ? 1u : 0u;
            L.out[p] = res;
            if (TB) L.ncig[p] = 0;
          }
        } else {
          const uint8_t* rs = P.read_seq + P.read_off[p];
          const uint8_t* ws = P.win_seq + P.win_off[p];
          for (int i = gl; i < m; i += G) pb[i] = __ldg(rs + i);
          for (int i = gl; i < n; i += G) tb[i] = __ldg(ws + i);
          int S = L.max_score_pp ? L.max_score_pp[p] : L.max_score;
          if (!L.max_score_pp && S < 0) S = wfa_budget(m, L);
          // The all-insertion path reaches the pattern end by cost o + ei*m, so
          // the exact search ends by then; a pruned search advances its furthest
          // point by an antidiagonal at least every max(x, o + ei).
          const int64_t cap = L.drop < 0 ? (int64_t)L.o + (int64_t)L.ei * m
                                         : (int64_t)max(x, oi) * (2 * m + n + 2);
          S_loop = (int)max((int64_t)0, min((int64_t)S, cap));  // score 0 always runs
          tbf = L.tbf_pp ? L.tbf_pp[p] : L.tbf;
          tbf = min(max(tbf, 0), max(n - 1, 0));
          s = 0;
          top = 0;
          last_live = 0;
          phase = 1;
        }
      }
    }
    __syncwarp();
    if (__all_sync(kFull, phase == 2)) break;

    // ---- one score step of every searching group
    const bool fwd = phase == 1;
    int2 mv = wfa_empty();
    if (fwd && s > 0 && gl < 5) {  // M[s-x], M[s-o-ei], M[s-o-ed], I[s-ei], D[s-ed]
      const int sc = gl == 0 ? s - x : gl == 1 ? s - oi : gl == 2 ? s - od
                     : gl == 3 ? s - L.ei : s - L.ed;
      const int layer = gl < 3 ? 0 : gl - 2;
      if (sc >= 0 && sc < s) mv = ring[((uint32_t)sc % R) * 3u + layer];
    }
    WfaWave src[5];
#pragma unroll
    for (int t = 0; t < 5; ++t)
      src[t] = wfa_unpack(make_int2(__shfl_sync(kFull, mv.x, gbase + t),
                                    __shfl_sync(kFull, mv.y, gbase + t)));
    const WfaWave& mx = src[0];
    const WfaWave& moi = src[1];
    const WfaWave& mod = src[2];
    const WfaWave& ie = src[3];
    const WfaWave& de = src[4];
    int ilo = INT32_MAX, ihi = INT32_MIN, dlo = INT32_MAX, dhi = INT32_MIN;
    int mlo = INT32_MAX, mhi = INT32_MIN;
    if (fwd) {
      if (s == 0) {
        mlo = 0;
        mhi = tbf;
      } else {
        if (moi.hi >= moi.lo) ilo = min(ilo, moi.lo - 1), ihi = max(ihi, moi.hi - 1);
        if (ie.hi >= ie.lo) ilo = min(ilo, ie.lo - 1), ihi = max(ihi, ie.hi - 1);
        if (mod.hi >= mod.lo) dlo = min(dlo, mod.lo + 1), dhi = max(dhi, mod.hi + 1);
        if (de.hi >= de.lo) dlo = min(dlo, de.lo + 1), dhi = max(dhi, de.hi + 1);
        if (mx.hi >= mx.lo) mlo = min(mlo, mx.lo), mhi = max(mhi, mx.hi);
        if (ilo <= ihi) mlo = min(mlo, ilo), mhi = max(mhi, ihi);
        if (dlo <= dhi) mlo = min(mlo, dlo), mhi = max(mhi, dhi);
      }
    }
    const int iw = ilo <= ihi ? ihi - ilo + 1 : 0;
    const int dw = dlo <= dhi ? dhi - dlo + 1 : 0;
    const int mw = mlo <= mhi ? mhi - mlo + 1 : 0;
    uint32_t ib = 0, db = 0, mb = 0;
    int fin = 0;  // 1: found, 2: no alignment, 3: history bound exceeded
    if (fwd) {
      if (TB) {
        ib = top;
        db = ib + (uint32_t)iw;
        mb = db + (uint32_t)dw;
        top = mb + (uint32_t)mw;
        if (top > L.hist_cap || (uint32_t)s >= L.meta_slots) fin = 3;
      } else {
        const uint32_t sl = ((uint32_t)s % R) * 3u * L.ring_width;
        mb = sl;
        ib = sl + L.ring_width;
        db = sl + 2u * L.ring_width;
        if ((uint32_t)max(mw, max(iw, dw)) > L.ring_width) fin = 3;
      }
    }
    const int nch = fwd && !fin ? (mw + G - 1) / G : 0;
    const int maxch = __reduce_max_sync(kFull, nch);

    // Pass 1: I, D, M per diagonal; extension; trimming and done ballots.
    int ifirst = INT32_MAX, ilast = INT32_MIN, dfirst = INT32_MAX, dlast = INT32_MIN;
    int mfirst = INT32_MAX, mlast = INT32_MIN, kdone = INT32_MAX, mad = INT32_MIN;
    for (int c = 0; c < maxch; ++c) {
      const int c0 = mlo + c * G;
      const int k = c0 + gl;
      const bool act = c < nch && k <= mhi;
      int vi = kWfaNone, vd = kWfaNone, vm = kWfaNone;
      if (act) {
        if (s == 0) {
          vm = 0;
        } else {
          if (k >= ilo && k <= ihi) {
            const int a = wfa_get(H, moi, k + 1), b = wfa_get(H, ie, k + 1);
            if (a != kWfaNone && a < m) vi = max(vi, a + 1);
            if (b != kWfaNone && b < m) vi = max(vi, b + 1);
            H[ib + (uint32_t)(k - ilo)] = wfa_enc(vi);
          }
          if (k >= dlo && k <= dhi) {
            const int a = wfa_get(H, mod, k - 1), b = wfa_get(H, de, k - 1);
            if (a != kWfaNone && a + k <= n) vd = max(vd, a);
            if (b != kWfaNone && b + k <= n) vd = max(vd, b);
            H[db + (uint32_t)(k - dlo)] = wfa_enc(vd);
          }
          const int a = wfa_get(H, mx, k);
          if (a != kWfaNone && a < m && a + k < n) vm = a + 1;
          vm = max(vm, max(vi, vd));
        }
        if (vm != kWfaNone) {
          vm = wfa_extend(pw, tw, m, n, k, vm);
          mad = max(mad, 2 * vm + k);
        }
        H[mb + (uint32_t)(k - mlo)] = wfa_enc(vm);
      }
      const unsigned bi = (__ballot_sync(kFull, vi != kWfaNone) >> gbase) & kGroupBits;
      const unsigned bd = (__ballot_sync(kFull, vd != kWfaNone) >> gbase) & kGroupBits;
      const unsigned bm = (__ballot_sync(kFull, vm != kWfaNone) >> gbase) & kGroupBits;
      const unsigned bx = (__ballot_sync(kFull, act && vm >= m) >> gbase) & kGroupBits;
      if (bi) ifirst = min(ifirst, c0 + wfa_low_bit(bi)), ilast = c0 + wfa_high_bit(bi);
      if (bd) dfirst = min(dfirst, c0 + wfa_low_bit(bd)), dlast = c0 + wfa_high_bit(bd);
      if (bm) mfirst = min(mfirst, c0 + wfa_low_bit(bm)), mlast = c0 + wfa_high_bit(bm);
      if (bx && kdone == INT32_MAX) kdone = c0 + wfa_low_bit(bx);
    }
    // Pass 2 (adaptive): prune_wavefront on the extended M, then the done test.
    if (L.drop >= 0) {
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) mad = max(mad, __shfl_xor_sync(kFull, mad, o));
      const bool prune = nch > 0 && mfirst <= mlast;
      const int th = prune ? mad - L.drop : 0;
      if (prune) mfirst = INT32_MAX, mlast = INT32_MIN, kdone = INT32_MAX;
      for (int c = 0; c < maxch; ++c) {
        const int c0 = mlo + c * G;
        const int k = c0 + gl;
        int v = kWfaNone;
        if (prune && c < nch && k <= mhi) {
          const uint32_t at = mb + (uint32_t)(k - mlo);
          v = wfa_dec(H[at]);
          if (v != kWfaNone && 2 * v + k < th) {
            v = kWfaNone;
            H[at] = wfa_enc(v);
          }
        }
        const unsigned bm = (__ballot_sync(kFull, v != kWfaNone) >> gbase) & kGroupBits;
        const unsigned bx = (__ballot_sync(kFull, v != kWfaNone && v >= m) >> gbase) & kGroupBits;
        if (prune) {
          if (bm) mfirst = min(mfirst, c0 + wfa_low_bit(bm)), mlast = c0 + wfa_high_bit(bm);
          if (bx && kdone == INT32_MAX) kdone = c0 + wfa_low_bit(bx);
        }
      }
    }
    if (fwd && !fin) {
      if (gl == 0) {
        const int2 wm = mfirst <= mlast ? wfa_pack(mfirst, mlast, mb + (uint32_t)(mfirst - mlo))
                                        : wfa_empty();
        const int2 wi = ifirst <= ilast ? wfa_pack(ifirst, ilast, ib + (uint32_t)(ifirst - ilo))
                                        : wfa_empty();
        const int2 wd = dfirst <= dlast ? wfa_pack(dfirst, dlast, db + (uint32_t)(dfirst - dlo))
                                        : wfa_empty();
        const uint32_t rs = ((uint32_t)s % R) * 3u;
        ring[rs + 0] = wm;
        ring[rs + 1] = wi;
        ring[rs + 2] = wd;
        if (TB) {
          meta[(uint32_t)s * 3u + 0] = wm;
          meta[(uint32_t)s * 3u + 1] = wi;
          meta[(uint32_t)s * 3u + 2] = wd;
        }
      }
      if (kdone != INT32_MAX) {
        fin = 1;
      } else if (s >= S_loop) {
        fin = 2;
      } else {
        // Nothing reached within the look-back window: no later score reaches anything.
        if (mfirst <= mlast || ifirst <= ilast || dfirst <= dlast) last_live = s;
        if (s - last_live > L.lookback) fin = 2;
        else ++s;
      }
    }
    __syncwarp();

    // ---- finish
    if (fwd && fin) {
      if (gl == 0) {
        kira_wfa_result res{};
        res.cost = -1;
        uint32_t nops = 0;
        if (fin == 3) {
          atomicOr(L.flags, 2u);
        } else if (fin == 1) {
          res.found = 1;
          res.cost = s;
          res.score = L.scored ? m * L.match - s : s;
          res.text_end = (uint32_t)(m + kdone);
          if (TB) {
            bool ovf = false;
            uint32_t* slot = L.slots + (size_t)p * L.slot_cap;
            const int k0 = wfa_traceback(L, meta, H, pw, tw, m, n, s, kdone, slot, nops, ovf);
            res.text_start = (uint32_t)max(k0, 0);
            if (ovf) atomicOr(L.flags, 1u);
          }
        }
        if (TB) L.ncig[p] = nops;
        L.out[p] = res;
      }
      phase = 0;
    }
    __syncwarp();
  }
}

// Fixed-window WFA: one warp per pair, lane l owns diagonals win_base + 32 j + l
// (j < NH) for the whole search. Every cell the recurrence can reach by score
// win_smax lies in the window (an inserted base moves one diagonal down for at
// least ei, a deleted base one up for at least ed, the seeds sit on
// 0..text_begin_free), so up to that score the window is the whole wavefront and
// no range is tracked; a 32-diagonal segment that no reached diagonal can touch
// this score (new cells lie within one diagonal of the reached range) stays
// "none" without being computed. The last lookback + 1 scores live in a shared
// ring of int16 rows with a guard column on each side (the k - 1 / k + 1
// neighbours of the edge diagonals read "none"); "none" is any negative value, so
// the reference's checks become plain max / select: an unreached source stays
// negative through the +1s of a search. A pair not done by win_smax (and not
// exhausted) goes to fb_list for the general kernel, which redoes it from scratch.
template <int NH, bool TB>
__global__ void __launch_bounds__(128) wfa_window_kernel(DevPairs P, WfaLaunch L) {
  constexpr int kW = 32 * NH;  // diagonals of the window
  constexpr int kRow = kW + 2; // + 2 guards
  constexpr int kNone16 = -32000;
  extern __shared__ __align__(16) uint8_t wfa_smem[];
  const int lane = threadIdx.x & 31;
  const uint32_t wib = threadIdx.x >> 5;
  const uint32_t stage = L.smem_group - L.ring_bytes;  // pattern + text bytes per warp
  uint8_t* my = wfa_smem + (size_t)wib * (L.win_ring_bytes + stage);
  int16_t* ring = (int16_t*)my;
  uint32_t* pw = (uint32_t*)(my + L.win_ring_bytes + 16);
  uint32_t* tw = (uint32_t*)(my + L.win_ring_bytes + L.pat_region + 16);
  uint8_t* pb = (uint8_t*)pw;
  uint8_t* tb = (uint8_t*)tw;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + wib;
  int16_t* hist = TB ? L.win_hist + (size_t)warp * (L.win_smax + 1) * 3 * kW : nullptr;
  const int R = (int)L.ring_len;
  const int x = L.x, oi = L.o + L.ei, od = L.o + L.ed, ei = L.ei, ed = L.ed;
  const int xr = x % R, oir = oi % R, odr = od % R, eir = ei % R, edr = ed % R;
  const int base = L.win_base;
  for (int r = lane; r < R * 3; r += 32) {  // guard columns stay "none"
    ring[r * kRow] = (int16_t)kNone16;
    ring[r * kRow + kRow - 1] = (int16_t)kNone16;
  }
  for (;;) {
    uint32_t p = 0;
    if (lane == 0) p = atomicAdd(L.work, 1u);
    p = __shfl_sync(kFull, p, 0);
    if (p >= L.n) break;
    const int m = (int)P.read_len[p], n = (int)P.win_len[p];
    if (!L.valid || m == 0) {  // WfaCosts::scored refused: None; empty read: wfa.rs:555-563
      if (lane == 0) {
        kira_wfa_result res{};
        res.cost = L.valid ? 0 : -1;
        res.found = L.valid ? 1u : 0u;
        L.out[p] = res;
        if (TB) L.ncig[p] = 0;
      }
      continue;
    }
    const uint8_t* rs = P.read_seq + P.read_off[p];
    const uint8_t* ws = P.win_seq + P.win_off[p];
    __syncwarp();
    for (int i = lane; i < m; i += 32) pb[i] = __ldg(rs + i);
    for (int i = lane; i < n; i += 32) tb[i] = __ldg(ws + i);
    int S = L.max_score_pp ? L.max_score_pp[p] : L.max_score;
    if (!L.max_score_pp && S < 0) S = wfa_budget(m, L);
    const int64_t cap = L.drop < 0 ? (int64_t)L.o + (int64_t)L.ei * m
                                   : (int64_t)max(x, oi) * (2 * m + n + 2);
    const int S_loop = (int)max((int64_t)0, min((int64_t)S, cap));
    const int s_lim = min(S_loop, L.win_smax);
    int tbf = L.tbf_pp ? L.tbf_pp[p] : L.tbf;
    tbf = min(max(tbf, 0), max(n - 1, 0));
    __syncwarp();
    int done_s = -1, k_end = 0, last_live = 0, slot = 0;
    int lo_seen = 0, hi_seen = tbf;  // reached diagonals so far (the seeds: 0 .. tbf)
    bool dead = false;
    for (int s = 0; s <= s_lim; ++s) {
      bool need[NH];
#pragma unroll
      for (int h = 0; h < NH; ++h)
        need[h] = lo_seen - 1 <= base + 32 * h + 31 && hi_seen + 1 >= base + 32 * h;
      auto row = [&](int back, int backr, int layer) -> const int16_t* {
        int sl = slot - backr;
        if (sl < 0) sl += R;
        return (s - back >= 0) ? ring + (sl * 3 + layer) * kRow : nullptr;
      };
      const int16_t* rMx = row(x, xr, 0);
      const int16_t* rMoi = row(oi, oir, 0);
      const int16_t* rMod = row(od, odr, 0);
      const int16_t* rIe = row(ei, eir, 1);
      const int16_t* rDe = row(ed, edr, 2);
      int16_t* wM = ring + (slot * 3 + 0) * kRow;
      int16_t* wI = ring + (slot * 3 + 1) * kRow;
      int16_t* wD = ring + (slot * 3 + 2) * kRow;
      int vm2[NH], vi2[NH], vd2[NH];
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const int col = 1 + h * 32 + lane;
        const int k = base + h * 32 + lane;
        int vi = kNone16, vd = kNone16, vm = kNone16;
        if (!need[h]) {
          // this segment stays "none"
        } else if (s == 0) {
          vm = (k >= 0 && k <= tbf) ? 0 : kNone16;
        } else {
          if (rMoi) {
            const int a = rMoi[col + 1];
            vi = a < m ? a + 1 : kNone16;
          }
          if (rIe) {
            const int b = rIe[col + 1];
            vi = max(vi, b < m ? b + 1 : kNone16);
          }
          if (rMod) {
            const int a = rMod[col - 1];
            vd = a + k <= n ? a : kNone16;
          }
          if (rDe) {
            const int b = rDe[col - 1];
            vd = max(vd, b + k <= n ? b : kNone16);
          }
          if (rMx) {
            const int a = rMx[col];
            vm = (a < m && a + k < n) ? a + 1 : kNone16;
          }
          vm = max(vm, max(vi, vd));
        }
        if (vm >= 0) vm = wfa_extend(pw, tw, m, n, k, vm);
        vm2[h] = vm, vi2[h] = vi, vd2[h] = vd;
      }
#pragma unroll
      for (int h = 0; h < NH; ++h) {  // extend the reached range by this score's cells
        const unsigned q = __ballot_sync(kFull, vm2[h] >= 0 || vi2[h] >= 0 || vd2[h] >= 0);
        if (q) {
          lo_seen = min(lo_seen, base + 32 * h + wfa_low_bit(q));
          hi_seen = max(hi_seen, base + 32 * h + wfa_high_bit(q));
        }
      }
      if (L.drop >= 0) {  // prune_wavefront (wfa.rs:293-346) on the extended M
        int mad = INT32_MIN;
#pragma unroll
        for (int h = 0; h < NH; ++h)
          if (vm2[h] >= 0) mad = max(mad, 2 * vm2[h] + base + h * 32 + lane);
        mad = __reduce_max_sync(kFull, mad);
        if (mad != INT32_MIN) {
          const int th = mad - L.drop;
#pragma unroll
          for (int h = 0; h < NH; ++h)
            if (vm2[h] >= 0 && 2 * vm2[h] + base + h * 32 + lane < th) vm2[h] = kNone16;
        }
      }
      int kd = INT32_MAX;  // lowest done diagonal
      bool live = false;
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const int col = 1 + h * 32 + lane;
        wM[col] = (int16_t)vm2[h];
        wI[col] = (int16_t)vi2[h];
        wD[col] = (int16_t)vd2[h];
        if (TB) {
          int16_t* hs = hist + (size_t)s * 3 * kW + h * 32 + lane;
          hs[0] = (int16_t)vm2[h];
          hs[kW] = (int16_t)vi2[h];
          hs[2 * kW] = (int16_t)vd2[h];
        }
        const unsigned bd = __ballot_sync(kFull, vm2[h] >= m);
        if (bd && kd == INT32_MAX) kd = base + 32 * h + wfa_low_bit(bd);
        live |= (vm2[h] & vi2[h] & vd2[h]) >= 0;  // some value >= 0 unless all negative
      }
      live = __any_sync(kFull, live);
      __syncwarp();
      if (kd != INT32_MAX) {
        done_s = s;
        k_end = kd;
        break;
      }
      // Nothing reached within the look-back window: no later score reaches anything.
      if (live) last_live = s;
      else if (s - last_live > L.lookback) {
        dead = true;
        break;
      }
      if (++slot == R) slot = 0;
    }
    if (lane == 0) {
      if (done_s < 0 && !dead && S_loop > s_lim) {
        L.fb_list[atomicAdd(L.fb_count, 1u)] = p;  // the general kernel redoes it
      } else {
        kira_wfa_result res{};
        res.cost = -1;
        uint32_t nops = 0;
        if (done_s >= 0) {
          res.found = 1;
          res.cost = done_s;
          res.score = L.scored ? m * L.match - done_s : done_s;
          res.text_end = (uint32_t)(m + k_end);
          if (TB) {
            auto get = [&](int layer, int sc, int kk) -> int {
              if (sc < 0 || kk < base || kk > base + kW - 1) return kWfaNone;
              const int v = hist[(size_t)sc * 3 * kW + layer * kW + (kk - base)];
              return v >= 0 ? v : kWfaNone;
            };
            bool ovf = false;
            uint32_t* sl = L.slots + (size_t)p * L.slot_cap;
            const int k0 = wfa_traceback_t(L, get, pw, tw, m, n, done_s, k_end, sl, nops, ovf);
            res.text_start = (uint32_t)max(k0, 0);
            if (ovf) atomicOr(L.flags, 1u);
          }
        }
        if (TB) L.ncig[p] = nops;
        L.out[p] = res;
      }
    }
    __syncwarp();
  }
}

// cigar_off / n_cigar of every result and the ops in pair order (each pair's
// slot holds its ops in reverse).
__global__ void __launch_bounds__(256) wfa_compact_kernel(WfaCompact C) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < C.n; p += stride) {
    const uint32_t off = C.off[p], n = C.ncig[p];
    C.out[p].cigar_off = off;
    C.out[p].n_cigar = n;
    if ((uint64_t)off + n > C.cap || n > C.slot_cap) continue;
    const uint32_t* src = C.slots + (size_t)p * C.slot_cap;
    for (uint32_t t = 0; t < n; ++t) C.ops[off + t] = src[n - 1u - t];
  }
}

}  // namespace

template <int G>
static cudaError_t wfa_occupancy(bool traceback, size_t smem, int threads, int* per_sm) {
  auto kern = traceback ? wfa_kernel<G, true> : wfa_kernel<G, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, threads, smem);
}

cudaError_t wfa_blocks_per_sm(int group, bool traceback, size_t smem, int threads, int* per_sm) {
  switch (group) {
    case 8: return wfa_occupancy<8>(traceback, smem, threads, per_sm);
    case 16: return wfa_occupancy<16>(traceback, smem, threads, per_sm);
    case 32: return wfa_occupancy<32>(traceback, smem, threads, per_sm);
    default: return cudaErrorInvalidValue;
  }
}

template <int G>
static void wfa_launch_g(const DevPairs& P, const WfaLaunch& L, uint32_t blocks, uint32_t threads,
                         size_t smem, bool traceback, cudaStream_t st) {
  if (traceback) (wfa_kernel<G, true><<<blocks, threads, smem, st>>>(P, L), count_launch());
  else (wfa_kernel<G, false><<<blocks, threads, smem, st>>>(P, L), count_launch());
}

cudaError_t launch_wfa(const DevPairs& P, const WfaLaunch& L, uint32_t blocks,
                       uint32_t warps_per_block, bool traceback, cudaStream_t st) {
  const uint32_t groups = warps_per_block * (32u / (uint32_t)L.group);
  const size_t smem = (size_t)L.smem_group * groups;
  const uint32_t threads = 32u * warps_per_block;
  switch (L.group) {
    case 8: wfa_launch_g<8>(P, L, blocks, threads, smem, traceback, st); break;
    case 16: wfa_launch_g<16>(P, L, blocks, threads, smem, traceback, st); break;
    case 32: wfa_launch_g<32>(P, L, blocks, threads, smem, traceback, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t wfa_window_blocks_per_sm(int segments, bool traceback, size_t smem, int* per_sm) {
  auto kern = segments == 4 ? (traceback ? wfa_window_kernel<4, true> : wfa_window_kernel<4, false>)
                            : (traceback ? wfa_window_kernel<2, true> : wfa_window_kernel<2, false>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, 128, smem);
}

cudaError_t launch_wfa_window(const DevPairs& P, const WfaLaunch& L, uint32_t blocks,
                              bool traceback, cudaStream_t st) {
  const size_t smem = (size_t)4 * (L.win_ring_bytes + L.smem_group - L.ring_bytes);
  if (L.win_segments == 4) {
    if (traceback) (wfa_window_kernel<4, true><<<blocks, 128, smem, st>>>(P, L), count_launch());
    else (wfa_window_kernel<4, false><<<blocks, 128, smem, st>>>(P, L), count_launch());
  } else {
    if (traceback) (wfa_window_kernel<2, true><<<blocks, 128, smem, st>>>(P, L), count_launch());
    else (wfa_window_kernel<2, false><<<blocks, 128, smem, st>>>(P, L), count_launch());
  }
  return cudaGetLastError();
}

cudaError_t launch_wfa_compact(const WfaCompact& C, int sms, cudaStream_t st) {
  uint64_t b = (C.n + 255) / 256;
  if (b < 1) b = 1;
  if (b > (uint64_t)sms * 8) b = (uint64_t)sms * 8;
  (wfa_compact_kernel<<<(int)b, 256, 0, st>>>(C), count_launch());
  return cudaGetLastError();
}

}  // namespace kira
