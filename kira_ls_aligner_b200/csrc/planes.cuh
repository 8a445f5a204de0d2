// planes.cuh -- 2-bit + valid bit planes of ASCII sequence arenas.
//
// Block b of a plane arena covers bases 32b .. 32b+31 of the byte arena it was
// built from: {x: code bit 0, y: code bit 1, z: ACGT-valid, w: 0}, one bit per
// base (bit i = base 32b + i). Codes and validity are encode_base / is_acgt of
// src/alignment/bitpacked.rs:12-20,89-91 (A0 C1 G2 T3, lower case folded, every
// other byte code 0 and invalid). Sieve and Myers need nothing else from a base,
// so both read their sequences as plane words: 32 consecutive bases starting at
// any position are two 16-byte loads and one funnel shift per plane.
#pragma once

#include "common.cuh"

namespace kira {

struct PlaneWord {
  uint32_t b0, b1, v;
};

// 32 bases starting at base position `pos` of the arena (bits beyond the arena's
// end are whatever padding the planes hold; callers mask by length).
__device__ __forceinline__ PlaneWord plane_word_at(const uint4* __restrict__ planes, uint64_t pos) {
  const uint64_t blk = pos >> 5;
  const uint32_t off = (uint32_t)pos & 31u;
  const uint4 a = __ldg(planes + blk);
  const uint4 b = __ldg(planes + blk + 1);
  PlaneWord w;
  w.b0 = __funnelshift_r(a.x, b.x, off);
  w.b1 = __funnelshift_r(a.y, b.y, off);
  w.v = __funnelshift_r(a.z, b.z, off);
  return w;
}

__device__ __forceinline__ uint32_t low_mask(uint32_t nbits) {
  return nbits >= 32u ? 0xFFFFFFFFu : ((1u << nbits) - 1u);
}

}  // namespace kira

namespace kira {

// ---------------------------------------------------------------------------
// Lane-per-pair sieve on plane words (scan_best_with_second_raw semantics,
// src/alignment/bitpacked.rs:154-199; checked mode: a non-ACGT base in the read
// or the window gives None, as packed_scan_scratch, src/alignment/mod.rs:594-621).
// Per shift and 32 read bases: 2 funnel shifts, XOR, LOP3, POPC, add.
// ---------------------------------------------------------------------------
struct LaneSieve {
  bool hit;
  uint32_t shift, mism, second;  // second = 0xFFFFFFFF when absent
};

template <int RW>
__device__ __forceinline__ LaneSieve sieve_lane_rw(const uint4* __restrict__ rp, uint64_t rpos,
                                                   uint32_t q, const uint4* __restrict__ wp,
                                                   uint64_t wpos, uint32_t w) {
  LaneSieve o{false, 0, 0, 0xFFFFFFFFu};
  uint32_t r0[RW], r1[RW];
  uint32_t bad = 0;
  const uint32_t tail_mask = low_mask(q - 32u * (RW - 1));
#pragma unroll
  for (int k = 0; k < RW; ++k) {
    const PlaneWord pw = plane_word_at(rp, rpos + 32u * k);
    const uint32_t m = k == RW - 1 ? tail_mask : 0xFFFFFFFFu;
    r0[k] = pw.b0 & m;
    r1[k] = pw.b1 & m;
    bad |= ~pw.v & m;
  }
  uint32_t w0[RW + 1], w1[RW + 1];
#pragma unroll
  for (int k = 0; k <= RW; ++k) {
    const PlaneWord pw = plane_word_at(wp, wpos + 32u * k);
    w0[k] = pw.b0;
    w1[k] = pw.b1;
    const uint32_t base = 32u * k;
    if (base < w) bad |= ~pw.v & low_mask(w - base);
  }
  const uint32_t n_shifts = w - q + 1u;
  uint32_t best = 0xFFFFFFFFu, second = 0xFFFFFFFFu;
  uint32_t t = 0;
  for (uint32_t blk = 0;; ++blk) {
    const uint32_t tend = min(n_shifts, t + 32u);
    for (; t < tend; ++t) {
      const uint32_t sh = t & 31u;
      uint32_t mism = 0;
#pragma unroll
      for (int k = 0; k < RW; ++k) {
        const uint32_t a0 = __funnelshift_r(w0[k], w0[k + 1], sh);
        const uint32_t a1 = __funnelshift_r(w1[k], w1[k + 1], sh);
        uint32_t x = (r0[k] ^ a0) | (r1[k] ^ a1);
        if (k == RW - 1) x &= tail_mask;
        mism += __popc(x);
      }
      const uint32_t key = (mism << 20) | t;
      if (key < best) {
        second = best;
        best = key;
      } else if (key < second) {
        second = key;
      }
    }
    if (t >= n_shifts) break;
    // slide one word: window words blk+1 .. blk+1+RW
#pragma unroll
    for (int k = 0; k < RW; ++k) {
      w0[k] = w0[k + 1];
      w1[k] = w1[k + 1];
    }
    const uint32_t base = 32u * (blk + 1u + RW);
    const PlaneWord pw = plane_word_at(wp, wpos + base);
    w0[RW] = pw.b0;
    w1[RW] = pw.b1;
    if (base < w) bad |= ~pw.v & low_mask(w - base);
  }
  if (bad) return o;
  o.hit = true;
  o.shift = best & 0xFFFFFu;
  o.mism = best >> 20;
  o.second = second == 0xFFFFFFFFu ? 0xFFFFFFFFu : (second >> 20);
  return o;
}

template <int RWMAX>
__device__ __forceinline__ LaneSieve sieve_lane(const uint4* rp, uint64_t rpos, uint32_t q,
                                                const uint4* wp, uint64_t wpos, uint32_t w) {
  LaneSieve none{false, 0, 0, 0xFFFFFFFFu};
  if (q == 0 || w < q) return none;
  switch ((q + 31u) / 32u) {
#define KIRA_LSIEVE_CASE(n) \
  case n:                   \
    if (n <= RWMAX) return sieve_lane_rw<(n <= RWMAX ? n : 1)>(rp, rpos, q, wp, wpos, w); \
    break;
    KIRA_LSIEVE_CASE(1) KIRA_LSIEVE_CASE(2) KIRA_LSIEVE_CASE(3) KIRA_LSIEVE_CASE(4)
    KIRA_LSIEVE_CASE(5) KIRA_LSIEVE_CASE(6) KIRA_LSIEVE_CASE(7) KIRA_LSIEVE_CASE(8)
    KIRA_LSIEVE_CASE(9) KIRA_LSIEVE_CASE(10) KIRA_LSIEVE_CASE(11) KIRA_LSIEVE_CASE(12)
    KIRA_LSIEVE_CASE(13) KIRA_LSIEVE_CASE(14) KIRA_LSIEVE_CASE(15) KIRA_LSIEVE_CASE(16)
#undef KIRA_LSIEVE_CASE
    default:
      break;
  }
  return none;
}

}  // namespace kira
