// qgram.cuh -- exact 4-gram prefilter in front of the Myers stage.
//
// The Myers stage (bounded_edit_distance, src/alignment/myers.rs:47-70) answers
// None unless the read aligns to some substring T' of the window with at most k
// edits. Each edit (substitution, deletion from the read, or insertion between
// two read bases) touches at most four of the read's m - 3 overlapping 4-grams;
// every untouched read 4-gram occurs verbatim in T', hence in the window. So
//
//     ed <= k  implies  #{p : read[p, p+4) occurs in the window} >= m - 3 - 4k.
//
// A pair whose count is below that bound is a Myers None for certain, and the
// filter answers exactly that (the same MYERS_REJECT result and detail). Bases
// outside ACGT match nothing in Myers: a read 4-gram containing one can never
// be untouched and is not counted, and window 4-grams containing one are not
// inserted. The filter only ever removes pairs Myers would reject, so every
// output is unchanged; survivors still run Myers.
//
// Lane-per-pair: the window's 4-gram set is a 256-bit bitmap per lane in shared
// memory, 16 words of 16 used bits laid out [word][lane] (each lane owns one
// bank); bases come from the 2-bit + valid plane arenas, one 32-base word at a
// time. A 4-gram is its four bit-1 plane bits (the word) and its four bit-0 plane
// bits (the bit in it), each one bit-field extract, the previous word supplying
// the first three bases of a word; the positions whose four bases are all valid
// come from one AND of shifted valid masks per word. An insert is one shared-memory
// atomic OR (each lane owns its column, so nothing contends). Window and read use
// the same index, so the count is the count.
#pragma once

#include "common.cuh"
#include "planes.cuh"

namespace kira {

// Bits [b - 3, b] of the base stream ... prev | cur (b in 0..31, compile-time).
template <int B>
__device__ __forceinline__ uint32_t qgram_nibble(uint32_t prev, uint32_t cur) {
  if constexpr (B >= 3) return (cur >> (B - 3)) & 0xFu;
  else return __funnelshift_r(prev, cur, 29 + B) & 0xFu;
}

// Positions of a word whose 4-gram (this base and the three before) is all ACGT.
__device__ __forceinline__ uint32_t qgram_valid4(uint32_t pv, uint32_t v, uint32_t lim) {
  uint32_t v4 = v & __funnelshift_l(pv, v, 1) & __funnelshift_l(pv, v, 2) &
                __funnelshift_l(pv, v, 3);
  return lim < 32u ? v4 & ((1u << lim) - 1u) : v4;
}


// Where the count of read 4-grams found in the window falls against two bounds
// lo <= hi: 0 when count >= hi, 1 when lo <= count < hi, 2 when count < lo; the
// read walk stops as soon as that is decided. With hi <= 0 or a window of fewer
// than four bases the answer is 0 (nothing is proved). `set` points at this
// lane's column of a [16][32] word bitmap in shared memory.
__device__ __forceinline__ uint32_t qgram4_outcome(const uint4* __restrict__ rplanes,
                                                   uint64_t rpos, uint32_t m,
                                                   const uint4* __restrict__ wplanes,
                                                   uint64_t wpos, uint32_t n, int32_t lo,
                                                   int32_t hi, uint32_t* set) {
  if (hi <= 0 || n < 4u) return 0u;
#pragma unroll
  for (int w = 0; w < 16; ++w) set[w * 32] = 0u;
  uint32_t p0 = 0, p1 = 0, pv = 0;
  for (uint32_t blk = 0; blk * 32u < n; ++blk) {
    const PlaneWord pw = plane_word_at(wplanes, wpos + 32u * blk);
    const uint32_t v4 = qgram_valid4(pv, pw.v, min(32u, n - 32u * blk));
#define KIRA_QG_INS(B) \
  atomicOr(&set[qgram_nibble<(B)>(p1, pw.b1) * 32u], 1u << qgram_nibble<(B)>(p0, pw.b0));
#define KIRA_QG_SET(B) \
  if ((v4 >> (B)) & 1u) KIRA_QG_INS(B)
#define KIRA_QG_ALL(M)                                                                   \
  M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) \
  M(16) M(17) M(18) M(19) M(20) M(21) M(22) M(23) M(24) M(25) M(26) M(27) M(28) M(29)   \
  M(30) M(31)
    // A word whose 32 positions are all valid (no N near it) skips the per-position tests.
    if (v4 == 0xFFFFFFFFu) {
      KIRA_QG_ALL(KIRA_QG_INS)
    } else {
      KIRA_QG_ALL(KIRA_QG_SET)
    }
#undef KIRA_QG_SET
#undef KIRA_QG_INS
    p0 = pw.b0, p1 = pw.b1, pv = pw.v;
  }
  int32_t count = 0;
  p0 = p1 = pv = 0;
  for (uint32_t blk = 0; blk * 32u < m; ++blk) {
    const PlaneWord pw = plane_word_at(rplanes, rpos + 32u * blk);
    const uint32_t lim = min(32u, m - 32u * blk);
    const uint32_t v4 = qgram_valid4(pv, pw.v, lim);
#define KIRA_QG_HIT(B) \
  count += (int32_t)((set[qgram_nibble<(B)>(p1, pw.b1) * 32u] >> qgram_nibble<(B)>(p0, pw.b0)) & 1u);
#define KIRA_QG_COUNT(B) \
  if ((v4 >> (B)) & 1u) KIRA_QG_HIT(B)
    if (v4 == 0xFFFFFFFFu) {
      KIRA_QG_ALL(KIRA_QG_HIT)
    } else {
      KIRA_QG_ALL(KIRA_QG_COUNT)
    }
#undef KIRA_QG_COUNT
#undef KIRA_QG_HIT
    p0 = pw.b0, p1 = pw.b1, pv = pw.v;
    // Decided once the count reaches a bound or can no longer reach it.
    const int32_t left = (int32_t)m - (int32_t)(32u * blk + lim);
    if (count >= hi) return 0u;
    if (count + left < lo) return 2u;
    if (count >= lo && count + left < hi) return 1u;
  }
  return count < lo ? 2u : count < hi ? 1u : 0u;
}
#undef KIRA_QG_ALL

// True when the read provably has edit distance > k to every window substring.
__device__ __forceinline__ bool qgram4_reject(const uint4* __restrict__ rplanes, uint64_t rpos,
                                              uint32_t m, const uint4* __restrict__ wplanes,
                                              uint64_t wpos, uint32_t n, uint32_t k,
                                              uint32_t* set) {
  const int32_t need = (int32_t)m - 3 - 4 * (int32_t)k;
  return qgram4_outcome(rplanes, rpos, m, wplanes, wpos, n, need, need, set) != 0u;
}

}  // namespace kira
