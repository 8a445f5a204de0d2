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
// memory laid out [word][lane] (each lane owns one bank); bases come from the
// 2-bit + valid plane arenas, one 32-base word at a time.
#pragma once

#include "common.cuh"
#include "planes.cuh"

namespace kira {

// True when the read provably has edit distance > k to every window substring.
// `set` points at this lane's column of an [8][32] word bitmap in shared memory.
__device__ __forceinline__ bool qgram4_reject(const uint4* __restrict__ rplanes, uint64_t rpos,
                                              uint32_t m, const uint4* __restrict__ wplanes,
                                              uint64_t wpos, uint32_t n, uint32_t k,
                                              uint32_t* set) {
  const int32_t need = (int32_t)m - 3 - 4 * (int32_t)k;
  if (need <= 0 || n < 4u) return false;
#pragma unroll
  for (int w = 0; w < 8; ++w) set[w * 32] = 0u;
  uint32_t code = 0, vrun = 0;
  for (uint32_t blk = 0; blk * 32u < n; ++blk) {
    const PlaneWord pw = plane_word_at(wplanes, wpos + 32u * blk);
    const uint32_t lim = min(32u, n - 32u * blk);
#pragma unroll
    for (uint32_t b = 0; b < 32u; ++b) {
      if (b < lim) {
        code = ((code << 2) | (((pw.b1 >> b) & 1u) << 1) | ((pw.b0 >> b) & 1u)) & 0xFFu;
        vrun = ((pw.v >> b) & 1u) ? vrun + 1u : 0u;
        if (vrun >= 4u) set[(code >> 5) * 32u] |= 1u << (code & 31u);
      }
    }
  }
  int32_t count = 0;
  code = 0;
  vrun = 0;
  for (uint32_t blk = 0; blk * 32u < m; ++blk) {
    const PlaneWord pw = plane_word_at(rplanes, rpos + 32u * blk);
    const uint32_t lim = min(32u, m - 32u * blk);
#pragma unroll
    for (uint32_t b = 0; b < 32u; ++b) {
      if (b < lim) {
        code = ((code << 2) | (((pw.b1 >> b) & 1u) << 1) | ((pw.b0 >> b) & 1u)) & 0xFFu;
        vrun = ((pw.v >> b) & 1u) ? vrun + 1u : 0u;
        if (vrun >= 4u) count += (int32_t)((set[(code >> 5) * 32u] >> (code & 31u)) & 1u);
      }
    }
    // Decided either way once the count reaches the bound or can no longer.
    const int32_t left = (int32_t)m - (int32_t)(32u * blk + lim);
    if (count >= need) return false;
    if (count + left < need) return true;
  }
  return count < need;
}

}  // namespace kira
