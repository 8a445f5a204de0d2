// wfa.cuh -- wavefront alignment (src/alignment/wfa.rs), one (read, window) pair
// per warp.
//
// The recurrence is the reference's: per score s three wavefronts M, I, D hold
// the furthest pattern offset reached on each diagonal k = j - i,
//   I[s][k] = max(M[s-o-ei][k+1] + 1, I[s-ei][k+1] + 1)   (source offset < m)
//   D[s][k] = max(M[s-o-ed][k-1],     D[s-ed][k-1])       (offset + k <= n)
//   M[s][k] = max(M[s-x][k] + 1 (offset < m, offset + k < n), I[s][k], D[s][k])
// followed by greedy extension along matches, optional adaptive pruning, and the
// done test (the lowest diagonal whose offset reached m). step (wfa.rs:374-526),
// extend_wavefront (:277-291), prune_wavefront (:293-346), check_done (:348-358),
// build_cigar (:762-952).
//
// B200 mapping: the 32 lanes of a warp own 32 consecutive diagonals of a score
// step (chunks of 32 for wider fronts), so the sources of a chunk are 64-byte
// coalesced int16 loads and the extension of each diagonal runs in its own lane
// over the pair's bytes staged in shared memory (8 bytes per compare). Offsets
// live in a per-warp history in device memory (int16, INT16_MIN = none): every
// score when a traceback follows, a ring of lookback + 1 scores otherwise (the
// layer retirement of wfa_score_only, wfa.rs:672-745). Each stored wavefront is
// trimmed to its first and last reached diagonal; the trimmed-away diagonals
// read as "none" exactly like diagonals outside the reference's range, so no
// offset changes. The traceback walks back in lane 0 with the reference's edge
// order, comparing matches 4 bytes at a time.
#pragma once

#include "common.cuh"

namespace kira {

constexpr int32_t kWfaNone = INT32_MIN / 4;  // NONE_OFFSET (wfa.rs:6)

struct WfaWave {
  int lo, hi;     // diagonal range; empty when hi < lo
  uint32_t base;  // history index of diagonal lo
};

__device__ __forceinline__ int2 wfa_pack(int lo, int hi, uint32_t base) {
  return make_int2((int)(((uint32_t)lo & 0xFFFFu) | ((uint32_t)hi << 16)), (int)base);
}

__device__ __forceinline__ WfaWave wfa_unpack(int2 v) {
  return WfaWave{(int)(int16_t)(v.x & 0xFFFF), v.x >> 16, (uint32_t)v.y};
}

__device__ __forceinline__ int2 wfa_empty() { return wfa_pack(1, 0, 0); }

__device__ __forceinline__ int16_t wfa_enc(int v) {
  return v == kWfaNone ? (int16_t)INT16_MIN : (int16_t)v;
}

__device__ __forceinline__ int wfa_dec(int16_t v) { return v == INT16_MIN ? kWfaNone : (int)v; }

// WaveFront::get (wfa.rs:143-151) on a stored wavefront.
__device__ __forceinline__ int wfa_get(const int16_t* __restrict__ H, const WfaWave& w, int k) {
  return (k < w.lo || k > w.hi) ? kWfaNone : wfa_dec(H[w.base + (uint32_t)(k - w.lo)]);
}

// Four bytes starting at byte p (any alignment, p >= -4) of a shared-memory word array.
__device__ __forceinline__ uint32_t wfa_ld4(const uint32_t* w, int p) {
  const int q = p >> 2;
  return __byte_perm(w[q], w[q + 1], 0x3210u + 0x1111u * (uint32_t)(p & 3));
}

// extend_diagonal (wfa.rs:205-275): offset after the run of equal bytes from
// (i, j) = (v, v + k), stopping at the end of either sequence.
__device__ __forceinline__ int wfa_extend(const uint32_t* pw, const uint32_t* tw, int m, int n,
                                          int k, int v) {
  const int j = v + k;
  if (j < 0) return v;
  const int lim = min(m - v, n - j);
  int run = 0;
  while (run < lim) {
    const uint32_t d0 = wfa_ld4(pw, v + run) ^ wfa_ld4(tw, j + run);
    const uint32_t d1 = wfa_ld4(pw, v + run + 4) ^ wfa_ld4(tw, j + run + 4);
    if (d0) {
      run += (__ffs(d0) - 1) >> 3;
      break;
    }
    if (d1) {
      run += 4 + ((__ffs(d1) - 1) >> 3);
      break;
    }
    run += 8;
  }
  return v + max(0, min(run, lim));
}

// Backward match walk of the traceback (wfa.rs:807-853): from offset `off` on
// diagonal k, the number of consecutive equal bytes pattern[w-1] == text[w-1+k]
// for w = off, off-1, ..., never passing below `low`.
__device__ __forceinline__ int wfa_back_run(const uint32_t* pw, const uint32_t* tw, int k, int off,
                                            int low) {
  const int lim = off - low;
  int run = 0;
  while (run < lim) {
    const int p = off - run - 4;
    const uint32_t d = wfa_ld4(pw, p) ^ wfa_ld4(tw, p + k);
    if (d) {
      run += __clz(d) >> 3;
      break;
    }
    run += 4;
  }
  return max(0, min(run, lim));
}

}  // namespace kira
