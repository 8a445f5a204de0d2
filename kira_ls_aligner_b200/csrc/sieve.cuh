// sieve.cuh -- warp-cooperative 2-bit multi-shift Hamming sieve.
//
// Semantics: scan_best_with_second_raw (src/alignment/bitpacked.rs:154-199) and
// mismatch_count_u64 (:238-270): for every shift t in [0, w-q] the number of
// positions whose 2-bit codes differ; best = minimum count at the lowest shift,
// second = minimum count over every other shift (ties with best included).
//
// B200 mapping (one warp per pair):
//   * the read and the window are turned into two bit planes (low / high code
//     bit, one bit per base) by __ballot_sync over 32 positions at a time, so no
//     4x pre-shifted window copies exist anywhere (the reference ships four,
//     src/cuda/backend.rs:134-148);
//   * lane l evaluates shifts t = 32r + l; the window word at bit offset t is one
//     __funnelshift_r of two uniform plane words, so a shift costs per 32 bases
//     2 funnel shifts, 1 XOR, 1 LOP3, 1 POPC and 1 add;
//   * window plane words slide through registers (RW + 1 live words), one new
//     word per 32 shifts, so windows of any length need no shared memory;
//   * (mism << 20 | shift) keys are reduced with __shfl_xor_sync into the best
//     and second-best keys of the warp.
#pragma once

#include "common.cuh"

namespace kira {

constexpr uint32_t kNoKey = 0xFFFFFFFFu;

struct SieveOut {
  bool hit;          // false: q == 0, w < q or (checked inputs) a non-ACGT base
  uint32_t shift;
  uint32_t mism;
  uint32_t second;   // kNoKey when there is no other shift
};

// Builds one plane word pair (codes of positions 32*word .. +31) from `code(p)`.
// Returns the invalid-position mask for positions < limit.
template <class CodeFn>
__device__ __forceinline__ void plane_word(CodeFn code, uint32_t word, uint32_t limit,
                                           uint32_t lane, uint32_t& p0, uint32_t& p1,
                                           uint32_t& bad) {
  const uint32_t pos = word * 32u + lane;
  const bool in = pos < limit;
  const uint32_t c = in ? code(pos) : 4u;  // padding: code 0, valid
  p0 = __ballot_sync(0xFFFFFFFFu, c & 1u);
  p1 = __ballot_sync(0xFFFFFFFFu, c & 2u);
  bad = __ballot_sync(0xFFFFFFFFu, in && !(c & 4u));
}

// All 32 lanes must call this with identical q, w (warp-uniform control flow).
// RW = (q + 31) / 32 exactly: the word loops are fully unrolled with no guards.
template <int RW, class ReadCode, class WinCode>
__device__ __forceinline__ SieveOut sieve_warp_rw(uint32_t q, uint32_t w, ReadCode rcode,
                                                  WinCode wcode, bool check_valid) {
  constexpr int RWMAX = RW;
  SieveOut o{false, 0, 0, kNoKey};
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t rw = RW;
  uint32_t r0[RWMAX], r1[RWMAX];
  uint32_t w0[RWMAX + 1], w1[RWMAX + 1];
  uint32_t bad = 0;
  // Issue every byte load of the read and of the first window words before the
  // ballots, so the pair pays one memory latency instead of one per word.
  uint32_t rc[RWMAX], wc[RWMAX + 1];
#pragma unroll
  for (int k = 0; k < RWMAX; ++k) {
    const uint32_t pos = (uint32_t)k * 32u + lane;
    rc[k] = pos < q ? rcode(pos) : 4u;
  }
#pragma unroll
  for (int k = 0; k <= RWMAX; ++k) {
    const uint32_t pos = (uint32_t)k * 32u + lane;
    wc[k] = pos < w ? wcode(pos) : 4u;
  }
#pragma unroll
  for (int k = 0; k < RWMAX; ++k) {
    r0[k] = __ballot_sync(0xFFFFFFFFu, rc[k] & 1u);
    r1[k] = __ballot_sync(0xFFFFFFFFu, rc[k] & 2u);
    bad |= __ballot_sync(0xFFFFFFFFu, !(rc[k] & 4u));
  }
#pragma unroll
  for (int k = 0; k <= RWMAX; ++k) {
    w0[k] = __ballot_sync(0xFFFFFFFFu, wc[k] & 1u);
    w1[k] = __ballot_sync(0xFFFFFFFFu, wc[k] & 2u);
    bad |= __ballot_sync(0xFFFFFFFFu, !(wc[k] & 4u));
  }
  const uint32_t tail = q & 31u;
  const uint32_t tail_mask = tail ? ((1u << tail) - 1u) : 0xFFFFFFFFu;
  const uint32_t n_shifts = w - q + 1u;
  const uint32_t blocks = (n_shifts + 31u) / 32u;
  uint32_t best = kNoKey, second = kNoKey;
  // Code of the window word needed by the next slide, loaded one block ahead.
  uint32_t next_c = 4u;
  {
    const uint32_t pos = (1u + rw) * 32u + lane;
    if (blocks > 1u) next_c = pos < w ? wcode(pos) : 4u;
  }
  for (uint32_t r = 0; r < blocks; ++r) {
    const uint32_t t = r * 32u + lane;
    uint32_t mism = 0;
#pragma unroll
    for (int k = 0; k < RWMAX; ++k) {
      if ((uint32_t)k < rw) {
        const uint32_t a0 = __funnelshift_r(w0[k], w0[k + 1], lane);
        const uint32_t a1 = __funnelshift_r(w1[k], w1[k + 1], lane);
        uint32_t x = (r0[k] ^ a0) | (r1[k] ^ a1);
        if ((uint32_t)k == rw - 1u) x &= tail_mask;
        mism += __popc(x);
      }
    }
    if (t < n_shifts) {
      const uint32_t key = (mism << 20) | t;
      if (key < best) {
        second = best;
        best = key;
      } else if (key < second) {
        second = key;
      }
    }
    if (r + 1u < blocks) {  // slide: words r+1 .. r+1+rw
#pragma unroll
      for (int k = 0; k < RWMAX; ++k) {
        if ((uint32_t)k < rw) {
          w0[k] = w0[k + 1];
          w1[k] = w1[k + 1];
        }
      }
      const uint32_t n0 = __ballot_sync(0xFFFFFFFFu, next_c & 1u);
      const uint32_t n1 = __ballot_sync(0xFFFFFFFFu, next_c & 2u);
      bad |= __ballot_sync(0xFFFFFFFFu, !(next_c & 4u));
      if (r + 2u < blocks) {
        const uint32_t pos = (r + 2u + rw) * 32u + lane;
        next_c = pos < w ? wcode(pos) : 4u;
      }
#pragma unroll
      for (int k = 0; k <= RWMAX; ++k)
        if ((uint32_t)k == rw) {
          w0[k] = n0;
          w1[k] = n1;
        }
    }
  }
  // Warp reduction of (best, second) key pairs.
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const uint32_t ob = __shfl_xor_sync(0xFFFFFFFFu, best, off);
    const uint32_t os = __shfl_xor_sync(0xFFFFFFFFu, second, off);
    const uint32_t lo = min(best, ob), hi = max(best, ob);
    second = min(hi, min(second, os));
    best = lo;
  }
  // The scan also covered every window position, so `bad` holds both validity checks.
  if (check_valid && bad) return o;
  o.hit = best != kNoKey;
  o.shift = best & 0xFFFFFu;
  o.mism = best >> 20;
  o.second = second == kNoKey ? kNoKey : (second >> 20);
  return o;
}

// Dispatch on the read's word count; reads up to 32 * RWMAX bases.
template <int RWMAX, class ReadCode, class WinCode>
__device__ __forceinline__ SieveOut sieve_warp(uint32_t q, uint32_t w, ReadCode rcode,
                                               WinCode wcode, bool check_valid) {
  SieveOut none{false, 0, 0, kNoKey};
  if (q == 0 || w < q) return none;
  switch ((q + 31u) / 32u) {
#define KIRA_SIEVE_CASE(n) \
  case n:                  \
    if (n <= RWMAX) return sieve_warp_rw<(n <= RWMAX ? n : 1)>(q, w, rcode, wcode, check_valid); \
    break;
    KIRA_SIEVE_CASE(1) KIRA_SIEVE_CASE(2) KIRA_SIEVE_CASE(3) KIRA_SIEVE_CASE(4)
    KIRA_SIEVE_CASE(5) KIRA_SIEVE_CASE(6) KIRA_SIEVE_CASE(7) KIRA_SIEVE_CASE(8)
    KIRA_SIEVE_CASE(9) KIRA_SIEVE_CASE(10) KIRA_SIEVE_CASE(11) KIRA_SIEVE_CASE(12)
    KIRA_SIEVE_CASE(13) KIRA_SIEVE_CASE(14) KIRA_SIEVE_CASE(15) KIRA_SIEVE_CASE(16)
#undef KIRA_SIEVE_CASE
    default:
      break;
  }
  return none;
}

}  // namespace kira
