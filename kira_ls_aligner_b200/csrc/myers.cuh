// myers.cuh -- Myers (1999) bit-parallel bounded edit distance, one pair per lane.
//
// Semantics: bounded_edit_distance (src/alignment/myers.rs:47-70) with the
// fixed/heap recurrences of :101-204 / :206-324 (identical results): semi-global
// (free text ends, whole pattern), best = minimum column score with the LAST
// column on ties (`err <= best`), exact early reject when neither the running
// best nor the current column can reach k. Text bytes outside ACGT match
// nothing; pattern bytes outside ACGT set no Peq bit.
//
// B200 mapping: the bit vector is held as L 32-bit limbs in registers (the
// reference uses 64-bit blocks; bits below m never depend on bits above m, so
// the limb width does not change any result). A warp owns 32 pairs. Global
// loads stay coalesced: for each pair the whole warp loads 32 consecutive bytes
// and __ballot_sync turns them into the owning lane's Peq words (pattern) or
// into three text planes (code bit 0, code bit 1, ACGT-valid) kept in shared
// memory, so each lane's column loop reads one shared word per 32 columns.
#pragma once

#include "common.cuh"

namespace kira {

// Shared-memory text planes of one warp: [32 pairs][tw words][3].
struct MyersSmem {
  uint32_t* planes;
  uint32_t tw;  // words per pair (ceil(max window / 32))
};

template <int L>
struct MyersPeq {
  uint32_t a[L], c[L], g[L], t[L];
};

// Loads pair p's pattern into lane p's Peq (all lanes participate).
template <int L>
__device__ __forceinline__ void myers_load_pattern(const uint8_t* pat, uint32_t m, uint32_t p,
                                                   uint32_t lane, MyersPeq<L>& peq) {
#pragma unroll
  for (int k = 0; k < L; ++k) {
    const uint32_t pos = (uint32_t)k * 32u + lane;
    const uint32_t code = pos < m ? base_code(ldb(pat, pos)) : 0u;
    const uint32_t ba = __ballot_sync(0xFFFFFFFFu, code == 4u);
    const uint32_t bc = __ballot_sync(0xFFFFFFFFu, code == 5u);
    const uint32_t bg = __ballot_sync(0xFFFFFFFFu, code == 6u);
    const uint32_t bt = __ballot_sync(0xFFFFFFFFu, code == 7u);
    if (lane == p) {
      peq.a[k] = ba;
      peq.c[k] = bc;
      peq.g[k] = bg;
      peq.t[k] = bt;
    }
  }
}

// Converts pair p's text into planes in shared memory (all lanes participate).
__device__ __forceinline__ void myers_load_text(const uint8_t* text, uint32_t n, uint32_t p,
                                                uint32_t lane, MyersSmem sm) {
  const uint32_t words = (n + 31u) / 32u;
  uint32_t* dst = sm.planes + (size_t)p * sm.tw * 3u;
  for (uint32_t x = 0; x < words; ++x) {
    const uint32_t pos = x * 32u + lane;
    const uint32_t code = pos < n ? base_code(ldb(text, pos)) : 0u;
    const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, code & 1u);
    const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, code & 2u);
    const uint32_t bv = __ballot_sync(0xFFFFFFFFu, code & 4u);
    if (lane == 0) {
      dst[3 * x + 0] = b0;
      dst[3 * x + 1] = b1;
      dst[3 * x + 2] = bv;
    }
  }
}

// Runs the recurrence for this lane's pair. Returns true with (dist, end) on a
// hit <= max_k. L >= ceil(m / 32); limbs above the pattern stay masked to zero.
template <int L>
__device__ __forceinline__ bool myers_lane(const MyersPeq<L>& peq, uint32_t m, uint32_t n,
                                           uint32_t max_k, const uint32_t* planes,
                                           uint32_t& dist, uint32_t& end_pos) {
  if (m == 0) {  // myers.rs:50-54
    dist = 0;
    end_pos = 0;
    return true;
  }
  if (n == 0) {  // myers.rs:55-58
    dist = m;
    end_pos = 0;
    return m <= max_k;
  }
  const uint32_t nl = (m + 31u) / 32u;
  const uint32_t top_used = m - 32u * (nl - 1u);
  const uint32_t top_mask = top_used == 32u ? 0xFFFFFFFFu : ((1u << top_used) - 1u);
  const uint32_t high = 1u << (top_used - 1u);
  uint32_t vp[L], vn[L], lm[L];
#pragma unroll
  for (int k = 0; k < L; ++k) {
    lm[k] = (uint32_t)k + 1u < nl ? 0xFFFFFFFFu : ((uint32_t)k + 1u == nl ? top_mask : 0u);
    vp[k] = lm[k];
    vn[k] = 0u;
  }
  uint32_t err = m, best = m, pos = 0;
  uint32_t t0 = 0, t1 = 0, tv = 0;
  for (uint32_t j = 0; j < n; ++j) {
    const uint32_t bit = j & 31u;
    if (bit == 0u) {
      const uint32_t x = j >> 5;
      t0 = planes[3 * x + 0];
      t1 = planes[3 * x + 1];
      tv = planes[3 * x + 2];
    }
    const bool c0 = (t0 >> bit) & 1u, c1 = (t1 >> bit) & 1u, v = (tv >> bit) & 1u;
    uint32_t carry = 0, hin_p = 0, hin_n = 0, hp_top = 0, hn_top = 0;
#pragma unroll
    for (int k = 0; k < L; ++k) {
      uint32_t eq = c1 ? (c0 ? peq.t[k] : peq.g[k]) : (c0 ? peq.c[k] : peq.a[k]);
      eq = v ? eq : 0u;
      const uint32_t vpk = vp[k], vnk = vn[k];
      const uint32_t x = eq | vnk;
      const uint64_t s = (uint64_t)(eq & vpk) + (uint64_t)vpk + (uint64_t)carry;
      const uint32_t sum = (uint32_t)s;
      carry = (uint32_t)(s >> 32);
      const uint32_t d0 = (sum ^ vpk) | x;
      const uint32_t hp = vnk | ~(d0 | vpk);
      const uint32_t hn = d0 & vpk;
      const uint32_t hps = (hp << 1) | hin_p;
      const uint32_t hns = (hn << 1) | hin_n;
      hin_p = hp >> 31;
      hin_n = hn >> 31;
      vp[k] = (hns | ~(d0 | hps)) & lm[k];
      vn[k] = (d0 & hps) & lm[k];
      if ((uint32_t)k + 1u == nl) {
        hp_top = hp;
        hn_top = hn;
      }
    }
    if (hp_top & high) err += 1u;
    if (hn_top & high) err -= 1u;
    if (err <= best) {
      best = err;
      pos = j + 1u;
    }
    const uint32_t rem = n - 1u - j;
    const uint32_t sat = err > rem ? err - rem : 0u;
    if (best > max_k && sat > max_k) return false;  // myers.rs:194
  }
  if (best <= max_k) {
    dist = best;
    end_pos = pos;
    return true;
  }
  return false;
}

}  // namespace kira
