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
// the limb width does not change any result). One lane per pair:
//   * pattern and text come from the 2-bit + valid plane arenas (planes.cuh):
//     one 32-base word is two 16-byte loads and a funnel shift, no cross-lane work;
//   * Peq lives in shared memory as [k][code][lane] with code 4 = "matches
//     nothing" (all zero), so every per-lane read is bank-conflict-free.
//   * Per column and limb: one LDS for Eq (instead of a 4-way select), the
//     (Eq & VP) + VP carry chain on the PTX carry flag (add.cc / addc), and one
//     funnel shift for each of the HP / HN shifts across limbs.
#pragma once

#include "addchain.cuh"
#include "common.cuh"
#include "planes.cuh"

namespace kira {

// Shared memory of one warp: Peq[k][code][lane], code 4 = "matches nothing".
struct MyersSmem {
  uint32_t* peq;  // [L][5][32]
};

// Builds this lane's Peq columns from the pattern's plane words (no cross-lane
// work): eq_A = ~b1 & ~b0 & valid, ... for the bases below m.
template <int L>
__device__ __forceinline__ void myers_build_peq(const uint4* __restrict__ planes, uint64_t pos,
                                                uint32_t m, uint32_t lane, MyersSmem sm) {
#pragma unroll
  for (int k = 0; k < L; ++k) {
    const PlaneWord pw = plane_word_at(planes, pos + 32u * k);
    const uint32_t base = 32u * (uint32_t)k;
    const uint32_t lm = base < m ? low_mask(m - base) : 0u;
    const uint32_t v = pw.v & lm;
    uint32_t* col = sm.peq + (uint32_t)k * 160u + lane;
    col[0] = ~pw.b1 & ~pw.b0 & v;
    col[32] = ~pw.b1 & pw.b0 & v;
    col[64] = pw.b1 & ~pw.b0 & v;
    col[96] = pw.b1 & pw.b0 & v;
    col[128] = 0u;
  }
}

// Runs the recurrence for this lane's pair. Returns true with (dist, end) on a
// hit <= max_k. UNIFORM: every lane of the warp has ceil(m / 32) == L (no limb
// masks below the top limb). Otherwise limbs above the pattern stay masked to 0.
template <int L, bool UNIFORM>
__device__ __forceinline__ bool myers_lane(uint32_t m, uint32_t n, uint32_t max_k,
                                           MyersSmem sm, const uint4* __restrict__ tplanes,
                                           uint64_t tpos, uint32_t lane, uint32_t& dist,
                                           uint32_t& end_pos) {
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
    if (UNIFORM)
      lm[k] = k + 1 < L ? 0xFFFFFFFFu : top_mask;
    else
      lm[k] = (uint32_t)k + 1u < nl ? 0xFFFFFFFFu : ((uint32_t)k + 1u == nl ? top_mask : 0u);
    vp[k] = lm[k];
    vn[k] = 0u;
  }
  const uint32_t* peq = sm.peq + lane;
  uint32_t err = m, best = m, pos = 0;
  // Software pipelined over the text: the Peq words of column j + 1 are loaded while
  // column j is computed, and the text plane word of the next 32 columns one block
  // ahead, so neither load's latency sits on the column-to-column chain.
  // Column code: 0-3 for ACGT, 4 (an all-zero Peq row) for any other base.
  auto code_at = [](uint32_t bit, const PlaneWord& w) {
    return ((w.v >> bit) & 1u) ? (((w.b0 >> bit) & 1u) | (((w.b1 >> bit) & 1u) << 1)) : 4u;
  };
  PlaneWord cw = plane_word_at(tplanes, tpos);
  PlaneWord nw = n > 32u ? plane_word_at(tplanes, tpos + 32u) : cw;
  uint32_t eqn[L];
  {
    const uint32_t* pc = peq + code_at(0u, cw) * 32u;
#pragma unroll
    for (int k = 0; k < L; ++k) eqn[k] = pc[k * 160];
  }
  for (uint32_t j = 0; j < n; ++j) {
    uint32_t eq[L], av[L], sum[L];
#pragma unroll
    for (int k = 0; k < L; ++k) {
      eq[k] = eqn[k];
      av[k] = eq[k] & vp[k];
    }
    if ((j & 31u) == 31u) {  // column j + 1 opens the next block of 32
      cw = nw;
      if (j + 33u < n) nw = plane_word_at(tplanes, tpos + j + 33u);
    }
    if (j + 1u < n) {
      const uint32_t* pc = peq + code_at((j + 1u) & 31u, cw) * 32u;
#pragma unroll
      for (int k = 0; k < L; ++k) eqn[k] = pc[k * 160];
    }
    add_chain<L>(av, vp, sum);
    uint32_t hp_prev = 0, hn_prev = 0, hp_top = 0, hn_top = 0;
#pragma unroll
    for (int k = 0; k < L; ++k) {
      const uint32_t vpk = vp[k], vnk = vn[k];
      const uint32_t d0 = (sum[k] ^ vpk) | eq[k] | vnk;
      const uint32_t hp = vnk | ~(d0 | vpk);
      const uint32_t hn = d0 & vpk;
      const uint32_t hps = k ? __funnelshift_l(hp_prev, hp, 1) : (hp << 1);
      const uint32_t hns = k ? __funnelshift_l(hn_prev, hn, 1) : (hn << 1);
      hp_prev = hp;
      hn_prev = hn;
      vp[k] = (hns | ~(d0 | hps)) & lm[k];
      vn[k] = (d0 & hps) & lm[k];
      if (UNIFORM) {
        if (k == L - 1) {
          hp_top = hp;
          hn_top = hn;
        }
      } else if ((uint32_t)k + 1u == nl) {
        hp_top = hp;
        hn_top = hn;
      }
    }
    err += (hp_top & high) ? 1u : 0u;
    err -= (hn_top & high) ? 1u : 0u;
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
