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

// Where wavefront (score s, layer) lives: traceback keeps every score, score-only
// a ring of meta_slots scores with ring_width entries per layer.
__device__ __forceinline__ uint32_t wfa_slot(const WfaLaunch& L, int s) {
  return L.ring_width ? (uint32_t)s % L.meta_slots : (uint32_t)s;
}

// Traceback in one lane (build_cigar, wfa.rs:762-952). Ops are pushed in reverse
// order into the pair's slot with push_cigar's merging (wfa.rs:954-962); returns
// the diagonal at termination (the alignment's text start).
__device__ int wfa_traceback(const WfaLaunch& L, const int2* __restrict__ meta,
                             const int16_t* __restrict__ H, const uint32_t* pw,
                             const uint32_t* tw, int m, int n, int s, int k,
                             uint32_t* __restrict__ slot, uint32_t& nops, bool& overflow) {
  auto get = [&](int layer, int sc, int kk) -> int {
    if (sc < 0) return kWfaNone;
    return wfa_get(H, wfa_unpack(meta[(uint32_t)sc * 3u + layer]), kk);
  };
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

template <bool TB>
__global__ void __launch_bounds__(128) wfa_kernel(DevPairs P, WfaLaunch L) {
  extern __shared__ __align__(16) uint8_t wfa_smem[];
  const int lane = threadIdx.x & 31;
  const uint32_t wib = threadIdx.x >> 5;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + wib;
  uint8_t* my = wfa_smem + (size_t)wib * L.smem_warp;
  uint32_t* pw = (uint32_t*)(my + 16);
  uint32_t* tw = (uint32_t*)(my + L.pat_region + 16);
  uint8_t* pb = (uint8_t*)pw;
  uint8_t* tb = (uint8_t*)tw;
  uint8_t* scr = L.scratch + (size_t)warp * L.warp_bytes;
  int2* meta = (int2*)scr;
  int16_t* H = (int16_t*)(scr + L.meta_bytes);
  const int x = L.x, oi = L.o + L.ei, od = L.o + L.ed;

  for (;;) {
    uint32_t p = 0;
    if (lane == 0) p = atomicAdd(L.work, 1u);
    p = __shfl_sync(kFull, p, 0);
    if (p >= L.n) break;
    const int m = (int)P.read_len[p], n = (int)P.win_len[p];
    kira_wfa_result res{};
    res.cost = -1;
    res.score = 0;
    if (!L.valid) {  // WfaCosts::scored refused the configuration: None
      if (lane == 0) {
        L.out[p] = res;
        if (TB) L.ncig[p] = 0;
      }
      continue;
    }
    if (m == 0) {  // wfa.rs:555-563
      if (lane == 0) {
        res.found = 1;
        res.cost = 0;
        L.out[p] = res;
        if (TB) L.ncig[p] = 0;
      }
      continue;
    }
    const uint8_t* rs = P.read_seq + P.read_off[p];
    const uint8_t* ws = P.win_seq + P.win_off[p];
    for (int i = lane; i < m; i += 32) pb[i] = __ldg(rs + i);
    for (int i = lane; i < n; i += 32) tb[i] = __ldg(ws + i);
    int S = L.max_score_pp ? L.max_score_pp[p] : L.max_score;
    if (!L.max_score_pp && S < 0) S = wfa_budget(m, L);
    // The all-insertion path reaches the pattern end by cost o + ei*m, so the
    // exact search ends by then; a pruned search advances its furthest point
    // by an antidiagonal at least every max(x, o + ei).
    const int64_t cap = L.drop < 0 ? (int64_t)L.o + (int64_t)L.ei * m
                                   : (int64_t)max(x, oi) * (2 * m + n + 2);
    const int S_loop = (int)max((int64_t)0, min((int64_t)S, cap));  // score 0 always runs
    int tbf = L.tbf_pp ? L.tbf_pp[p] : L.tbf;
    tbf = min(max(tbf, 0), max(n - 1, 0));
    __syncwarp();

    uint32_t top = 0;  // traceback mode: next free history entry
    int done_s = -1, k_end = 0, last_live = 0;
    bool overflow = false;
    for (int s = 0; s <= S_loop; ++s) {
      // Sources: lanes 0..4 fetch M[s-x], M[s-o-ei], M[s-o-ed], I[s-ei], D[s-ed].
      int2 mv = wfa_empty();
      if (s > 0 && lane < 5) {
        const int sc = lane == 0 ? s - x : lane == 1 ? s - oi : lane == 2 ? s - od
                       : lane == 3 ? s - L.ei : s - L.ed;
        const int layer = lane < 3 ? 0 : lane - 2;
        if (sc >= 0 && sc < s) mv = meta[wfa_slot(L, sc) * 3u + layer];
      }
      WfaWave src[5];
#pragma unroll
      for (int t = 0; t < 5; ++t)
        src[t] = wfa_unpack(make_int2(__shfl_sync(kFull, mv.x, t), __shfl_sync(kFull, mv.y, t)));
      const WfaWave& mx = src[0];
      const WfaWave& moi = src[1];
      const WfaWave& mod = src[2];
      const WfaWave& ie = src[3];
      const WfaWave& de = src[4];
      int ilo = INT32_MAX, ihi = INT32_MIN, dlo = INT32_MAX, dhi = INT32_MIN;
      int mlo = INT32_MAX, mhi = INT32_MIN;
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
      const int iw = ilo <= ihi ? ihi - ilo + 1 : 0;
      const int dw = dlo <= dhi ? dhi - dlo + 1 : 0;
      const int mw = mlo <= mhi ? mhi - mlo + 1 : 0;
      uint32_t ib, db, mb;
      if (L.ring_width) {
        const uint32_t sl = wfa_slot(L, s) * 3u * L.ring_width;
        mb = sl;
        ib = sl + L.ring_width;
        db = sl + 2u * L.ring_width;
        if ((uint32_t)max(mw, max(iw, dw)) > L.ring_width) overflow = true;
      } else {
        ib = top;
        db = ib + (uint32_t)iw;
        mb = db + (uint32_t)dw;
        top = mb + (uint32_t)mw;
        if (top > L.hist_cap || (uint32_t)s >= L.meta_slots) overflow = true;
      }
      if (overflow) break;

      // Pass 1: I, D, M per diagonal; extension; trimming and done ballots.
      int ifirst = INT32_MAX, ilast = INT32_MIN, dfirst = INT32_MAX, dlast = INT32_MIN;
      int mfirst = INT32_MAX, mlast = INT32_MIN, kdone = INT32_MAX, mad = INT32_MIN;
      for (int c0 = mlo; c0 <= mhi; c0 += 32) {
        const int k = c0 + lane;
        const bool act = k <= mhi;
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
        const unsigned bi = __ballot_sync(kFull, vi != kWfaNone);
        const unsigned bd = __ballot_sync(kFull, vd != kWfaNone);
        const unsigned bm = __ballot_sync(kFull, vm != kWfaNone);
        const unsigned bx = __ballot_sync(kFull, act && vm >= m);
        if (bi) ifirst = min(ifirst, c0 + wfa_low_bit(bi)), ilast = c0 + wfa_high_bit(bi);
        if (bd) dfirst = min(dfirst, c0 + wfa_low_bit(bd)), dlast = c0 + wfa_high_bit(bd);
        if (bm) mfirst = min(mfirst, c0 + wfa_low_bit(bm)), mlast = c0 + wfa_high_bit(bm);
        if (bx && kdone == INT32_MAX) kdone = c0 + wfa_low_bit(bx);
      }
      // Pass 2 (adaptive): prune_wavefront on the extended M, then the done test.
      if (L.drop >= 0 && mfirst <= mlast) {
        const int th = __reduce_max_sync(kFull, mad) - L.drop;
        mfirst = INT32_MAX, mlast = INT32_MIN, kdone = INT32_MAX;
        for (int c0 = mlo; c0 <= mhi; c0 += 32) {
          const int k = c0 + lane;
          int v = kWfaNone;
          if (k <= mhi) {
            const uint32_t at = mb + (uint32_t)(k - mlo);
            v = wfa_dec(H[at]);
            if (v != kWfaNone && 2 * v + k < th) {
              v = kWfaNone;
              H[at] = wfa_enc(v);
            }
          }
          const unsigned bm = __ballot_sync(kFull, v != kWfaNone);
          const unsigned bx = __ballot_sync(kFull, v != kWfaNone && v >= m);
          if (bm) mfirst = min(mfirst, c0 + wfa_low_bit(bm)), mlast = c0 + wfa_high_bit(bm);
          if (bx && kdone == INT32_MAX) kdone = c0 + wfa_low_bit(bx);
        }
      }
      if (lane == 0) {
        const uint32_t sl = wfa_slot(L, s) * 3u;
        meta[sl + 0] = mfirst <= mlast ? wfa_pack(mfirst, mlast, mb + (uint32_t)(mfirst - mlo))
                                       : wfa_empty();
        meta[sl + 1] = ifirst <= ilast ? wfa_pack(ifirst, ilast, ib + (uint32_t)(ifirst - ilo))
                                       : wfa_empty();
        meta[sl + 2] = dfirst <= dlast ? wfa_pack(dfirst, dlast, db + (uint32_t)(dfirst - dlo))
                                       : wfa_empty();
      }
      __syncwarp();
      if (kdone != INT32_MAX) {
        done_s = s;
        k_end = kdone;
        break;
      }
      // Nothing reached within the look-back window: no later score can reach anything.
      if (mfirst <= mlast || ifirst <= ilast || dfirst <= dlast) last_live = s;
      else if (s - last_live > L.lookback) break;
    }

    if (overflow) {
      if (lane == 0) atomicOr(L.flags, 2u);
    } else if (done_s >= 0) {
      res.found = 1;
      res.cost = done_s;
      res.score = L.scored ? m * L.match - done_s : done_s;
      res.text_end = (uint32_t)(m + k_end);
    }
    if (lane == 0) {
      if (TB) {
        uint32_t nops = 0;
        if (res.found) {
          bool ovf = false;
          uint32_t* slot = L.slots + (size_t)p * L.slot_cap;
          const int k0 = wfa_traceback(L, meta, H, pw, tw, m, n, done_s, k_end, slot, nops, ovf);
          res.text_start = (uint32_t)max(k0, 0);
          if (ovf) atomicOr(L.flags, 1u);
        }
        L.ncig[p] = nops;
      }
      L.out[p] = res;
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

cudaError_t wfa_blocks_per_sm(bool traceback, size_t smem, int threads, int* per_sm) {
  auto kern = traceback ? wfa_kernel<true> : wfa_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, threads, smem);
}

cudaError_t launch_wfa(const DevPairs& P, const WfaLaunch& L, uint32_t blocks,
                       uint32_t warps_per_block, bool traceback, cudaStream_t st) {
  const size_t smem = (size_t)L.smem_warp * warps_per_block;
  const uint32_t threads = 32u * warps_per_block;
  if (traceback) wfa_kernel<true><<<blocks, threads, smem, st>>>(P, L);
  else wfa_kernel<false><<<blocks, threads, smem, st>>>(P, L);
  return cudaGetLastError();
}

cudaError_t launch_wfa_compact(const WfaCompact& C, int sms, cudaStream_t st) {
  uint64_t b = (C.n + 255) / 256;
  if (b < 1) b = 1;
  if (b > (uint64_t)sms * 8) b = (uint64_t)sms * 8;
  wfa_compact_kernel<<<(int)b, 256, 0, st>>>(C);
  return cudaGetLastError();
}

}  // namespace kira
