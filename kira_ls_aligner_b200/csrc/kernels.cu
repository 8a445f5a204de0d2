// kernels.cu -- device kernels of libkira_gpu and their launchers.
#include <atomic>
#include <cuda_runtime.h>

#include "bsw.cuh"
#include "bsw16.cuh"
#include "internal.h"
#include "myers.cuh"
#include "nmmd.cuh"
#include "planes.cuh"
#include "qgram.cuh"
#include "sieve.cuh"

namespace kira {

// ---------------------------------------------------------------------------
// Sieve drop-in: CudaBackend::run_batch semantics (src/cuda/backend.rs:95-249,
// src/cuda/spectral.cu:136-213). Inputs are the packed read and the packed
// phase-0 window of each job, concatenated in two device arenas.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sieve_dropin_kernel(SieveJobsDev J,
                                                           kira_sieve_result* __restrict__ out) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < J.n; p += warps) {
    const uint32_t q = J.read_nucs[p], w = J.ref_nucs[p];
    const uint8_t* rb = J.read_bits + J.read_off[p];
    const uint8_t* wb = J.ref_bits + J.ref_off[p];
    auto rcode = [&](uint32_t pos) { return ((ldb(rb, pos >> 2) >> ((pos & 3u) * 2u)) & 3u) | 4u; };
    auto wcode = [&](uint32_t pos) { return ((ldb(wb, pos >> 2) >> ((pos & 3u) * 2u)) & 3u) | 4u; };
    const SieveOut so = sieve_warp<8>(q, w, rcode, wcode, false);
    if (lane == 0) {
      kira_sieve_result r;
      if (q == 0 || w < q) {  // spectral.cu:156-163
        r.shift = -1;
        r.mismatches = INT32_MAX;
        r.second_mismatches = INT32_MAX;
      } else {
        const uint32_t limit = min(J.max_mism[p], q);  // backend.rs:185-188
        const bool acc = so.mism <= limit;
        r.shift = acc ? (int32_t)so.shift : -1;
        r.mismatches = acc ? (int32_t)so.mism : INT32_MAX;
        r.second_mismatches = so.second == kNoKey ? INT32_MAX : (int32_t)so.second;
      }
      out[p] = r;
    }
  }
}

// ---------------------------------------------------------------------------
// Plane packing: a warp covers 512 bases (16 plane blocks); lane l loads bases
// 16l .. 16l+15 as one 16-byte load and turns each 4-byte word into three nibbles
// (code bit 0, code bit 1, valid) with SWAR byte arithmetic: the 2-bit code of
// every byte is ((b >> 1) ^ (b >> 2)) & 3 (base_code), a PRMT table lookup gives
// the letter that code stands for, and the case-folded byte equals it exactly for
// A, C, G, T. A multiply by 0x01020408 gathers bit 0 of each byte into bits
// 24..27. The even lane of each pair stores the block of its 32 bases.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void plane_nibbles(uint32_t w, uint32_t& n0, uint32_t& n1,
                                              uint32_t& nv) {
  const uint32_t x = (w >> 1) ^ (w >> 2);       // bits 0-1 of each byte: the code
  const uint32_t y = x & 0x03030303u;
  const uint32_t z = y | (y >> 4);              // bytes 0 and 2: two codes each
  uint32_t sel, letter;
  asm("prmt.b32 %0, %1, 0, 0x4420;" : "=r"(sel) : "r"(z));
  asm("prmt.b32 %0, %1, 0, %2;" : "=r"(letter) : "r"(0x54474341u), "r"(sel));  // "ACGT"
  const uint32_t t = (w & 0xDFDFDFDFu) ^ letter;  // zero byte: an ACGT base (any case)
  const uint32_t ok = ~(((t & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | t) & 0x80808080u;
  const uint32_t v = ok >> 7;                   // 0x01 per valid byte
  n0 = ((x & v) * 0x01020408u) >> 24;
  n1 = (((x >> 1) & v) * 0x01020408u) >> 24;
  nv = (v * 0x01020408u) >> 24;
}

__global__ void __launch_bounds__(256) pack_planes_kernel(const uint8_t* __restrict__ seq,
                                                          uint64_t len, uint4* __restrict__ out,
                                                          uint64_t nblocks) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const bool aligned = ((uintptr_t)seq & 15u) == 0u;
  for (uint64_t sp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       sp * 16u < nblocks; sp += nwarps) {
    const uint64_t p0 = sp * 512u + lane * 16u;
    uint32_t w[4];
    if (aligned && p0 + 16u <= len) {
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(seq + p0));
      w[0] = q.x, w[1] = q.y, w[2] = q.z, w[3] = q.w;
    } else {  // the arena's ragged end (or an unaligned arena): byte loads, zeros past len
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        uint32_t x = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const uint64_t p = p0 + 4u * k + b;
          x |= (p < len ? ldb(seq, p) : 0u) << (8 * b);
        }
        w[k] = x;
      }
    }
    uint32_t b0 = 0, b1 = 0, bv = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t n0, n1, nv;
      plane_nibbles(w[k], n0, n1, nv);
      b0 |= n0 << (4 * k);
      b1 |= n1 << (4 * k);
      bv |= nv << (4 * k);
    }
    const uint32_t o0 = __shfl_down_sync(0xFFFFFFFFu, b0, 1);
    const uint32_t o1 = __shfl_down_sync(0xFFFFFFFFu, b1, 1);
    const uint32_t ov = __shfl_down_sync(0xFFFFFFFFu, bv, 1);
    const uint64_t blk = sp * 16u + (lane >> 1);
    if (!(lane & 1u) && blk < nblocks)
      out[blk] = make_uint4(b0 | (o0 << 16), b1 | (o1 << 16), bv | (ov << 16), 0u);
  }
}

// Number of positions i in [0, len) with a[i] != b[i], stopping once above
// `limit` (bounded_hamming, src/alignment/mod.rs:764-776). Warp-cooperative.
__device__ __forceinline__ uint32_t warp_bounded_hamming(const uint8_t* a, const uint8_t* b,
                                                         uint32_t len, uint32_t limit,
                                                         uint32_t lane) {
  uint32_t m = 0;
  for (uint32_t c = 0; c < len; c += 32u) {
    const uint32_t i = c + lane;
    const bool ne = i < len && ldb(a, i) != ldb(b, i);
    m += __popc(__ballot_sync(0xFFFFFFFFu, ne));
    if (m > limit) break;
  }
  return m;
}

// spectral_hit_is_certified (src/alignment/mod.rs:688-762), warp-cooperative.
__device__ bool warp_certify(const uint8_t* read, const uint8_t* ref, uint32_t len, uint32_t mism,
                             uint32_t second, uint32_t max_mism, bool strict, uint32_t lane) {
  if (mism > max_mism) return false;
  if (second != kNoKey && second <= mism + 1u) return false;
  if (mism == 0) return true;
  if (mism > 2) return false;
  uint32_t n = 0, pos0 = 0xFFFFFFFFu, pos1 = 0xFFFFFFFFu;
  for (uint32_t c = 0; c < len; c += 32u) {
    const uint32_t i = c + lane;
    const bool ne = i < len && ldb(read, i) != ldb(ref, i);
    uint32_t b = __ballot_sync(0xFFFFFFFFu, ne);
    while (b) {
      const uint32_t at = c + (uint32_t)(__ffs(b) - 1);
      if (n == 0) pos0 = at;
      else if (n == 1) pos1 = at;
      ++n;
      b &= b - 1u;
    }
  }
  if (n != mism) return false;
  const uint32_t edge = min(len, 8u);
  if (pos0 < edge || pos0 + edge >= len) return false;
  if (n == 2 && (pos1 < edge || pos1 + edge >= len)) return false;
  if (n == 2 && (pos1 > pos0 ? pos1 - pos0 : 0u) <= 4u) return false;
  const uint32_t p = pos0;
  const uint32_t suffix = len > p + 1u ? len - (p + 1u) : 0u;
  const uint32_t min_suffix = strict ? 4u : 8u;
  if (suffix >= min_suffix) {
    if (warp_bounded_hamming(read + p + 1, ref + p, len - p - 1u, 1u, lane) <= 1u) return false;
    if (warp_bounded_hamming(read + p, ref + p + 1, len - p - 1u, 1u, lane) <= 1u) return false;
    if (strict && suffix >= 6u) {
      if (warp_bounded_hamming(read + p + 2, ref + p, len - p - 2u, 1u, lane) <= 1u) return false;
      if (warp_bounded_hamming(read + p, ref + p + 2, len - p - 2u, 1u, lane) <= 1u) return false;
    }
  }
  return true;
}

// spectral_hit_is_certified (src/alignment/mod.rs:688-762) for one lane's pair.
__device__ __forceinline__ uint32_t lane_bounded_hamming(const uint8_t* a, const uint8_t* b,
                                                         uint32_t len, uint32_t limit) {
  uint32_t m = 0;
  for (uint32_t i = 0; i < len; ++i) {
    m += ldb(a, i) != ldb(b, i) ? 1u : 0u;
    if (m > limit) break;
  }
  return m;
}

__device__ bool lane_certify(const uint8_t* read, const uint8_t* ref, uint32_t len, uint32_t mism,
                             uint32_t second, uint32_t max_mism, bool strict) {
  if (mism > max_mism) return false;
  if (second != 0xFFFFFFFFu && second <= mism + 1u) return false;
  if (mism == 0) return true;
  if (mism > 2) return false;
  uint32_t n = 0, pos0 = 0xFFFFFFFFu, pos1 = 0xFFFFFFFFu;
  for (uint32_t i = 0; i < len; ++i) {
    if (ldb(read, i) != ldb(ref, i)) {
      if (n == 0) pos0 = i;
      else if (n == 1) pos1 = i;
      ++n;
      if (n > mism) break;  // decided: n != mism
    }
  }
  if (n != mism) return false;
  const uint32_t edge = min(len, 8u);
  if (pos0 < edge || pos0 + edge >= len) return false;
  if (n == 2 && (pos1 < edge || pos1 + edge >= len)) return false;
  if (n == 2 && (pos1 > pos0 ? pos1 - pos0 : 0u) <= 4u) return false;
  const uint32_t p = pos0;
  const uint32_t suffix = len > p + 1u ? len - (p + 1u) : 0u;
  const uint32_t min_suffix = strict ? 4u : 8u;
  if (suffix >= min_suffix) {
    if (lane_bounded_hamming(read + p + 1, ref + p, len - p - 1u, 1u) <= 1u) return false;
    if (lane_bounded_hamming(read + p, ref + p + 1, len - p - 1u, 1u) <= 1u) return false;
    if (strict && suffix >= 6u) {
      if (lane_bounded_hamming(read + p + 2, ref + p, len - p - 2u, 1u) <= 1u) return false;
      if (lane_bounded_hamming(read + p, ref + p + 2, len - p - 2u, 1u) <= 1u) return false;
    }
  }
  return true;
}

__device__ __forceinline__ uint32_t sieve_threshold_for(int32_t thr, uint32_t q) {
  // router::spectral_max_mismatches (src/alignment/router.rs:191-195), defaults 3 % / 2.
  return thr < 0 ? max((q * 3u) / 100u, 2u) : (uint32_t)thr;
}

__device__ __forceinline__ uint32_t myers_k_for(int32_t k, uint32_t q) {
  // router::myers_reject_bound (src/alignment/router.rs:199-203), defaults 15 % + 4.
  return k < 0 ? (q * 15u) / 100u + 4u : (uint32_t)k;
}

// Result rows of the sieve stage.
__device__ __forceinline__ void write_myers_reject(const VerifyDev& V, uint32_t p) {
  kira_sw_result r{};
  r.status = KIRA_PAIR_MYERS_REJECT;
  V.out[p] = r;
  V.ncig[p] = 0;
}

// build_certified_spectral_alignment (mod.rs:636-686).
__device__ __forceinline__ void write_certified(const VerifyDev& V, uint32_t p, uint32_t q,
                                                const LaneSieve& so) {
  kira_sw_result r;
  r.score = (int32_t)(q - so.mism) * V.sw.match - (int32_t)so.mism * V.sw.mismatch;
  r.ref_start = so.shift;
  r.ref_end = so.shift + q;
  r.read_start = 0;
  r.read_end = (int32_t)q;
  r.cigar_off = 0;
  r.n_cigar = 1;
  r.status = KIRA_PAIR_CERTIFIED;
  r.early_abort = 0;
  r.reserved = 0;
  V.out[p] = r;
  V.ncig[p] = 1;
}

// Warp-aggregated append of `value` for the lanes with `take` (all 32 lanes call).
__device__ __forceinline__ void warp_append(bool take, uint32_t value, uint32_t* count,
                                            uint32_t* list) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t need = __ballot_sync(0xFFFFFFFFu, take);
  uint32_t slot0 = 0;
  if (lane == 0 && need) slot0 = atomicAdd(count, (uint32_t)__popc(need));
  slot0 = __shfl_sync(0xFFFFFFFFu, slot0, 0);
  if (take) list[slot0 + __popc(need & ((1u << lane) - 1u))] = value;
}

// Sieve + certificate of pair p (scan_best_with_second_raw, then the certificate
// of mod.rs:636-686); writes the certified row when it certifies.
template <int RWMAX>
__device__ __forceinline__ bool sieve_certify(const DevPairs& P, const VerifyDev& V, uint32_t p,
                                              uint32_t q, LaneSieve& so) {
  so = sieve_lane<RWMAX>(P.read_planes, P.read_off[p], q, P.win_planes, P.win_off[p],
                         P.win_len[p]);
  const uint32_t thr = sieve_threshold_for(V.sieve_threshold, q);
  const bool cert = so.hit && so.mism <= thr &&
                    lane_certify(P.read_seq + P.read_off[p], P.win_seq + P.win_off[p] + so.shift,
                                 q, so.mism, so.second, thr, V.cert_strict != 0);
  if (cert) write_certified(V, p, q, so);
  return cert;
}

// Stage 1 of the composed path when detail rows are asked for or the filter is
// off: sieve + certificate of every pair, then the 4-gram filter, one lane per pair.
template <int RWMAX>
__global__ void __launch_bounds__(256) verify_sieve_kernel(DevPairs P, VerifyDev V) {
  __shared__ uint32_t qset[8][16 * 32];  // per warp: 4-gram bitmap [word][lane]
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t* myset = &qset[threadIdx.x >> 5][lane];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < P.n; base += stride) {
    const uint32_t p = base + threadIdx.x;
    const bool valid = p < P.n;
    bool cert = false;
    uint32_t q = 0;
    if (valid) {
      q = P.read_len[p];
      LaneSieve so{false, 0, 0, 0xFFFFFFFFu};
      cert = sieve_certify<RWMAX>(P, V, p, q, so);
      if (V.detail) {
        kira_verify_detail dt;
        dt.sieve_shift = so.hit ? (int32_t)so.shift : -1;
        dt.sieve_mism = so.hit ? (int32_t)so.mism : INT32_MAX;
        dt.sieve_second = so.hit && so.second != 0xFFFFFFFFu ? (int32_t)so.second : INT32_MAX;
        dt.myers_dist = -1;
        dt.myers_end = -1;
        V.detail[p] = dt;
      }
      if (!cert) V.sw_offset[p] = so.hit ? (int32_t)so.shift : 0;
    }
    // Exact 4-gram prefilter: a pair it rejects is a Myers None (same result).
    bool gone = false;
    if (valid && !cert && V.qgram) {
      const uint32_t k = myers_k_for(V.myers_k, q);
      gone = qgram4_reject(P.read_planes, P.read_off[p], q, P.win_planes, P.win_off[p],
                           P.win_len[p], k, myset);
      if (gone) write_myers_reject(V, p);
    }
    warp_append(valid && !cert && !gone, p, V.counters + 0, V.myers_list);
  }
}

// Stage 1, filter first (no detail rows): the 4-gram count of every pair decides
// two things. Myers rejects the pair when count < m - 3 - 4k (qgram.cuh). And the
// certificate needs a shift with at most min(threshold, 2) mismatches
// (lane_certify): a shift with d mismatches leaves at least m - 3 - 4d read
// 4-grams untouched, each found verbatim in the window, so count < m - 3 -
// 4 min(threshold, 2) proves no shift certifies. A pair below both bounds is a
// Myers reject whatever its sieve says, and its sieve is never run; the others go
// to verify_sieve_list_kernel, tagged when the count already rejects them unless
// they certify. Rows are those of verify_sieve_kernel.
__global__ void __launch_bounds__(256) verify_filter_kernel(DevPairs P, VerifyDev V) {
  __shared__ uint32_t qset[8][16 * 32];
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t* myset = &qset[threadIdx.x >> 5][lane];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < P.n; base += stride) {
    const uint32_t p = base + threadIdx.x;
    const bool valid = p < P.n;
    uint32_t outcome = 0;
    if (valid) {
      const uint32_t q = P.read_len[p];
      const int32_t thr2 = (int32_t)min(sieve_threshold_for(V.sieve_threshold, q), 2u);
      const int32_t hi = (int32_t)q - 3 - 4 * (int32_t)myers_k_for(V.myers_k, q);
      const int32_t lo = min(hi, (int32_t)q - 3 - 4 * thr2);
      outcome = qgram4_outcome(P.read_planes, P.read_off[p], q, P.win_planes, P.win_off[p],
                               P.win_len[p], lo, hi, myset);
      if (outcome == 2u) write_myers_reject(V, p);
    }
    warp_append(valid && outcome != 2u, p | (outcome == 1u ? 0x80000000u : 0u), V.sieve_count,
                V.sieve_list);
  }
}

// Stage 1, second pass: sieve + certificate of the listed pairs; a pair that does
// not certify is a Myers reject when tagged, else it goes to the Myers list with
// its sieve shift as the banded-SW offset.
template <int RWMAX>
__global__ void __launch_bounds__(256, 4) verify_sieve_list_kernel(DevPairs P, VerifyDev V) {
  const uint32_t count = *V.sieve_count;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
    const uint32_t idx = base + threadIdx.x;
    const bool valid = idx < count;
    bool to_myers = false;
    uint32_t p = 0;
    if (valid) {
      const uint32_t e = V.sieve_list[idx];
      p = e & 0x7FFFFFFFu;
      LaneSieve so{false, 0, 0, 0xFFFFFFFFu};
      if (!sieve_certify<RWMAX>(P, V, p, P.read_len[p], so)) {
        if (e >> 31) {
          write_myers_reject(V, p);
        } else {
          V.sw_offset[p] = so.hit ? (int32_t)so.shift : 0;
          to_myers = true;
        }
      }
    }
    warp_append(to_myers, p, V.counters + 0, V.myers_list);
  }
}

// One thread per pair: 12-byte packed descriptors -> the pipeline's arrays.
__global__ void __launch_bounds__(256) unpack_pairs_kernel(const PackedPair* __restrict__ src,
                                                           uint32_t n, uint64_t* read_off,
                                                           uint32_t* read_len, uint64_t* win_off,
                                                           uint32_t* win_len, int lens) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    const PackedPair d = src[p];
    read_off[p] = d.read_off;
    win_off[p] = d.win_off;
    if (lens) {
      read_len[p] = d.read_len;
      win_len[p] = d.win_len;
    }
  }
}

// ---------------------------------------------------------------------------
// Myers over a work list (one pair per lane; 32 pairs per warp).
// ---------------------------------------------------------------------------
template <int L>
__device__ void myers_warp(const DevPairs& P, const MyersLaunch& M, uint32_t base,
                           uint32_t count, MyersSmem sm) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t item = base + lane;
  const bool valid = item < count;
  const uint32_t pair = valid ? (M.list ? M.list[item] : item) : 0u;
  const uint32_t m = valid ? P.read_len[pair] : 0u;
  if (valid) myers_build_peq<L>(P.read_planes, P.read_off[pair], m, lane, sm);
  __syncwarp();
  uint32_t dist = 0, endp = 0;
  bool hit = false;
  const bool uniform = __all_sync(0xFFFFFFFFu, !valid || (m + 31u) / 32u == (uint32_t)L);
  if (valid) {
    const uint32_t n = P.win_len[pair];
    const uint32_t k = M.per_pair_k ? myers_k_for(M.k, m) : (uint32_t)M.k;
    hit = uniform ? myers_lane<L, true>(m, n, k, sm, P.win_planes, P.win_off[pair], lane, dist,
                                        endp)
                  : myers_lane<L, false>(m, n, k, sm, P.win_planes, P.win_off[pair], lane, dist,
                                         endp);
  }
  __syncwarp();
  if (M.cascade) {
    const uint32_t hits = __ballot_sync(0xFFFFFFFFu, valid && hit);
    uint32_t base_slot = 0;
    if (lane == 0 && hits)
      base_slot = atomicAdd(M.sw_count ? M.sw_count : M.counters + 1, (uint32_t)__popc(hits));
    base_slot = __shfl_sync(0xFFFFFFFFu, base_slot, 0);
    if (valid) {
      if (M.detail) {
        M.detail[pair].myers_dist = hit ? (int32_t)dist : -1;
        M.detail[pair].myers_end = hit ? (int32_t)endp : -1;
      }
      if (hit) {
        const uint32_t rank = (uint32_t)__popc(hits & ((1u << lane) - 1u));
        M.sw_list[base_slot + rank] = M.sw_base + pair;
      } else {
        kira_sw_result r;
        r.score = 0;
        r.ref_start = r.ref_end = 0;
        r.read_start = r.read_end = 0;
        r.cigar_off = 0;
        r.n_cigar = 0;
        r.status = KIRA_PAIR_MYERS_REJECT;
        r.early_abort = 0;
        r.reserved = 0;
        M.out[pair] = r;
        M.ncig[pair] = 0;
      }
    }
  } else if (valid) {
    M.dist[pair] = hit ? (int32_t)dist : -1;
    M.end[pair] = hit ? (int32_t)endp : -1;
  }
}

template <int LMAX>
__global__ void __launch_bounds__(128) myers_kernel(DevPairs P, MyersLaunch M) {
  extern __shared__ uint32_t myers_smem[];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp_in_block = threadIdx.x >> 5;
  MyersSmem sm{myers_smem + (size_t)warp_in_block * M.lmax * 160u};
  const uint32_t count = M.count_dev ? *M.count_dev : M.count;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp_in_block) * 32u; base < count;
       base += nwarps * 32u) {
    const uint32_t item = base + lane;
    uint32_t m = 0;
    if (item < count) m = P.read_len[M.list ? M.list[item] : item];
    uint32_t mx = m;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, off));
    const uint32_t limbs = max((mx + 31u) / 32u, 1u);
    switch (limbs) {
#define KIRA_MYERS_CASE(n)                                     \
  case n:                                                      \
    if (n <= LMAX) {                                           \
      myers_warp<(n <= LMAX ? n : 1)>(P, M, base, count, sm);  \
      break;                                                   \
    }
      KIRA_MYERS_CASE(1) KIRA_MYERS_CASE(2) KIRA_MYERS_CASE(3) KIRA_MYERS_CASE(4)
      KIRA_MYERS_CASE(5) KIRA_MYERS_CASE(6) KIRA_MYERS_CASE(7) KIRA_MYERS_CASE(8)
      KIRA_MYERS_CASE(9) KIRA_MYERS_CASE(10) KIRA_MYERS_CASE(11) KIRA_MYERS_CASE(12)
      KIRA_MYERS_CASE(13) KIRA_MYERS_CASE(14) KIRA_MYERS_CASE(15) KIRA_MYERS_CASE(16)
#undef KIRA_MYERS_CASE
      default: {  // longer patterns: the host rejects them; flag and answer None
        const uint32_t it = base + lane;
        if (it < count) {
          const uint32_t pair = M.list ? M.list[it] : it;
          if (M.cascade) {
            kira_sw_result r{};
            r.status = KIRA_PAIR_MYERS_REJECT;
            M.out[pair] = r;
            M.ncig[pair] = 0;
          } else {
            M.dist[pair] = -1;
            M.end[pair] = -1;
          }
        }
        if (lane == 0 && M.flags) atomicOr(M.flags, 4u);
        break;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Banded SW: DP sweep (group of G lanes per item) and traceback (thread per item)
// ---------------------------------------------------------------------------
// The items [lo, end) of a launch: its trace round, or with B.split one of the two
// halves of the (device-side) item count that run on two streams at once.
__device__ __forceinline__ void bsw_range(const BswLaunch& B, uint32_t& lo, uint32_t& end) {
  const uint32_t count = B.count_dev ? *B.count_dev : B.count;
  if (B.split) {
    const uint32_t mid = (count + 1u) / 2u;
    lo = B.split == 1u ? 0u : mid;
    end = B.split == 1u ? mid : count;
    return;
  }
  lo = B.item_lo;
  end = B.item_hi ? min(count, B.item_hi) : count;
}

template <int G, int K, int T, int MINB, bool FULL>
__global__ void __launch_bounds__(T, MINB) bsw_dp_kernel(DevPairs P, BswLaunch B) {
  extern __shared__ int32_t bsw_smem[];
  constexpr int CAP = G * K;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t g = lane % G;
  const uint32_t gw = lane / G;
  const uint32_t gmask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << (gw * G));
  const uint32_t groups_per_block = blockDim.x / G;
  const uint32_t group_in_block = threadIdx.x / G;
  int32_t* rowbuf = bsw_smem + (size_t)(threadIdx.x >> 5) * 2u * K * 32u;  // per warp
  uint32_t lo, count;
  bsw_range(B, lo, count);
  const uint32_t ngroups = gridDim.x * groups_per_block;
  uint32_t item = lo + blockIdx.x * groups_per_block + group_in_block;
  for (;;) {
    if (B.work) {  // dynamic fetch: the group leader takes the next item
      uint32_t t = 0;
      if (g == 0) t = lo + atomicAdd(B.work, 1u);
      item = __shfl_sync(gmask, t, gw * G);
    }
    if (item >= count) break;
    const uint32_t slot_item = item - B.item_lo;
    const uint32_t pair = B.list ? B.list[item] : item;
    const uint32_t q = P.read_len[pair], w = P.win_len[pair];
    const int32_t band = max(P.bandwidth ? P.bandwidth[pair] : B.sp.band, 1);
    const int32_t offset = B.offset ? B.offset[pair] : 0;
    const int32_t abort_score = P.abort_score ? P.abort_score[pair] : kAbortOff;
    DpEnd end;
    uint64_t cells = 0;
    if (q > B.max_q || (FULL ? (int32_t)w > CAP : 2 * band + 1 > CAP)) {  // outside the shape
      if (g == 0) {
        B.ends[item] = DpEnd{0, 0, 0, kEndOutsideShape};
        atomicOr(B.flags, 2u);
      }
      if (!B.work) item += ngroups;
      continue;
    }
    bsw_group_sweep<G, K, FULL>(
        P.read_seq + P.read_off[pair], q, P.win_seq + P.win_off[pair], w, band, offset,
        abort_score, B.sp, rowbuf, gw * G, B.tg.trace + (size_t)slot_item * B.tg.slot_bytes,
        B.tg.meta + (size_t)slot_item * B.tg.meta_stride, g, gmask, end, cells,
        B.rowkeys ? B.rowkeys + (size_t)item * B.tg.meta_stride : nullptr);
    if (g == 0) {
      B.ends[item] = end;
      if (B.cells) atomicAdd(B.cells, (unsigned long long)cells);
    }
    if (!B.work) item += ngroups;
  }
}

// Packed int16 sweep (bsw16.cuh); same item loop and outputs as bsw_dp_kernel.
template <int G, int K, int T, int MINB>
__global__ void __launch_bounds__(T, MINB) bsw16_dp_kernel(DevPairs P, BswLaunch B) {
  // Dynamic shared memory: each group's trace strip (one interleave block,
  // kStripBytes), then each group's realignment buffer (4 * G * K halves).
  extern __shared__ __align__(128) uint32_t bsw16_smem[];
  constexpr int CAP = 2 * G * K;
  constexpr uint32_t kStripWords = Bsw16Shape<G, K>::kStripBytes / 4u;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t g = lane % G;
  const uint32_t gw = lane / G;
  const uint32_t gmask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << (gw * G));
  const uint32_t groups_per_block = blockDim.x / G;
  const uint32_t group_in_block = threadIdx.x / G;
  uint32_t* strip = bsw16_smem + (size_t)group_in_block * kStripWords;
  uint16_t* rowbuf = reinterpret_cast<uint16_t*>(bsw16_smem + (size_t)(T / G) * kStripWords) +
                     (size_t)group_in_block * 4u * G * K;  // per group
  uint32_t lo, count;
  bsw_range(B, lo, count);
  const uint32_t ngroups = gridDim.x * groups_per_block;
  uint32_t item = lo + blockIdx.x * groups_per_block + group_in_block;
  for (;;) {
    if (B.work) {
      uint32_t t = 0;
      if (g == 0) t = lo + atomicAdd(B.work, 1u);
      item = __shfl_sync(gmask, t, gw * G);
    }
    if (item >= count) break;
    const uint32_t slot_item = item - B.item_lo;
    const uint32_t pair = B.list ? B.list[item] : item;
    const uint32_t q = P.read_len[pair], w = P.win_len[pair];
    const int32_t band = max(P.bandwidth ? P.bandwidth[pair] : B.sp.band, 1);
    const int32_t offset = B.offset ? B.offset[pair] : 0;
    const int32_t abort_score = P.abort_score ? P.abort_score[pair] : kAbortOff;
    DpEnd end;
    uint64_t cells = 0;
    if (q > B.max_q || 2 * band + 1 > CAP) {  // outside the shape
      if (g == 0) {
        B.ends[item] = DpEnd{0, 0, 0, kEndOutsideShape};
        atomicOr(B.flags, 2u);
      }
      if (!B.work) item += ngroups;
      continue;
    }
    bsw16_group_sweep<G, K>(P.read_seq + P.read_off[pair], q, P.win_seq + P.win_off[pair], w,
                            band, offset, abort_score, B.sp, B.bias, rowbuf, strip,
                            B.tg.trace + (size_t)slot_item * B.tg.slot_bytes,
                            B.tg.meta + (size_t)slot_item * B.tg.meta_stride, g, gmask, end, cells);
    if (g == 0) {
      B.ends[item] = end;
      if (B.cells) atomicAdd(B.cells, (unsigned long long)cells);
    }
    if (!B.work) item += ngroups;
  }
  if (g == 0) bulk_copies_done();  // the trace copies this lane issued
}

// One warp per item (warp_walk over the trace of shape <G, K>, packed or int32);
// lane 0 writes the item's result row.
constexpr uint32_t kTbStageBytes = 4096;  // per warp: metadata + read + window of a walk

template <int G, int K, bool PACKED>
__global__ void __launch_bounds__(128) bsw_tb_kernel(DevPairs P, BswLaunch B) {
  __shared__ uint32_t tb_stage[PACKED ? 4 : 1][PACKED ? kTbStageBytes / 4 : 1];
  uint32_t lo, count;
  bsw_range(B, lo, count);
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  const bool lead = (threadIdx.x & 31u) == 0u;
  for (uint32_t item = lo + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       item < count; item += warps) {
    const uint32_t pair = B.list ? B.list[item] : item;
    const DpEnd e = B.ends[item];
    int32_t i = e.end_i, j = e.end_j;
    uint32_t overflow = 0;
    const uint32_t slot_item = item - B.item_lo;
    const uint8_t* tr = B.tg.trace + (size_t)slot_item * B.tg.slot_bytes;
    const uint32_t* mt = B.tg.meta + (size_t)slot_item * B.tg.meta_stride;
    uint32_t* ops = B.cig_slots + (size_t)item * B.slot_cap;
    uint32_t n = 0;
    const bool outside = e.early_abort == kEndOutsideShape;  // uniform over the warp
    if (outside) {
      i = j = 0;
    } else if constexpr (PACKED) {
      // The walk's row metadata, read and window go to this warp's shared-memory
      // strip when they fit (one coalesced pass), so each round of the walk waits on
      // one global load (its codes) instead of a metadata load and then the codes.
      const uint32_t q = P.read_len[pair], w = P.win_len[pair];
      const uint8_t* rd = P.read_seq + P.read_off[pair];
      const uint8_t* wn = P.win_seq + P.win_off[pair];
      if (4u * (q + 1u) + q + w <= kTbStageBytes) {
        uint32_t* smeta = tb_stage[threadIdx.x >> 5];
        uint8_t* sseq = reinterpret_cast<uint8_t*>(smeta + q + 1u);
        const uint32_t ln = threadIdx.x & 31u;
        for (uint32_t t = ln; t <= q; t += 32u) smeta[t] = __ldg(mt + t);
        for (uint32_t t = ln; t < q; t += 32u) sseq[t] = __ldg(rd + t);
        for (uint32_t t = ln; t < w; t += 32u) sseq[q + t] = __ldg(wn + t);
        __syncwarp();
        n = warp_walk_scored(Bsw16Code<G, K, true>{tr, smeta, B.sp.gap_open}, i, j, e.score,
                             sseq, sseq + q, B.sp, ops, B.slot_cap, overflow);
        __syncwarp();
      } else {
        n = warp_walk_scored(Bsw16Code<G, K>{tr, mt, B.sp.gap_open}, i, j, e.score, rd, wn,
                             B.sp, ops, B.slot_cap, overflow);
      }
    } else {
      n = warp_walk(BswCode<G, K>{tr, mt}, i, j, ops, B.slot_cap, overflow);
    }
    if (!lead) continue;
    kira_sw_result r;
    r.score = e.score;
    r.ref_start = (uint32_t)j;
    r.ref_end = (uint32_t)e.end_j;
    r.read_start = i;
    r.read_end = e.end_i;
    r.cigar_off = 0;
    r.n_cigar = n;
    r.status = outside ? KIRA_PAIR_OUT_OF_BOUNDS : KIRA_PAIR_SW;
    r.early_abort = outside ? 0 : (uint8_t)e.early_abort;
    r.reserved = overflow ? 1 : 0;
    B.out[pair] = r;
    B.ncig[pair] = n;
    B.item_of_pair[pair] = B.item_base + item;
    if (overflow) atomicOr(B.flags, 1u);
  }
}

// Full-window group abort rule of sw_batch_avx2_inner (mod.rs:2058-2081): after
// each row a lane with an active bound is done once best + remaining * match <
// abort; the batch stops after the first row where every lane of the group is
// done. Pass 1 finds each item's first firing row from its per-row keys.
__global__ void __launch_bounds__(128) bsw_full_done_kernel(DevPairs P, BswLaunch B) {
  const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= B.count) return;
  const uint32_t q = P.read_len[item];
  const int32_t abort_score = P.abort_score ? P.abort_score[item] : kAbortOff;
  uint32_t done = 0xFFFFFFFFu;
  if (abort_score > kAbortOff) {
    const uint32_t* keys = B.rowkeys + (size_t)item * B.tg.meta_stride;
    int32_t best = 0;
    for (uint32_t i = 1; i <= q; ++i) {
      best = max(best, (int32_t)(keys[i] >> kKeyIdxBits));
      if (best + (int32_t)(q - i) * B.sp.match < abort_score) {
        done = i;
        break;
      }
    }
  }
  B.done_row[item] = done;
}

// Pass 2: the group's stop row R (max of the members' firing rows, if all fire),
// then best / end / early flag as of row R with the clip rule (mod.rs:2104-2132).
__global__ void __launch_bounds__(128) bsw_full_resolve_kernel(DevPairs P, BswLaunch B) {
  const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= B.count) return;
  const uint32_t g0 = (item / B.group) * B.group;
  const uint32_t g1 = min(g0 + B.group, B.count);
  uint32_t stop = 0;
  for (uint32_t t = g0; t < g1; ++t) stop = max(stop, B.done_row[t]);
  const uint32_t q = P.read_len[item];
  const uint32_t last = stop == 0xFFFFFFFFu ? q : min(stop, q);
  const uint32_t* keys = B.rowkeys + (size_t)item * B.tg.meta_stride;
  int32_t best = 0, bi = 0, bj = 0;
  for (uint32_t i = 1; i <= last; ++i) {
    const int32_t rb = (int32_t)(keys[i] >> kKeyIdxBits);
    if (rb > best) {
      best = rb;
      bi = (int32_t)i;
      bj = 1 + (1023 - (int32_t)(keys[i] & 1023u));
    }
  }
  if (last == q && q > 0) {
    const int32_t bq = (int32_t)(keys[q] >> kKeyIdxBits);
    const int32_t bqj = 1 + (1023 - (int32_t)(keys[q] & 1023u));
    if (bq > 0 && sat_add(bq, B.sp.clip) > best) {
      best = bq;
      bi = (int32_t)q;
      bj = bqj;
    }
  }
  B.ends[item] = DpEnd{best, bi, bj, B.done_row[item] <= last ? 1u : 0u};
}

// ---------------------------------------------------------------------------
// Exclusive scan of per-pair CIGAR counts and compaction into the output array.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanChunk = kScanThreads * kScanPerThread;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh,
                                                         uint32_t& total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, x, off);
    if ((int)lane >= off) x += t;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = blockDim.x >> 5;
    uint32_t y = lane < nw ? sh[lane] : 0u;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, y, off);
      if ((int)lane >= off) y += t;
    }
    if (lane < nw) sh[lane] = y;
  }
  __syncthreads();
  const uint32_t warp_prefix = warp ? sh[warp - 1] : 0u;
  total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_chunk_sums(const uint32_t* __restrict__ v,
                                                                uint32_t n,
                                                                uint32_t* __restrict__ sums) {
  __shared__ uint32_t sh[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanPerThread;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k)
    if (base + k < n) s += v[base + k];
  uint32_t total;
  block_exclusive_scan(s, sh, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// With `accumulate` the scan continues from *total_out (ops already placed by
// earlier chunks of the same batch) and leaves the running total there.
__global__ void __launch_bounds__(kScanThreads) scan_sums(uint32_t* __restrict__ sums,
                                                          uint32_t nchunks,
                                                          uint64_t* __restrict__ total_out,
                                                          int accumulate) {
  __shared__ uint32_t sh[32];
  uint32_t carry = accumulate && total_out ? (uint32_t)*total_out : 0u;
  __syncthreads();
  for (uint32_t base = 0; base < nchunks; base += kScanThreads) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < nchunks ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, sh, total);
    if (i < nchunks) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply(const uint32_t* __restrict__ v,
                                                           uint32_t n,
                                                           const uint32_t* __restrict__ sums,
                                                           uint32_t* __restrict__ off) {
  __shared__ uint32_t sh[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanPerThread;
  uint32_t vals[kScanPerThread];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    vals[k] = base + k < n ? v[base + k] : 0u;
    s += vals[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, sh, total) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    if (base + k < n) off[base + k] = ex;
    ex += vals[k];
  }
}

// Writes cigar_off into the results and the ops into the packed output.
__global__ void __launch_bounds__(256) cigar_compact_kernel(CompactLaunch C) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < C.n; p += stride) {
    const uint32_t off = C.off[p];
    const uint32_t n = C.ncig[p];
    kira_sw_result* r = C.out + p;
    r->cigar_off = off;
    if ((uint64_t)off + n > C.cap) continue;
    if (r->status == KIRA_PAIR_CERTIFIED) {
      C.ops[off] = ((uint32_t)r->read_end << 4) | 0u;
    } else if (r->status == KIRA_PAIR_SW) {
      const uint32_t* src = C.slots + (size_t)C.item_of_pair[p] * C.slot_cap;
      for (uint32_t t = 0; t < n; ++t) C.ops[off + t] = src[n - 1u - t];
    }
  }
}

// NM / MD:Z of every pair's alignment, one thread per pair (nmmd.cuh). Pass 1
// (write = 0) stores NM and the MD length, pass 2 the MD bytes at their offsets.
__global__ void __launch_bounds__(128) nmmd_kernel(DevPairs P, NmMdLaunch L, int write) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < L.n; p += stride) {
    const kira_sw_result r = L.res[p];
    uint32_t nm = 0xFFFFFFFFu, len = 0;
    if (r.n_cigar) {
      if ((uint64_t)r.cigar_off + r.n_cigar > L.n_ops || r.read_start < 0) {
        if (!write) atomicOr(L.flags, 1u);
      } else {
        len = nmmd_walk(P.read_seq + P.read_off[p], P.read_len[p], P.win_seq + P.win_off[p],
                        P.win_len[p], (uint32_t)r.read_start, r.ref_start, L.ops + r.cigar_off,
                        r.n_cigar, nm, write ? L.md + L.off[p] : nullptr);
      }
    }
    if (!write) {
      L.nm[p] = nm;
      L.len[p] = len;
    }
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
// Kernels launched by this library in this process (graph replays add the
// kernels of the replayed graph); read by kira_gpu_launch_count.
static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

static int grid_for(uint64_t units, int per_block, int max_blocks) {
  uint64_t b = (units + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > (uint64_t)max_blocks) b = max_blocks;
  return (int)b;
}

cudaError_t launch_sieve_dropin(const SieveJobsDev& J, kira_sieve_result* out, int sms,
                                cudaStream_t st) {
  const int blocks = grid_for(J.n, 8, sms * 16);
  (sieve_dropin_kernel<<<blocks, 256, 0, st>>>(J, out), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_pack_planes(const uint8_t* seq, uint64_t len, uint4* out, uint64_t nblocks,
                               int sms, cudaStream_t st) {
  const int blocks = grid_for((nblocks + 15) / 16, 8, sms * 16);
  (pack_planes_kernel<<<blocks, 256, 0, st>>>(seq, len, out, nblocks), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_unpack_pairs(const PackedPair* src, uint32_t n, uint64_t* read_off,
                                uint32_t* read_len, uint64_t* win_off, uint32_t* win_len,
                                bool lens, int sms, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int blocks = grid_for(n, 256, sms * 8);
  (unpack_pairs_kernel<<<blocks, 256, 0, st>>>(src, n, read_off, read_len, win_off, win_len,
                                                lens ? 1 : 0),
   count_launch());
  return cudaGetLastError();
}

cudaError_t launch_verify_sieve(const DevPairs& P, const VerifyDev& V, uint32_t max_q, int sms,
                                cudaStream_t st) {
  const int blocks = grid_for(P.n, 256, sms * 8);
  const uint32_t rw = (max_q + 31) / 32;
  if (V.sieve_list && !V.detail && V.qgram && P.n < 0x80000000u) {
    cudaError_t e = cudaMemsetAsync(V.sieve_count, 0, 4, st);
    if (e != cudaSuccess) return e;
    (verify_filter_kernel<<<blocks, 256, 0, st>>>(P, V), count_launch());
    if (rw <= 5) (verify_sieve_list_kernel<5><<<blocks, 256, 0, st>>>(P, V), count_launch());
    else if (rw <= 8) (verify_sieve_list_kernel<8><<<blocks, 256, 0, st>>>(P, V), count_launch());
    else (verify_sieve_list_kernel<16><<<blocks, 256, 0, st>>>(P, V), count_launch());
    return cudaGetLastError();
  }
  if (rw <= 5) (verify_sieve_kernel<5><<<blocks, 256, 0, st>>>(P, V), count_launch());
  else if (rw <= 8) (verify_sieve_kernel<8><<<blocks, 256, 0, st>>>(P, V), count_launch());
  else (verify_sieve_kernel<16><<<blocks, 256, 0, st>>>(P, V), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_myers(const DevPairs& P, const MyersLaunch& M, uint32_t max_items, int sms,
                         cudaStream_t st) {
  const size_t smem = (size_t)4 * M.lmax * 160 * sizeof(uint32_t);
  const int blocks = grid_for(max_items, 128, sms * 8);
  if (M.lmax <= 5) (myers_kernel<5><<<blocks, 128, smem, st>>>(P, M), count_launch());
  else if (M.lmax <= 8) (myers_kernel<8><<<blocks, 128, smem, st>>>(P, M), count_launch());
  else if (M.lmax <= 12) (myers_kernel<12><<<blocks, 128, smem, st>>>(P, M), count_launch());
  else (myers_kernel<16><<<blocks, 128, smem, st>>>(P, M), count_launch());
  return cudaGetLastError();
}

template <int G, int K, int T, int MINB>
static cudaError_t launch_bsw_shape(const DevPairs& P, const BswLaunch& B, uint32_t max_items,
                                    int sms, cudaStream_t st, cudaEvent_t between, int parts) {
  cudaError_t e = cudaSuccess;
  if (parts & kBswPartDp) {
    constexpr int threads = T;
    const size_t smem = (size_t)(threads / 32) * 2 * K * 32 * sizeof(int32_t);
    auto kern = B.full ? bsw_dp_kernel<G, K, T, MINB, true> : bsw_dp_kernel<G, K, T, MINB, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1) per_sm = 1;
    const int blocks = grid_for(max_items, threads / G, sms * per_sm);
    (kern<<<blocks, threads, smem, st>>>(P, B), count_launch());
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (B.full && B.rowkeys) {
      const int rb = (int)((B.count + 127) / 128);
      (bsw_full_done_kernel<<<rb, 128, 0, st>>>(P, B), count_launch());
      (bsw_full_resolve_kernel<<<rb, 128, 0, st>>>(P, B), count_launch());
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
  }
  if (between) cudaEventRecord(between, st);
  if (parts & kBswPartTb) {
    const int tb_blocks = grid_for(max_items, 4, sms * 16);  // a warp per item
    (bsw_tb_kernel<G, K, false><<<tb_blocks, 128, 0, st>>>(P, B), count_launch());
    e = cudaGetLastError();
  }
  return e;
}

template <int G, int K, int T, int MINB>
static cudaError_t launch_bsw16_shape(const DevPairs& P, const BswLaunch& B, uint32_t max_items,
                                      int sms, cudaStream_t st, cudaEvent_t between, int parts) {
  cudaError_t e = cudaSuccess;
  if (parts & kBswPartDp) {
    // per group: a trace strip of kStripBytes and 4 * G * K halves
    const size_t smem = (size_t)(T / G) * Bsw16Shape<G, K>::kStripBytes + (size_t)T * 8u * K;
    auto kern = bsw16_dp_kernel<G, K, T, MINB>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T, smem);
    if (per_sm < 1) per_sm = 1;
    const int blocks = grid_for(max_items, T / G, sms * per_sm);
    (kern<<<blocks, T, smem, st>>>(P, B), count_launch());
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (between) cudaEventRecord(between, st);
  if (parts & kBswPartTb) {
    const int tb_blocks = grid_for(max_items, 4, sms * 16);  // a warp per item
    (bsw_tb_kernel<G, K, true><<<tb_blocks, 128, 0, st>>>(P, B), count_launch());
    e = cudaGetLastError();
  }
  return e;
}

// Launch shapes (lanes per pair, cells per lane, threads per block, min resident
// blocks per SM). The host picks the first shape whose G*K covers 2*band+1
// unless a tuned choice is installed for the band (autotuner / override).
const BswShapeInfo kBswShapes[] = {
    {4, 10, 256, 2, 0},  {4, 17, 128, 4, 0},  {4, 17, 128, 3, 0}, {8, 10, 256, 2, 0},
    {8, 17, 128, 3, 0},  {16, 17, 128, 3, 0}, {32, 17, 128, 3, 0},
    // packed int16: K words = 2K cells per lane
    {2, 9, 256, 2, 1},   {4, 5, 256, 2, 1},   {4, 9, 256, 2, 1},  {8, 5, 256, 2, 1},
    {8, 9, 256, 2, 1},   {16, 9, 256, 2, 1},  {32, 9, 256, 2, 1}, {2, 17, 128, 3, 1},
    {2, 18, 128, 3, 1},
    // the same packed sweeps held to more resident blocks (fewer registers, some spilled)
    {4, 9, 256, 3, 1},   {2, 17, 128, 4, 1},
    // 34 words a lane: one lane per pair (no cross-lane exchange, a row's scalar
    // work done once), and 2 / 4 lanes for bands up to 67 / 135
    {1, 34, 128, 2, 1},  {2, 34, 128, 2, 1},  {4, 34, 128, 2, 1},
    // one lane per pair in smaller blocks (a block's SMs free up at a finer grain
    // at the end of a launch)
    {1, 34, 64, 4, 1},   {1, 34, 32, 8, 1},
};
const int kNumBswShapes = sizeof(kBswShapes) / sizeof(kBswShapes[0]);

cudaError_t launch_bsw(int shape, const DevPairs& P, const BswLaunch& B, uint32_t max_items,
                       int sms, cudaStream_t st, cudaEvent_t between, int parts) {
  switch (shape) {
    case 0: return launch_bsw_shape<4, 10, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 1: return launch_bsw_shape<4, 17, 128, 4>(P, B, max_items, sms, st, between, parts);
    case 2: return launch_bsw_shape<4, 17, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 3: return launch_bsw_shape<8, 10, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 4: return launch_bsw_shape<8, 17, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 5: return launch_bsw_shape<16, 17, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 6: return launch_bsw_shape<32, 17, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 7: return launch_bsw16_shape<2, 9, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 8: return launch_bsw16_shape<4, 5, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 9: return launch_bsw16_shape<4, 9, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 10: return launch_bsw16_shape<8, 5, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 11: return launch_bsw16_shape<8, 9, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 12: return launch_bsw16_shape<16, 9, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 13: return launch_bsw16_shape<32, 9, 256, 2>(P, B, max_items, sms, st, between, parts);
    case 14: return launch_bsw16_shape<2, 17, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 15: return launch_bsw16_shape<2, 18, 128, 3>(P, B, max_items, sms, st, between, parts);
    case 16: return launch_bsw16_shape<4, 9, 256, 3>(P, B, max_items, sms, st, between, parts);
    case 17: return launch_bsw16_shape<2, 17, 128, 4>(P, B, max_items, sms, st, between, parts);
    case 18: return launch_bsw16_shape<1, 34, 128, 2>(P, B, max_items, sms, st, between, parts);
    case 19: return launch_bsw16_shape<2, 34, 128, 2>(P, B, max_items, sms, st, between, parts);
    case 20: return launch_bsw16_shape<4, 34, 128, 2>(P, B, max_items, sms, st, between, parts);
    case 21: return launch_bsw16_shape<1, 34, 64, 4>(P, B, max_items, sms, st, between, parts);
    case 22: return launch_bsw16_shape<1, 34, 32, 8>(P, B, max_items, sms, st, between, parts);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_cigar_scan(const uint32_t* ncig, uint32_t n, uint32_t* off, uint32_t* chunk_sums,
                              uint64_t* total_dev, cudaStream_t st, bool accumulate) {
  const uint32_t chunks = (n + kScanChunk - 1) / kScanChunk;
  if (chunks == 0) return cudaSuccess;
  (scan_chunk_sums<<<chunks, kScanThreads, 0, st>>>(ncig, n, chunk_sums), count_launch());
  (scan_sums<<<1, kScanThreads, 0, st>>>(chunk_sums, chunks, total_dev, accumulate ? 1 : 0), count_launch());
  (scan_apply<<<chunks, kScanThreads, 0, st>>>(ncig, n, chunk_sums, off), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_nm_md(const DevPairs& P, const NmMdLaunch& L, bool write, int sms,
                         cudaStream_t st) {
  const int blocks = grid_for(L.n, 128, sms * 16);
  (nmmd_kernel<<<blocks, 128, 0, st>>>(P, L, write ? 1 : 0), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_cigar_compact(const CompactLaunch& C, int sms, cudaStream_t st) {
  const int blocks = grid_for(C.n, 256, sms * 8);
  (cigar_compact_kernel<<<blocks, 256, 0, st>>>(C), count_launch());
  return cudaGetLastError();
}

// Compact result form: one status byte per pair and a keep flag (1 for a pair
// with an alignment: certified or banded SW).
__global__ void __launch_bounds__(256) status_keep_kernel(const kira_sw_result* __restrict__ rows,
                                                          uint32_t n, uint8_t* __restrict__ status,
                                                          uint32_t* __restrict__ keep) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    const uint8_t s = rows[p].status;
    status[p] = s;
    keep[p] = (s == KIRA_PAIR_CERTIFIED || s == KIRA_PAIR_SW) ? 1u : 0u;
  }
}

// Kept rows to their exclusive-scan slots (pair order); slots at or past cap skipped.
__global__ void __launch_bounds__(256) compact_rows_kernel(const kira_sw_result* __restrict__ rows,
                                                           uint32_t n, const uint32_t* __restrict__ keep,
                                                           const uint32_t* __restrict__ off,
                                                           kira_sw_result* __restrict__ dst,
                                                           uint64_t cap) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
    if (keep[p] && off[p] < cap) dst[off[p]] = rows[p];
}

cudaError_t launch_status_keep(const kira_sw_result* rows, uint32_t n, uint8_t* status,
                               uint32_t* keep, int sms, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int blocks = grid_for(n, 256, sms * 8);
  (status_keep_kernel<<<blocks, 256, 0, st>>>(rows, n, status, keep), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_compact_rows(const kira_sw_result* rows, uint32_t n, const uint32_t* keep,
                                const uint32_t* off, kira_sw_result* dst, uint64_t cap, int sms,
                                cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int blocks = grid_for(n, 256, sms * 8);
  (compact_rows_kernel<<<blocks, 256, 0, st>>>(rows, n, keep, off, dst, cap), count_launch());
  return cudaGetLastError();
}

}  // namespace kira

extern "C" uint64_t kira_gpu_launch_count(void) { return kira::launch_count(); }

// ---------------------------------------------------------------------------
// Integer issue-rate probe (the denominator of the DP kernels' integer roofline).
// Every thread updates 16 independent packed words per round: OP 0 the DPX
// add-max (__viaddmax_s16x2), OP 1 a three-input add, OP 2 a three-input logic
// op, OP 3 an integer multiply-add by one (the add form of the FMA pipe), OP 4
// alternating logic op and multiply-add, OP 5 alternating DPX add-max and
// multiply-add (the mixed forms show which kinds issue to separate pipes). The
// result is folded into a sink that is written only on an impossible value, which
// keeps every round live.
// ---------------------------------------------------------------------------
namespace kira {

template <int OP>
__global__ void __launch_bounds__(256) alu_probe_kernel(uint32_t rounds, uint32_t seed,
                                                        uint32_t* sink) {
  uint32_t x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = seed * (threadIdx.x + 977u * k + 31u * blockIdx.x + 1u);
  uint32_t y = seed ^ threadIdx.x;
  for (uint32_t r = 0; r < rounds; ++r) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint32_t nb = x[(k + 1) & 15];
      const int kind = OP < 3 ? OP : OP == 3 ? 3 : (k & 1) ? 3 : (OP == 4 ? 2 : 0);
      if (kind == 0) {
        x[k] = __viaddmax_s16x2(x[k], y, nb);
      } else if (kind == 1) {
        x[k] = x[k] + nb + y;
      } else if (kind == 2) {
        x[k] = (x[k] & nb) ^ y;
      } else {
        uint32_t r;
        asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(nb), "r"(y | 1u), "r"(x[k]));
        x[k] = r;
      }
    }
    y += 0x00010001u;
  }
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) acc ^= x[k];
  if (acc == 0x9E3779B9u) sink[0] = acc;
}

}  // namespace kira

extern "C" int kira_gpu_alu_probe(int device, int op, uint32_t rounds, double* thread_ops_per_s) {
  using namespace kira;
  if (!thread_ops_per_s || op < 0 || op > 5 || rounds == 0) return KIRA_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return KIRA_ERR_NO_DEVICE;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return KIRA_ERR_RUNTIME;
  uint32_t* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t st = nullptr;
  int rc = KIRA_OK;
  if (cudaMalloc(&sink, 16) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess ||
      cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    rc = KIRA_ERR_RUNTIME;
  } else {
    const int blocks = sms * 8, threads = 256;
    auto launch = [&](uint32_t n) {
      const uint32_t seed = 0x2545F491u;
      if (op == 0) alu_probe_kernel<0><<<blocks, threads, 0, st>>>(n, seed, sink);
      else if (op == 1) alu_probe_kernel<1><<<blocks, threads, 0, st>>>(n, seed, sink);
      else if (op == 2) alu_probe_kernel<2><<<blocks, threads, 0, st>>>(n, seed, sink);
      else if (op == 3) alu_probe_kernel<3><<<blocks, threads, 0, st>>>(n, seed, sink);
      else if (op == 4) alu_probe_kernel<4><<<blocks, threads, 0, st>>>(n, seed, sink);
      else alu_probe_kernel<5><<<blocks, threads, 0, st>>>(n, seed, sink);
      count_launch();
    };
    launch(rounds / 8 + 1);  // warm-up (clocks up, module loaded)
    cudaEventRecord(e0, st);
    launch(rounds);
    cudaEventRecord(e1, st);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
        cudaGetLastError() != cudaSuccess || ms <= 0.f) {
      rc = KIRA_ERR_RUNTIME;
    } else {
      *thread_ops_per_s = (double)blocks * threads * 16.0 * rounds / (ms * 1e-3);
    }
  }
  if (st) cudaStreamDestroy(st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  return rc;
}
