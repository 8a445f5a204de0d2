// prefilter.cu -- the ungapped extension prefilter (src/alignment/prefilter.rs:93-517)
// and the exact-match fast path (src/alignment/mod.rs:779-832), one warp per chain.
//
// The reference compares 32-byte blocks with count_mismatches and walks them with
// an x-drop on each side of the anchor; here the 32 lanes of a warp load one
// block (a coalesced 32-byte read of the read and of the reference), and one
// ballot + popc is the block's mismatch count, so every block of the walk, the
// span's Hamming count and the exact-match test cost a handful of warp
// instructions. MD:Z and NM of accepted spans (MdBuilder::columns, md.rs:77-96)
// are built the same way: a ballot marks the mismatching columns of 32, each
// mismatch lane derives its run length from the previous set bit, and a warp
// scan of the token lengths places its digits and reference letter. Pass 1
// decides, counts NM and sizes the CIGAR and MD; pass 2 writes them at the
// offsets the scans assign.
#include <cuda_runtime.h>

#include "internal.h"

namespace kira {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t pf_lower(uint32_t c) { return (c >= 'A' && c <= 'Z') ? c + 32u : c; }

__device__ __forceinline__ uint32_t pf_digits(uint32_t v) {
  uint32_t d = 1;
  while (v >= 10u) v /= 10u, ++d;
  return d;
}

__device__ __forceinline__ void pf_put(char* out, uint32_t v, uint32_t d) {
  for (uint32_t i = 0; i < d; ++i) {
    out[d - 1 - i] = (char)('0' + v % 10u);
    v /= 10u;
  }
}

// Mismatching bytes of a[0, len) and b[0, len) (kira-simd count_mismatches).
__device__ __forceinline__ uint32_t pf_count(const uint8_t* a, const uint8_t* b, uint32_t len,
                                             int lane) {
  uint32_t c = 0;
  for (uint32_t base = 0; base < len; base += 32) {
    const uint32_t i = base + (uint32_t)lane;
    const bool ne = i < len && __ldg(a + i) != __ldg(b + i);
    c += __popc(__ballot_sync(kFull, ne));
  }
  return c;
}

// One side of ungapped_extend (prefilter.rs:356-453): returns the extension.
__device__ uint32_t pf_extend_side(const uint8_t* read, const uint8_t* ref, const kira_chain& c,
                                   uint32_t maxe, bool left, const PrefilterLaunch& L, int lane) {
  int32_t score = 0, best = 0;
  uint32_t i = 0, ext = 0;
  bool broke = false;
  while (i + 32u <= maxe) {
    const uint32_t ro = left ? c.read_start - i - 32u : c.read_end + i;
    const uint32_t fo = left ? c.ref_start - i - 32u : c.ref_end + i;
    const int32_t mism = (int32_t)__popc(
        __ballot_sync(kFull, __ldg(read + ro + lane) != __ldg(ref + fo + lane)));
    score += (32 - mism) * L.match - mism * L.mismatch;
    if (score > best) {
      best = score;
      ext = i + 32u;
    } else if (best - score > L.xdrop) {
      broke = true;
      break;
    }
    i += 32u;
  }
  if (L.tail && !broke && i < maxe) {
    const uint32_t rem = maxe - i;
    const uint32_t ro = left ? c.read_start - i - rem : c.read_end + i;
    const uint32_t fo = left ? c.ref_start - i - rem : c.ref_end + i;
    const bool ne = (uint32_t)lane < rem && __ldg(read + ro + lane) != __ldg(ref + fo + lane);
    const int32_t mism = (int32_t)__popc(__ballot_sync(kFull, ne));
    score += ((int32_t)rem - mism) * L.match - mism * L.mismatch;
    if (score > best) ext = i + rem;
  }
  return ext;
}

// MdBuilder::columns over read[rs, rs + span) x ref[fs, fs + span): returns the
// MD length and NM; with `out` set, writes the text there.
__device__ uint32_t pf_md(const uint8_t* read, const uint8_t* ref, uint32_t rs, uint32_t fs,
                          uint32_t span, char* out, uint32_t& nm_out, int lane) {
  uint32_t wpos = 0, nm = 0;
  int last = -1;  // span index of the previous mismatching column
  for (uint32_t base = 0; base < span; base += 32) {
    const uint32_t i = base + (uint32_t)lane;
    const bool valid = i < span;
    const uint32_t q = valid ? __ldg(read + rs + i) : 0u;
    const uint32_t r = valid ? __ldg(ref + fs + i) : 0u;
    const bool match = q == '=' || pf_lower(q) == pf_lower(r);
    const uint32_t u = (q >= 'a' && q <= 'z') ? q - 32u : q;
    const bool edit = valid && match && !(u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == '=');
    const bool mm = valid && !match;
    const unsigned bm = __ballot_sync(kFull, mm);
    nm += __popc(bm) + __popc(__ballot_sync(kFull, edit));
    uint32_t tok = 0, run = 0;
    if (mm) {
      const unsigned below = bm & ((1u << lane) - 1u);
      const int prev = below ? (int)base + (31 - __clz(below)) : last;
      run = (uint32_t)((int)i - prev - 1);
      tok = pf_digits(run) + 1u;
    }
    if (!out) {  // sizing: the sum of the token lengths is enough
      wpos += __reduce_add_sync(kFull, tok);
    } else {
      uint32_t inc = tok;  // inclusive warp scan of the token lengths places each token
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
      }
      if (mm) {
        const uint32_t at = wpos + inc - tok;
        const uint32_t d = tok - 1u;
        pf_put(out + at, run, d);
        out[at + d] = (char)(((r >= 'A' && r <= 'Z') || (r >= 'a' && r <= 'z')) ? (r & 0xDFu) : 'N');
      }
      wpos += __shfl_sync(kFull, inc, 31);
    }
    if (bm) last = (int)base + (31 - __clz(bm));
  }
  const uint32_t tail = (uint32_t)((int)span - last - 1);
  const uint32_t d = pf_digits(tail);
  if (out && lane == 0) pf_put(out + wpos, tail, d);
  nm_out = nm;
  return wpos + d;
}

__global__ void __launch_bounds__(256) prefilter_kernel(DevPairs P, PrefilterLaunch L, int write) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < P.n; p += warps) {
    const uint8_t* read = P.read_seq + P.read_off[p];
    const uint8_t* ref = P.win_seq + P.win_off[p];
    const uint32_t rl = P.read_len[p], fl = P.win_len[p];
    const kira_chain c = L.chains[p];
    if (write) {
      const kira_prefilter_result r = L.out[p];
      if (r.n_cigar == 0) continue;
      if ((uint64_t)r.md_off + r.md_len > L.md_cap ||
          (uint64_t)r.cigar_off + r.n_cigar > L.cigar_cap)
        continue;  // the call reports the capacity it needs
      uint32_t nm;
      pf_md(read, ref, r.read_start, r.ref_start, r.len, L.md + r.md_off, nm, lane);
      if (lane == 0) {
        uint32_t* ops = L.ops + r.cigar_off;
        uint32_t k = 0;
        if (r.read_start > 0) ops[k++] = (r.read_start << 4) | 4u;
        ops[k++] = ((uint32_t)r.len << 4) | 0u;
        if (r.read_start + r.len < rl) ops[k++] = ((rl - r.read_start - r.len) << 4) | 4u;
      }
      continue;
    }
    kira_prefilter_result res{};
    bool aligned = false;  // accept or exact: span read_start / ref_start / len
    if (L.exact_first) {
      // exact_match_alignment (mod.rs:779-815) with exact_match_exists (mod.rs:819-832)
      const bool shape = c.read_start == 0 && c.read_end == rl && c.ref_end >= c.ref_start &&
                         c.ref_end - c.ref_start == rl && (uint64_t)c.ref_start + rl <= fl;
      if (shape && pf_count(read, ref + c.ref_start, rl, lane) == 0) {
        res.result = KIRA_PREFILTER_EXACT;
        res.len = (uint16_t)rl;
        res.score = L.match * (int32_t)rl;
        res.read_start = 0;
        res.ref_start = c.ref_start;
        aligned = true;
      }
    }
    if (!aligned) {
      const uint32_t anchor = c.read_end - c.read_start;
      auto other = [&](uint8_t code) {
        res.result = KIRA_PREFILTER_FALLBACK;
        res.reason = 9;
        res.other = code;
      };
      if (rl == 0) {
        other(1);
      } else if (c.read_start > c.read_end || c.ref_start > c.ref_end) {
        other(2);
      } else if (anchor == 0) {
        other(3);
      } else if (c.read_end > rl || c.ref_end > fl) {
        if (lane == 0) atomicOr(L.flags, 1u);  // the host validates; never reached
        other(6);
      } else {
        const uint32_t max_left = min(c.read_start, c.ref_start);
        const uint32_t max_right = min(rl - c.read_end, fl - c.ref_end);
        const uint32_t left = pf_extend_side(read, ref, c, max_left, true, L, lane);
        const uint32_t right = pf_extend_side(read, ref, c, max_right, false, L, lane);
        const uint32_t total = anchor + left + right;
        const uint32_t urs = c.read_start - left, ufs = c.ref_start - left;
        if (total == 0) {
          other(4);
        } else if (urs + total > rl || ufs + total > fl) {
          other(6);
        } else {
          const uint32_t ham = pf_count(read + urs, ref + ufs, total, lane);
          const int32_t score =
              (int32_t)(total - min(ham, total)) * L.match - (int32_t)ham * L.mismatch;
          const uint16_t len16 = (uint16_t)min(total, 65535u);
          const uint16_t mism16 = (uint16_t)min(min(ham, total), 65535u);
          // identity_x10000 (prefilter.rs:84-91)
          const uint64_t matches = total > ham ? total - ham : 0;
          const uint64_t prod = min(matches * (uint64_t)10000, (uint64_t)UINT32_MAX);
          const uint16_t id = (uint16_t)min(prod / total, (uint64_t)65535);
          res.has_metrics = 1;
          res.len = len16;
          res.mism = mism16;
          res.matches = len16 > mism16 ? (uint16_t)(len16 - mism16) : 0;
          res.identity_x10000 = id;
          res.score = score;
          res.read_start = urs;
          res.ref_start = ufs;
          // The decision cascade of prefilter_chain (prefilter.rs:187-294).
          const uint8_t top1 = L.is_top1 ? L.is_top1[p] : 1;
          const int32_t margin = L.score_margin ? L.score_margin[p] : INT32_MAX;
          uint32_t slack = 0;  // min_len_required (prefilter.rs:297-315)
          if (id >= 9933) slack = 15;
          else if (id >= 9900 && ham <= 2) slack = 10;
          else if (id >= 9870 && ham <= 3) slack = 5;
          if (L.span_slack > 0) slack = min(slack, L.span_slack);
          const uint32_t min_len = max(rl * 85u / 100u, rl > slack ? rl - slack : 0u);
          const uint32_t hard_max = (rl * 5u + 149u) / 150u;
          res.result = KIRA_PREFILTER_FALLBACK;
          if (total < rl / 2) res.result = KIRA_PREFILTER_REJECT, res.reason = 5;
          else if (!L.accept_enable) res.reason = 1;
          else if (L.multi) res.reason = 4;
          else if (L.only_top1 && !top1) res.reason = 3;
          else if (rl > L.long_read_threshold) res.reason = 2;
          else if (L.require_margin > 0 && margin < L.require_margin) res.reason = 9, res.other = 7;
          else if (c.ref_end - c.ref_start != c.read_end - c.read_start) res.reason = 8;
          else if (ham > min(L.max_mismatches, hard_max)) res.reason = 6;
          else if ((int32_t)id < L.identity_floor) res.reason = 7;
          else if (total < min_len) res.reason = 5;
          else res.result = KIRA_PREFILTER_ACCEPT, res.reason = 0, aligned = true;
        }
      }
    }
    if (aligned) {
      // build_ungapped_alignment (prefilter.rs:455-517): [S] M [S]; span = len (u16).
      const uint32_t span = res.len, re = res.read_start + span;
      res.n_cigar = 1u + (res.read_start > 0 ? 1u : 0u) + (re < rl ? 1u : 0u);
      uint32_t nm;
      res.md_len = pf_md(read, ref, res.read_start, res.ref_start, span, nullptr, nm, lane);
      res.nm = nm;
    }
    if (lane == 0) {
      L.out[p] = res;
      L.ncig[p] = res.n_cigar;
      L.mdlen[p] = res.md_len;
    }
  }
}

// Writes cigar_off / md_off from the scans into the results.
__global__ void __launch_bounds__(256) prefilter_offsets_kernel(uint32_t n,
                                                                kira_prefilter_result* out,
                                                                const uint32_t* cig_off,
                                                                const uint32_t* md_off) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    out[p].cigar_off = cig_off[p];
    out[p].md_off = md_off[p];
  }
}

// exact_match_exists (mod.rs:819-832) per chain.
__global__ void __launch_bounds__(256) exact_match_kernel(DevPairs P, const kira_chain* chains,
                                                          uint8_t* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < P.n; p += warps) {
    const kira_chain c = chains[p];
    const uint32_t rl = P.read_len[p], fl = P.win_len[p];
    const bool shape = c.read_start == 0 && c.read_end == rl && c.ref_end >= c.ref_start &&
                       c.ref_end - c.ref_start == rl && (uint64_t)c.ref_start + rl <= fl;
    uint8_t v = 0;
    if (shape)
      v = pf_count(P.read_seq + P.read_off[p], P.win_seq + P.win_off[p] + c.ref_start, rl, lane) == 0;
    if (lane == 0) out[p] = v;
  }
}

int pf_grid(uint32_t n, int sms) {
  uint64_t b = ((uint64_t)n + 7) / 8;
  if (b < 1) b = 1;
  if (b > (uint64_t)sms * 16) b = (uint64_t)sms * 16;
  return (int)b;
}

}  // namespace

cudaError_t launch_prefilter(const DevPairs& P, const PrefilterLaunch& L, bool write, int sms,
                             cudaStream_t st) {
  (prefilter_kernel<<<pf_grid(P.n, sms), 256, 0, st>>>(P, L, write ? 1 : 0), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_prefilter_offsets(uint32_t n, kira_prefilter_result* out,
                                     const uint32_t* cig_off, const uint32_t* md_off, int sms,
                                     cudaStream_t st) {
  uint64_t b = ((uint64_t)n + 255) / 256;
  if (b < 1) b = 1;
  if (b > (uint64_t)sms * 8) b = (uint64_t)sms * 8;
  (prefilter_offsets_kernel<<<(int)b, 256, 0, st>>>(n, out, cig_off, md_off), count_launch());
  return cudaGetLastError();
}

cudaError_t launch_exact_match(const DevPairs& P, const kira_chain* chains, uint8_t* out, int sms,
                               cudaStream_t st) {
  (exact_match_kernel<<<pf_grid(P.n, sms), 256, 0, st>>>(P, chains, out), count_launch());
  return cudaGetLastError();
}

}  // namespace kira
