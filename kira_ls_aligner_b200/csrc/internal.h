// internal.h -- host/device launch descriptors shared by kernels.cu and api.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace kira {

// Packed sieve jobs (the CudaJob drop-in) in device memory.
struct SieveJobsDev {
  uint32_t n;
  const uint8_t* read_bits;
  const uint64_t* read_off;
  const uint32_t* read_nucs;
  const uint8_t* ref_bits;
  const uint64_t* ref_off;
  const uint32_t* ref_nucs;
  const uint32_t* max_mism;
};

// Stage 1 (sieve + certificate) of the composed path.
struct VerifyDev {
  int32_t sieve_threshold;
  int32_t cert_strict;
  SwParams sw;
  kira_sw_result* out;
  kira_verify_detail* detail;  // may be null
  uint32_t* ncig;
  int32_t* sw_offset;
  uint32_t* myers_list;
  uint32_t* counters;          // [0] myers items, [1] sw items
  int32_t myers_k;             // < 0: router bound per read (myers_k_for)
  int32_t qgram;               // exact 4-gram prefilter before Myers (qgram.cuh)
  // Filter-first form (no detail rows, filter on): pairs the 4-gram count does not
  // settle, as pair | 1 << 31 when the count already rejects them unless they
  // certify; *sieve_count entries. Null: one kernel sieves every pair.
  uint32_t* sieve_list;
  uint32_t* sieve_count;
};

struct MyersLaunch {
  const uint32_t* list;       // null: identity over [0, count)
  const uint32_t* count_dev;  // null: use count
  uint32_t count;
  int32_t k;                  // per_pair_k: k < 0 -> router bound per read
  int32_t per_pair_k;
  uint32_t tw;                // text plane words per pair in shared memory
  uint32_t lmax;              // Peq limbs reserved per lane in shared memory
  int32_t cascade;
  // direct outputs
  int32_t* dist;
  int32_t* end;
  // cascade outputs
  kira_sw_result* out;
  kira_verify_detail* detail;
  uint32_t* ncig;
  uint32_t* sw_list;
  uint32_t* counters;
  uint32_t* flags;            // bit 2: pattern longer than the kernel supports
  // Banded-SW items of several calls gathered into one list: its count word (null:
  // counters[1]) and the batch index of this call's pair 0 (added to each entry).
  uint32_t* sw_count;
  uint32_t sw_base;
};

struct BswLaunch {
  const uint32_t* list;       // null: identity
  const uint32_t* count_dev;  // null: use count
  uint32_t count;
  SwParams sp;
  const int32_t* offset;      // per pair band offset (null -> 0)
  TraceGeom tg;
  DpEnd* ends;                // per item
  unsigned long long* cells;  // optional total
  uint32_t* cig_slots;        // per item slot_cap ops (reversed order)
  uint32_t slot_cap;
  kira_sw_result* out;        // per pair
  uint32_t* ncig;             // per pair
  uint32_t* item_of_pair;     // per pair
  uint32_t* flags;            // bit 0: CIGAR slot overflow, bit 1: item outside the launch shape
  uint32_t max_q;             // rows per trace slot - 1
  // full-window mode (align_batch_simd): per-row keys for the group abort rule
  int32_t full;
  uint32_t* rowkeys;          // [item][max_q + 1] or null when no abort bound is active
  uint32_t* done_row;         // [item] first row whose abort test fired (0xFFFFFFFF: never)
  uint32_t group;             // lanes per SIMD batch (16: AVX2 i16, 32: AVX-VNNI i8)
  // bucketed launches
  uint32_t* work;             // dynamic work counter (null: static grid-stride order)
  uint32_t item_base;         // global index of this launch's first item (CIGAR slots)
  int32_t bias;               // packed int16 shapes: value bias (packed_bias)
  // Trace round: this launch handles items [item_lo, item_hi) (item_hi 0: no
  // bound); trace slots and row metadata are indexed by item - item_lo, every
  // other per-item array by the item itself.
  uint32_t item_lo, item_hi;
  // 1 / 2: the first / second half of the item count (device-side), for the two
  // halves of a one-round batch run on two streams at once; 0: the round above.
  uint32_t split;
};

struct CompactLaunch {
  uint32_t n;
  kira_sw_result* out;
  const uint32_t* ncig;
  const uint32_t* off;
  const uint32_t* item_of_pair;
  const uint32_t* slots;
  uint32_t slot_cap;
  uint32_t* ops;
  uint64_t cap;
};

// NM / MD:Z pass over a batch's results (nmmd.cuh).
struct NmMdLaunch {
  uint32_t n;
  const kira_sw_result* res;  // per pair, from the alignment call
  const uint32_t* ops;        // that call's CIGAR ops
  uint64_t n_ops;
  uint32_t* nm;               // pass 1 out: NM (0xFFFFFFFF: no alignment)
  uint32_t* len;              // pass 1 out: MD length
  const uint32_t* off;        // pass 2 in: MD offset of each pair
  char* md;                   // pass 2 out
  uint32_t* flags;            // bit 0: a result's CIGAR range lies outside the ops
};

// WFA batch (wfa.cuh / wfa.cu): warp per pair over a per-warp history.
struct WfaLaunch {
  uint32_t n;
  int32_t valid;               // 0: the scored costs were refused (every pair None)
  int32_t x, o, ei, ed;        // WfaCosts (wfa.rs:22-52)
  int32_t lookback;            // max(x, o + ei, o + ed)
  int32_t scored, match;       // scored: score = read_len * match - cost
  int32_t max_score;           // < 0 (and no per-pair array): router budget per read
  int32_t budget_pct, budget_x, budget_o, budget_e;  // router::wfa_score_budget arguments
  const int32_t* max_score_pp; // per pair (may be null)
  int32_t tbf;                 // text_begin_free
  const int32_t* tbf_pp;       // per pair (may be null)
  int32_t drop;                // adaptive drop; < 0: exact
  int32_t group;               // lanes per pair: 8, 16 or 32
  uint8_t* scratch;            // per group: meta (traceback), global meta ring, history
  uint64_t group_bytes;
  uint32_t hist_off;           // byte offset of the history in a group's scratch
  uint32_t meta_slots;         // traceback: scores held in the global meta (S + 1)
  uint32_t hist_cap;           // traceback: int16 history entries per group
  uint32_t ring_len;           // scores in the meta ring (and the score-only history ring)
  uint32_t ring_width;         // score-only: entries per layer per ring slot; 0: traceback
  uint32_t ring_bytes;         // shared bytes of the meta ring per group; 0: ring in scratch
  uint32_t ring_goff;          // byte offset of the meta ring in scratch when not shared
  uint32_t pat_region;         // shared bytes per group before the text (pattern + guards)
  uint32_t smem_group;         // shared bytes per group
  uint32_t* work;              // dynamic pair counter
  kira_wfa_result* out;
  uint32_t* ncig;              // traceback: ops per pair
  uint32_t* slots;             // traceback: slot_cap ops per pair, newest first
  uint32_t slot_cap;
  uint32_t* flags;             // bit 0: CIGAR slot overflow, bit 1: history overflow
  // General kernel over a pair list (the window kernel's fallbacks): pair list[q]
  // for q < *list_count; null: every pair of [0, n).
  const uint32_t* list;
  const uint32_t* list_count;
  // Window kernel (wfa_window_kernel): 32 x win_segments diagonals from win_base
  // per pair, exact for every pair done by score win_smax; later pairs are
  // appended to fb_list for the general kernel.
  int32_t win_base, win_smax, win_segments;
  uint32_t win_ring_bytes;     // shared bytes of the score ring per warp
  uint32_t* fb_list;
  uint32_t* fb_count;
  int16_t* win_hist;           // traceback: per warp (win_smax + 1) x 3 x window offsets
};

struct WfaCompact {
  uint32_t n;
  kira_wfa_result* out;
  const uint32_t* ncig;
  const uint32_t* off;
  const uint32_t* slots;
  uint32_t slot_cap;
  uint32_t* ops;
  uint64_t cap;
};

// Ungapped prefilter (prefilter.cu): warp per chain.
struct PrefilterLaunch {
  const kira_chain* chains;
  const uint8_t* is_top1;       // may be null: every chain is the top one
  const int32_t* score_margin;  // may be null: INT32_MAX
  int32_t match, mismatch, xdrop;
  int32_t accept_enable, only_top1, multi, tail, exact_first;
  uint32_t span_slack, max_mismatches, long_read_threshold;
  int32_t require_margin, identity_floor;
  kira_prefilter_result* out;
  uint32_t* ncig;               // pass 1: CIGAR ops per chain
  uint32_t* mdlen;              // pass 1: MD bytes per chain
  uint32_t* ops;                // pass 2: CIGAR output
  uint64_t cigar_cap;
  char* md;                     // pass 2: MD output
  uint64_t md_cap;              // pass 2: chains whose CIGAR or MD would pass a cap are skipped
  uint32_t* flags;              // bit 0: a chain outside its read / window
};

// Banded-SW launch shape: G lanes per pair, K cells (int32) or K packed words of
// two int16 cells (packed) per lane.
struct BswShapeInfo {
  int g, k, threads, min_blocks, packed;
};
extern const BswShapeInfo kBswShapes[];
extern const int kNumBswShapes;

inline int shape_cap(const BswShapeInfo& s) { return (s.packed ? 2 : 1) * s.g * s.k; }
inline uint32_t shape_lane_bytes(const BswShapeInfo& s) {
  // packed: a 4-bit code per cell, four words (eight cells) per 4-byte slab;
  // int32: a 4-bit code per cell, eight cells per 4 bytes.
  return s.packed ? 4u * (uint32_t)((s.k + 3) / 4) : 4u * (uint32_t)((s.k + 7) / 8);
}
inline uint32_t shape_row_stride(const BswShapeInfo& s) {
  return (uint32_t)s.g * shape_lane_bytes(s);
}
// Rows per interleave block of the packed trace (Bsw16Shape::kInterleave).
inline uint32_t shape_row_interleave(const BswShapeInfo& s) {
  if (!s.packed) return 1u;
  return s.g == 1 ? 8u : s.g < 32 ? 32u / (uint32_t)s.g : 1u;
}
// Bytes of one item's trace slot for reads of up to `max_q` bases: rows 0..max_q
// rounded up to whole interleave blocks, then to 16 bytes.
inline uint64_t shape_slot_bytes(const BswShapeInfo& s, uint32_t max_q) {
  const uint64_t r = shape_row_interleave(s);
  const uint64_t rows = ((uint64_t)max_q + 1 + r - 1) / r * r;
  return (rows * shape_row_stride(s) + 15) & ~15ull;
}
inline TraceGeom shape_trace_geom(const BswShapeInfo& s, uint8_t* trace, uint32_t* meta,
                                  uint64_t slot_bytes, uint32_t meta_stride) {
  return TraceGeom{trace, meta, slot_bytes, shape_row_stride(s), shape_lane_bytes(s),
                   (uint32_t)s.k, meta_stride, s.packed ? (uint32_t)(s.g * s.k) : 0u};
}

// Bias of the packed int16 sweep: every biased DP value is >= 0 (F at the far
// end of a row included) and the first cell's F sentinel stays below H = 0.
inline int32_t packed_bias(const BswShapeInfo& s, const SwParams& sp) {
  return sp.gof + shape_cap(s) * sp.gap_extend + sp.mismatch + 1;
}

// Bits of the word index in the packed sweep's row-max keys (Bsw16Shape::kKeyBits).
inline int packed_key_bits(int k) {
  return k <= 2 ? 1 : k <= 4 ? 2 : k <= 8 ? 3 : k <= 16 ? 4 : k <= 32 ? 5 : 6;
}

// The packed sweep is exact when every biased value stays below 2^13, every
// difference its flags test stays below 2^11 (the F-extend flag at bit 11), and
// every biased H fits a row-max key (H << key bits below 2^16).
inline bool packed_fits(const BswShapeInfo& s, uint32_t max_q, const SwParams& sp) {
  if (!s.packed) return false;
  if (sp.match < 0 || sp.mismatch < 0 || sp.gap_open < 0 || sp.gap_extend < 0) return false;
  const int64_t top = (int64_t)max_q * sp.match;
  const int64_t cap = shape_cap(s);
  if (top + cap * sp.gap_extend + sp.gof >= 2048) return false;
  if (top + (int64_t)packed_bias(s, sp) >= (int64_t(1) << (16 - packed_key_bits(s.k))))
    return false;
  return top + (int64_t)packed_bias(s, sp) + cap * sp.gap_extend < 8192;
}

cudaError_t launch_sieve_dropin(const SieveJobsDev& J, kira_sieve_result* out, int sms,
                                cudaStream_t st);
cudaError_t launch_pack_planes(const uint8_t* seq, uint64_t len, uint4* out, uint64_t nblocks,
                               int sms, cudaStream_t st);
inline uint64_t plane_blocks(uint64_t len) { return (len + 31) / 32 + 4; }
// Pair descriptors as the chunked host path uploads them when the read arena and
// the window source are below 4 GiB (every checked offset then fits 32 bits).
struct PackedPair {
  uint32_t read_off, win_off;
  uint16_t read_len, win_len;
};
static_assert(sizeof(PackedPair) == 12, "PackedPair layout");

// Expands n packed descriptors into the pipeline's arrays; with lens == false the
// length arrays are left as they are (uploaded separately).
cudaError_t launch_unpack_pairs(const PackedPair* src, uint32_t n, uint64_t* read_off,
                                uint32_t* read_len, uint64_t* win_off, uint32_t* win_len,
                                bool lens, int sms, cudaStream_t st);
cudaError_t launch_verify_sieve(const DevPairs& P, const VerifyDev& V, uint32_t max_q, int sms,
                                cudaStream_t st);
cudaError_t launch_myers(const DevPairs& P, const MyersLaunch& M, uint32_t max_items, int sms,
                         cudaStream_t st);
// Banded SW: the DP sweep (kBswPartDp) and/or the traceback (kBswPartTb); an
// event given as `between` is recorded after the DP part.
constexpr int kBswPartDp = 1, kBswPartTb = 2;
cudaError_t launch_bsw(int shape, const DevPairs& P, const BswLaunch& B, uint32_t max_items,
                       int sms, cudaStream_t st, cudaEvent_t between = nullptr,
                       int parts = kBswPartDp | kBswPartTb);
cudaError_t launch_cigar_scan(const uint32_t* ncig, uint32_t n, uint32_t* off,
                              uint32_t* chunk_sums, uint64_t* total_dev, cudaStream_t st,
                              bool accumulate = false);
cudaError_t launch_cigar_compact(const CompactLaunch& C, int sms, cudaStream_t st);
// Compact result form of the composed path: status bytes + keep flags, then the
// kept rows at their scan offsets (kira_gpu_verify_batch_compact).
cudaError_t launch_status_keep(const kira_sw_result* rows, uint32_t n, uint8_t* status,
                               uint32_t* keep, int sms, cudaStream_t st);
cudaError_t launch_compact_rows(const kira_sw_result* rows, uint32_t n, const uint32_t* keep,
                                const uint32_t* off, kira_sw_result* dst, uint64_t cap, int sms,
                                cudaStream_t st);
cudaError_t launch_nm_md(const DevPairs& P, const NmMdLaunch& L, bool write, int sms,
                         cudaStream_t st);

cudaError_t wfa_blocks_per_sm(int group, bool traceback, size_t smem, int threads, int* per_sm);
cudaError_t wfa_window_blocks_per_sm(int segments, bool traceback, size_t smem, int* per_sm);
cudaError_t launch_wfa_window(const DevPairs& P, const WfaLaunch& L, uint32_t blocks,
                              bool traceback, cudaStream_t st);
cudaError_t launch_wfa(const DevPairs& P, const WfaLaunch& L, uint32_t blocks,
                       uint32_t warps_per_block, bool traceback, cudaStream_t st);
cudaError_t launch_wfa_compact(const WfaCompact& C, int sms, cudaStream_t st);

cudaError_t launch_prefilter(const DevPairs& P, const PrefilterLaunch& L, bool write, int sms,
                             cudaStream_t st);
cudaError_t launch_prefilter_offsets(uint32_t n, kira_prefilter_result* out,
                                     const uint32_t* cig_off, const uint32_t* md_off, int sms,
                                     cudaStream_t st);
cudaError_t launch_exact_match(const DevPairs& P, const kira_chain* chains, uint8_t* out, int sms,
                               cudaStream_t st);

int ctx_share_reference(kira_ctx* dst, const kira_ctx* src);

// Launch accounting (kernels.cu): every kernel launch of the library adds one.
void count_launch(unsigned long long k = 1);
unsigned long long launch_count();

// Why a banded-SW configuration is outside the supported domain (null: inside).
const char* sw_cfg_problem(const kira_sw_cfg& c, uint32_t max_q, uint32_t max_band);

}  // namespace kira
