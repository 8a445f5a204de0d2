// common.cuh -- shared device-side types and helpers of libkira_gpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kira_gpu.h"

namespace kira {

constexpr int32_t kNeg4 = INT32_MIN / 4;      // i32::MIN / 4 sentinel (mod.rs:1451-1453)
constexpr int32_t kAbortOff = INT32_MIN / 8;  // i32::MIN / 8: abort bound disabled
constexpr int kKeyIdxBits = 10;               // row argmax key: (h << 10) | (1023 - idx)
constexpr int kMaxBand = 1023;                // 2*band+1 cells must fit the 10-bit index
constexpr int kMaxRowLen = 2 * kMaxBand + 1;
constexpr int kWfaMaxLen = 30000;             // WFA offsets and diagonals fit int16

// Per-pair inputs in device memory (mirrors kira_pairs with device pointers).
struct DevPairs {
  uint32_t n;
  const uint8_t* read_seq;
  const uint64_t* read_off;
  const uint32_t* read_len;
  const uint8_t* win_seq;
  const uint64_t* win_off;
  const uint32_t* win_len;
  const int32_t* band_offset;  // may be null
  const int32_t* abort_score;  // may be null
  const int32_t* bandwidth;    // may be null
  const uint4* read_planes;    // planes of read_seq (sieve / Myers stages)
  const uint4* win_planes;     // planes of win_seq
};

// Banded SW parameters resolved on the host.
struct SwParams {
  int32_t match, mismatch, gap_open, gap_extend, band, dp_xdrop, clip, adaptive, max_drift;
  int32_t gof;  // gap_open saturating+ gap_extend (mod.rs:1483)
};

// Trace arena geometry of one SW launch: item slot s covers
// trace[s * slot_bytes ...] with row r at r * row_stride; lane g of the group
// owns bytes [g * lane_bytes, (g + 1) * lane_bytes) of a row, two cells per byte.
struct TraceGeom {
  uint8_t* trace;
  uint32_t* meta;       // per item: (q_max + 1) words: (row_start << 11) | row_len
  uint64_t slot_bytes;
  uint32_t row_stride;
  uint32_t lane_bytes;
  uint32_t k_cells;     // cells per lane (K); packed shapes: words per lane
  uint32_t meta_stride; // words per item
  uint32_t half;        // packed shapes: cells per half row (G*K); 0: int32 nibble trace
};

// Per-item DP result consumed by the traceback kernel.
struct DpEnd {
  int32_t score;
  int32_t end_i;
  int32_t end_j;
  uint32_t early_abort;  // kEndOutsideShape: the item was not run (outside the launch shape)
};
constexpr uint32_t kEndOutsideShape = 0xFFFFFFFFu;

__device__ __forceinline__ int32_t sat_add(int32_t a, int32_t b) {
  int64_t s = (int64_t)a + (int64_t)b;
  return s > INT32_MAX ? INT32_MAX : (s < INT32_MIN ? INT32_MIN : (int32_t)s);
}

// 2-bit code (A0 C1 G2 T3) with the ACGT-valid flag in bit 2; encode_base and
// is_acgt of bitpacked.rs:12-20,89-91. Arithmetic form of the table: for the
// eight ACGT/acgt bytes ((b >> 1) ^ (b >> 2)) & 3 is the code.
__device__ __forceinline__ uint32_t base_code(uint32_t b) {
  const uint32_t u = b & 0xDFu;  // fold lower case
  const bool valid = (u == 'A') | (u == 'C') | (u == 'G') | (u == 'T');
  const uint32_t code = ((b >> 1) ^ (b >> 2)) & 3u;
  return valid ? (code | 4u) : 0u;
}

// Load byte p of a sequence through the read-only path.
__device__ __forceinline__ uint32_t ldb(const uint8_t* s, uint64_t p) { return __ldg(s + p); }

}  // namespace kira
