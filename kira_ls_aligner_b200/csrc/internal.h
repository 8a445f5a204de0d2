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

struct BswShapeInfo {
  int g, k, threads, min_blocks;
};
extern const BswShapeInfo kBswShapes[];
extern const int kNumBswShapes;

cudaError_t launch_sieve_dropin(const SieveJobsDev& J, kira_sieve_result* out, int sms,
                                cudaStream_t st);
cudaError_t launch_pack_planes(const uint8_t* seq, uint64_t len, uint4* out, uint64_t nblocks,
                               int sms, cudaStream_t st);
inline uint64_t plane_blocks(uint64_t len) { return (len + 31) / 32 + 4; }
cudaError_t launch_verify_sieve(const DevPairs& P, const VerifyDev& V, uint32_t max_q, int sms,
                                cudaStream_t st);
cudaError_t launch_myers(const DevPairs& P, const MyersLaunch& M, uint32_t max_items, int sms,
                         cudaStream_t st);
cudaError_t launch_bsw(int shape, const DevPairs& P, const BswLaunch& B, uint32_t max_items,
                       int sms, cudaStream_t st, cudaEvent_t between = nullptr);
cudaError_t launch_cigar_scan(const uint32_t* ncig, uint32_t n, uint32_t* off,
                              uint32_t* chunk_sums, uint64_t* total_dev, cudaStream_t st);
cudaError_t launch_cigar_compact(const CompactLaunch& C, int sms, cudaStream_t st);

}  // namespace kira
