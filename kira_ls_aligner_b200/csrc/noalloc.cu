// noalloc.cu -- banded SW for callers that must not allocate device memory.
//
// kira_gpu_bsw_batch_noalloc runs the same kernels as kira_gpu_bsw_batch (DP
// sweep, traceback, CIGAR scan and compaction) but takes every input and output
// as a device pointer from the caller and keeps all of its scratch (trace arena,
// row metadata, per-item ends, CIGAR slots, scan buffers, flags) in one
// file-scope device array of KIRA_NOALLOC_SCRATCH_BYTES. It calls no cudaMalloc,
// cudaFree or allocating library routine, and creates no context object.
//
// Host code cannot use `g_noalloc_scratch` as a device address (in host code the
// name is a host-side stand-in), so the device address is fetched with
// cudaGetSymbolAddress once per device, with that device current, on the first
// call made on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "internal.h"
#include "kira_gpu.h"

namespace kira {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[KIRA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_dev[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_dev[dev] = p;
  }
  *out = g_scratch_dev[dev];
  return cudaSuccess;
}

// Carves the fixed scratch into the stage buffers; false when it does not fit.
struct Carve {
  unsigned char* base;
  uint64_t used, limit;
  template <class T>
  T* take(uint64_t count) {
    const uint64_t at = (used + 255) & ~uint64_t(255);
    const uint64_t bytes = count * sizeof(T);
    if (at + bytes > limit) {
      used = limit + 1;
      return nullptr;
    }
    used = at + bytes;
    return reinterpret_cast<T*>(base + at);
  }
};

}  // namespace
}  // namespace kira

using namespace kira;

extern "C" int kira_gpu_bsw_batch_noalloc(const kira_pairs* pairs, const kira_sw_cfg* cfg,
                                          kira_sw_result* out, uint32_t* cigar_ops,
                                          uint64_t cigar_cap, uint64_t* cigar_used,
                                          void* stream) {
  if (!pairs || !cfg || !out || !cigar_used) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  if (P.n == 0) return KIRA_OK;
  if (!P.max_read_len || !P.max_win_len || !P.read_seq || !P.win_seq)
    return KIRA_ERR_INVALID;
  const kira_sw_cfg& c = *cfg;
  const uint32_t max_q = P.max_read_len, max_w = P.max_win_len;
  const uint32_t max_band = P.bandwidth ? P.max_bandwidth : (uint32_t)std::max(c.bandwidth, 1);
  if (max_band == 0) return KIRA_ERR_INVALID;
  // Same domain as kira_gpu_bsw_batch (one shared check).
  if (sw_cfg_problem(c, max_q, max_band)) return KIRA_ERR_INVALID;
  const int need = 2 * (int)max_band + 1;
  int shape = -1;
  for (int s = 0; s < kNumBswShapes; ++s)
    if (!kBswShapes[s].packed && shape_cap(kBswShapes[s]) >= need) {
      shape = s;
      break;
    }
  if (shape < 0) return KIRA_ERR_INVALID;

  void* sp = nullptr;
  if (scratch_address(&sp) != cudaSuccess) return KIRA_ERR_RUNTIME;
  const uint32_t n = P.n;
  const BswShapeInfo sh = kBswShapes[shape];
  const uint64_t slot = shape_slot_bytes(sh, max_q);
  const uint32_t meta_stride = max_q + 1;
  const uint32_t slot_cap = max_q + max_w + 2;
  Carve cv{static_cast<unsigned char*>(sp), 0, KIRA_NOALLOC_SCRATCH_BYTES};
  uint8_t* trace = cv.take<uint8_t>(slot * n);
  uint32_t* meta = cv.take<uint32_t>((uint64_t)meta_stride * n);
  DpEnd* ends = cv.take<DpEnd>(n);
  uint32_t* slots = cv.take<uint32_t>((uint64_t)slot_cap * n);
  uint32_t* ncig = cv.take<uint32_t>(n);
  uint32_t* iop = cv.take<uint32_t>(n);
  uint32_t* off = cv.take<uint32_t>(n);
  uint32_t* sums = cv.take<uint32_t>(n / 4096 + 2);
  uint32_t* counters = cv.take<uint32_t>(4);
  if (cv.used > KIRA_NOALLOC_SCRATCH_BYTES || !counters) return KIRA_ERR_SCRATCH_LIMIT;

  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return KIRA_ERR_RUNTIME;
  // The array keeps the previous call's contents: clear the flags word.
  if (cudaMemsetAsync(counters, 0, 16, st) != cudaSuccess) return KIRA_ERR_RUNTIME;

  DevPairs D{n, P.read_seq, P.read_off, P.read_len, P.win_seq, P.win_off, P.win_len,
             P.band_offset, P.abort_score, P.bandwidth, nullptr, nullptr};
  BswLaunch B{};
  B.count = n;
  SwParams s;
  s.match = c.match_score;
  s.mismatch = c.mismatch;
  s.gap_open = c.gap_open;
  s.gap_extend = c.gap_extend;
  s.band = std::max(c.bandwidth, 1);
  s.dp_xdrop = c.dp_xdrop >= 0 ? c.dp_xdrop : c.xdrop;
  s.clip = c.clip_penalty;
  s.adaptive = c.adaptive ? 1 : 0;
  s.max_drift = std::max(c.max_drift, 0);
  s.gof = c.gap_open + c.gap_extend;
  B.sp = s;
  B.offset = P.band_offset;
  B.tg = shape_trace_geom(sh, trace, meta, slot, meta_stride);
  B.ends = ends;
  B.cells = nullptr;
  B.cig_slots = slots;
  B.slot_cap = slot_cap;
  B.out = out;
  B.ncig = ncig;
  B.item_of_pair = iop;
  B.flags = counters + 2;
  B.max_q = max_q;
  if (launch_bsw(shape, D, B, n, sms, st) != cudaSuccess) return KIRA_ERR_RUNTIME;
  if (launch_cigar_scan(ncig, n, off, sums, cigar_used, st) != cudaSuccess)
    return KIRA_ERR_RUNTIME;
  CompactLaunch C{n, out, ncig, off, iop, slots, slot_cap, cigar_ops, cigar_cap};
  if (launch_cigar_compact(C, sms, st) != cudaSuccess) return KIRA_ERR_RUNTIME;
  return KIRA_OK;
}
