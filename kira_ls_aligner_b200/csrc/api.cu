// api.cu -- the extern "C" entry points of libkira_gpu (include/kira_gpu.h).
#if defined(__SSE2__)
#include <emmintrin.h>
#endif
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <future>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "kira_gpu.h"

using namespace kira;

namespace {

enum BufId {
  B_NMMD_RES, B_NMMD_OPS, B_NMMD_NM, B_NMMD_LEN, B_NMMD_OFF, B_NMMD_OUT, B_NMMD_FLAGS,
  B_READ_SEQ, B_WIN_SEQ, B_READ_OFF, B_READ_LEN, B_WIN_OFF, B_WIN_LEN, B_BAND_OFF, B_ABORT,
  B_BANDW, B_OUT, B_DETAIL, B_CIGAR_OUT, B_NCIG, B_CIG_OFF, B_CHUNK_SUMS, B_SW_OFFSET,
  B_MYERS_LIST, B_SW_LIST, B_COUNTERS, B_ENDS, B_TRACE, B_META, B_CIG_SLOTS, B_ITEM_OF_PAIR,
  B_DIST, B_END, B_SIEVE_OUT, B_SIEVE_JOBS, B_CELLS, B_TOTAL, B_READ_PLANES, B_WIN_PLANES,
  B_ROWKEYS, B_DONE_ROW, B_WORK, B_WFA_MAXS, B_WFA_TBF, B_WFA_OUT, B_WFA_NCIG, B_WFA_SLOTS,
  B_WFA_SCRATCH, B_WFA_FLAGS, B_PF_CHAINS, B_PF_TOP1, B_PF_MARGIN, B_PF_OUT, B_PF_NCIG,
  B_PF_MDLEN, B_PF_MDOFF, B_PF_MD, B_PF_EXACT, B_WFA_FB, B_WFA_WHIST, B_SIEVE_LIST, B_PACKED, B_STATUS, B_KEEP, B_ROW_OFF,
  B_ROWS, B_ROW_SUMS, B_ROW_TOTAL, B_SW_GROUPS, B_COUNT
};

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// A packed pair descriptor into pinned staging memory, bypassing the CPU caches
// where the host has streaming stores (x86 SSE2), and the fence that orders them
// before the copy is enqueued.
inline void stage_store(PackedPair* dst, const PackedPair& v) {
#if defined(__SSE2__)
  uint32_t w[3];
  std::memcpy(w, &v, sizeof(w));
  int* d = reinterpret_cast<int*>(dst);
  _mm_stream_si32(d, (int)w[0]);
  _mm_stream_si32(d + 1, (int)w[1]);
  _mm_stream_si32(d + 2, (int)w[2]);
#else
  *dst = v;
#endif
}
inline void stage_fence() {
#if defined(__SSE2__)
  _mm_sfence();
#endif
}

// Host threads a context keeps for its per-pair host checks: run() hands every
// worker the same function once and returns at once; wait() returns when all of
// them finished it.
class HostPool {
 public:
  explicit HostPool(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void run(std::function<void()> fn) {
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = std::move(fn);
      ++gen_;
      busy_ = (int)th_.size();
    }
    cv_.notify_all();
  }
  void wait() {
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [&] { return busy_ == 0; });
  }

 private:
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        f = job_;
      }
      f();
      std::lock_guard<std::mutex> g(mu_);
      if (--busy_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::function<void()> job_;
  uint64_t gen_ = 0;
  int busy_ = 0;
  bool stop_ = false;
};

}  // namespace

constexpr int kStages = 5;  // sieve+certificate, Myers, SW DP, SW traceback, CIGAR compaction

constexpr int kBandClasses = 6;  // tuned-shape table: band <= 16, 33, 64, 128, 256, 511

inline int band_class(uint32_t b) {
  return b <= 16 ? 0 : b <= 33 ? 1 : b <= 64 ? 2 : b <= 128 ? 3 : b <= 256 ? 4 : 5;
}

struct kira_ctx {
  int device = 0;
  int tuned_shape[kBandClasses] = {-1, -1, -1, -1, -1, -1};
  bool plain = false;  // single-launch banded SW (no bucketing): the comparison baseline
  uint64_t trace_budget = 0;  // bytes for trace slots + row metadata (0: from free HBM)
  bool graphs = false;        // replay the bucketed banded-SW launches from a CUDA graph
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uint8_t> graph_key;  // launch parameters the cached graph was captured with
  uint64_t graph_replays = 0, graph_captures = 0;
  unsigned long long graph_kernels = 0;  // kernels in the cached graph (launch accounting)
  uint32_t last_rounds = 0;              // trace rounds of the last kira_gpu_bsw_batch
  cudaStream_t aux = nullptr;            // second half of a split banded-SW stage
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Bucketed banded SW: one stream per band class (DP then traceback), forked from
  // and joined back into the context's stream.
  cudaStream_t cls_st[kBandClasses] = {};
  cudaEvent_t ev_cls_fork = nullptr, ev_cls_join[kBandClasses] = {};
  cudaStream_t h2d = nullptr, d2h = nullptr;   // copy streams of the chunked host path
  int64_t chunk_pairs = -1;                    // chunked host path: -1 auto, 0 off, else pairs
  int wfa_lanes = 0;                           // WFA lanes per pair: 0 auto, else 8 / 16 / 32
  std::vector<cudaEvent_t> ev_up, ev_comp;     // per chunk: inputs landed / results ready
  int sms = 148;
  cudaStream_t stream = nullptr;
  std::string last_error;
  bool profile = false;
  cudaEvent_t ev[kStages + 1] = {};
  int ev_recorded = 0;
  uint8_t* ref_dev = nullptr;
  uint4* ref_planes = nullptr;  // 2-bit + valid planes of the resident reference
  uint64_t ref_len = 0;
  std::shared_ptr<void> ref_owner;  // frees ref_dev / ref_planes with the last holder
  std::unique_ptr<HostPool> pool;   // host threads of the chunked path's pair checks
  kira_ctx* twin = nullptr;          // second compute stream + scratch of the chunked path
  std::vector<cudaEvent_t> ev_pack, ev_scan;  // per chunk: planes packed / CIGARs placed
  PackedPair* stage = nullptr;  // pinned: packed descriptors of the chunked host path
  uint64_t stage_cap = 0;       // pairs
  DevBuf bufs[B_COUNT];
};

namespace {

int fail(kira_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return code;
}

int cuda_fail(kira_ctx* ctx, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? KIRA_ERR_OOM : KIRA_ERR_RUNTIME;
  return fail(ctx, code, "%s: %s", what, cudaGetErrorString(e));
}

// Grow-only device buffer (ensure_capacity_*, src/cuda/backend.rs:271-308);
// 16 bytes of slack so vector loads may read to the next 16-byte boundary. Growth
// is stream-ordered on the context's stream (cudaMallocAsync / cudaFreeAsync from
// the device's pool), so it never synchronises other contexts' streams; a buffer
// grows by at least a quarter to keep regrowth rare.
void* dbuf(kira_ctx* ctx, BufId id, size_t bytes, cudaError_t* err) {
  DevBuf& b = ctx->bufs[id];
  const size_t need = bytes + 16;
  if (b.bytes >= need) return b.p;
  const size_t cap = std::max(need, b.bytes + b.bytes / 4);
  if (b.p) cudaFreeAsync(b.p, ctx->stream);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMallocAsync(&b.p, cap, ctx->stream);
  if (e != cudaSuccess) {
    *err = e;
    b.p = nullptr;
    return nullptr;
  }
  b.bytes = cap;
  return b.p;
}

#define KIRA_DBUF(var, type, id, count)                                           \
  type* var = (type*)dbuf(ctx, id, sizeof(type) * (size_t)(count), &cerr);        \
  if (!var) return cuda_fail(ctx, cerr, "device allocation (" #id ")");

#define KIRA_CUDA(call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
  } while (0)

SwParams resolve(const kira_sw_cfg& c) {
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
  const int64_t g = (int64_t)c.gap_open + c.gap_extend;
  s.gof = g > INT32_MAX ? INT32_MAX : (int32_t)g;
  return s;
}

// Domain of the GPU banded SW (exactness conditions of the F prefix scan and of
// the packed row-argmax key).
}  // namespace

// Domain of the banded-SW entry points (exactness of the F scan and of the row
// keys); the reason when `c` is outside it, else null. Shared by every entry
// point that runs the banded SW, so their domains cannot drift apart.
const char* kira::sw_cfg_problem(const kira_sw_cfg& c, uint32_t max_q, uint32_t max_band) {
  if (c.gap_open < 0 || c.gap_extend < 0) return "gap_open and gap_extend must be >= 0";
  if ((int64_t)c.gap_open + c.gap_extend > (1 << 24) || c.gap_extend > (1 << 16))
    return "gap costs above the supported range";
  const int64_t step = std::max<int64_t>({(int64_t)c.match_score, -(int64_t)c.mismatch, 0});
  if ((int64_t)max_q * step >= (1 << 21)) return "read_len * max cell gain must be < 2^21";
  if (std::abs((int64_t)c.match_score) > (1 << 20) || std::abs((int64_t)c.mismatch) > (1 << 20))
    return "match/mismatch above the supported range";
  const int need = 2 * (int)std::max<uint32_t>(max_band, 1) + 1;
  int cap = 0;
  for (int s = 0; s < kNumBswShapes; ++s) cap = std::max(cap, shape_cap(kBswShapes[s]));
  if (need > cap) return "bandwidth above the supported maximum";
  return nullptr;
}

namespace {

int check_sw_cfg(kira_ctx* ctx, const kira_sw_cfg& c, uint32_t max_q, uint32_t max_band) {
  const char* why = sw_cfg_problem(c, max_q, max_band);
  if (why) return fail(ctx, KIRA_ERR_INVALID, "%s (band %u, read %u)", why, max_band, max_q);
  return KIRA_OK;
}

// The int32 shape of the one-launch path: the first whose row covers the band.
int plain_shape(uint32_t max_band) {
  const int need = 2 * (int)std::max<uint32_t>(max_band, 1) + 1;
  for (int s = 0; s < kNumBswShapes; ++s)
    if (!kBswShapes[s].packed && shape_cap(kBswShapes[s]) >= need) return s;
  return -1;
}

bool shape_fits(int s, uint32_t max_band) {
  return s >= 0 && s < kNumBswShapes &&
         shape_cap(kBswShapes[s]) >= 2 * (int)std::max<uint32_t>(max_band, 1) + 1;
}

// A shape can run a batch when its row covers the band and, for a packed int16
// shape, every value of the batch stays inside the exact int16 range.
bool shape_usable(int s, uint32_t max_band, uint32_t max_q, const SwParams& sp) {
  if (!shape_fits(s, max_band)) return false;
  return !kBswShapes[s].packed || packed_fits(kBswShapes[s], max_q, sp);
}

// Default: the first packed shape that covers the band and fits int16, else the
// int32 shape of the one-launch path.
int default_shape(uint32_t max_band, uint32_t max_q, const SwParams& sp) {
  for (int s = 0; s < kNumBswShapes; ++s)
    if (kBswShapes[s].packed && shape_usable(s, max_band, max_q, sp)) return s;
  return plain_shape(max_band);
}

struct Maxes {
  uint32_t q = 0, w = 0, band = 0;
};

HostPool* host_pool(kira_ctx* ctx) {
  if (!ctx->pool) {
    const unsigned hw = std::thread::hardware_concurrency();
    ctx->pool.reset(new HostPool((int)std::min(15u, std::max(2u, hw) - 1u)));
  }
  return ctx->pool.get();
}

// Per-pair host passes (bounds, maxima) read ~24 B per pair, ~3.5 ns per pair on
// one core: batches of more than one part of 2^15 pairs are split over the
// context's host threads and the calling thread. fn(lo, hi, part) fills the
// caller's per-part slot; host_parts(n) slots are needed.
constexpr uint32_t kHostPart = 1u << 15;
inline uint32_t host_parts(uint32_t n) { return std::max<uint32_t>(1, (n + kHostPart - 1) / kHostPart); }

template <class F>
void host_for(kira_ctx* ctx, uint32_t n, F&& fn) {
  const uint32_t parts = host_parts(n);
  if (parts == 1) {
    fn(0u, n, 0u);
    return;
  }
  std::atomic<uint32_t> next{0};
  auto body = [&] {
    for (;;) {
      const uint32_t k = next.fetch_add(1, std::memory_order_relaxed);
      if (k >= parts) return;
      fn(k * kHostPart, std::min(n, (k + 1) * kHostPart), k);
    }
  };
  HostPool* pool = host_pool(ctx);
  pool->run(body);
  body();
  pool->wait();
}

Maxes host_maxes(kira_ctx* ctx, const kira_pairs& P, int32_t cfg_band) {
  std::vector<Maxes> part(host_parts(P.n));
  const uint32_t cb = (uint32_t)std::max(cfg_band, 1);
  host_for(ctx, P.n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    uint32_t q = 0, w = 0, band = P.bandwidth ? 0u : cb;
    for (uint32_t i = lo; i < hi; ++i) {
      q = P.read_len[i] > q ? P.read_len[i] : q;
      w = P.win_len[i] > w ? P.win_len[i] : w;
    }
    if (P.bandwidth)
      for (uint32_t i = lo; i < hi; ++i) band = std::max(band, (uint32_t)std::max(P.bandwidth[i], 1));
    part[k] = Maxes{q, w, band};
  });
  Maxes m;
  for (const Maxes& x : part)
    m.q = std::max(m.q, x.q), m.w = std::max(m.w, x.w), m.band = std::max(m.band, x.band);
  return m;
}

// Copies the host batch into the ctx arena and returns its device view.
int upload_pairs(kira_ctx* ctx, const kira_pairs& P, DevPairs& D) {
  cudaError_t cerr = cudaSuccess;
  cudaStream_t st = ctx->stream;
  const uint32_t n = P.n;
  const uint64_t wlim = P.win_seq ? P.win_seq_bytes : ctx->ref_len;
  std::vector<int64_t> bad(host_parts(n), -1);  // first pair outside its arena, per part
  host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    uint64_t rend = 0, wend = 0;
    for (uint32_t i = lo; i < hi; ++i) {
      const uint64_t re = P.read_off[i] + P.read_len[i], we = P.win_off[i] + P.win_len[i];
      rend = re > rend ? re : rend;
      wend = we > wend ? we : wend;
    }
    if (rend <= P.read_seq_bytes && wend <= wlim) return;
    for (uint32_t i = lo; i < hi; ++i)
      if (P.read_off[i] + P.read_len[i] > P.read_seq_bytes || P.win_off[i] + P.win_len[i] > wlim) {
        bad[k] = i;
        return;
      }
  });
  for (const int64_t i : bad) {
    if (i < 0) continue;
    if (P.read_off[i] + P.read_len[i] > P.read_seq_bytes)
      return fail(ctx, KIRA_ERR_INVALID, "pair %u: read outside read_seq", (uint32_t)i);
    return fail(ctx, KIRA_ERR_INVALID, "pair %u: window outside %s", (uint32_t)i,
                P.win_seq ? "win_seq" : "the resident reference");
  }
  KIRA_DBUF(rs, uint8_t, B_READ_SEQ, P.read_seq_bytes);
  KIRA_CUDA(cudaMemcpyAsync(rs, P.read_seq, P.read_seq_bytes, cudaMemcpyHostToDevice, st));
  const uint8_t* ws = ctx->ref_dev;
  if (P.win_seq) {
    KIRA_DBUF(w, uint8_t, B_WIN_SEQ, P.win_seq_bytes);
    KIRA_CUDA(cudaMemcpyAsync(w, P.win_seq, P.win_seq_bytes, cudaMemcpyHostToDevice, st));
    ws = w;
  }
  KIRA_DBUF(ro, uint64_t, B_READ_OFF, n);
  KIRA_DBUF(rl, uint32_t, B_READ_LEN, n);
  KIRA_DBUF(wo, uint64_t, B_WIN_OFF, n);
  KIRA_DBUF(wl, uint32_t, B_WIN_LEN, n);
  KIRA_CUDA(cudaMemcpyAsync(ro, P.read_off, 8ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(rl, P.read_len, 4ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(wo, P.win_off, 8ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(wl, P.win_len, 4ull * n, cudaMemcpyHostToDevice, st));
  D = DevPairs{n, rs, ro, rl, ws, wo, wl, nullptr, nullptr, nullptr, nullptr, nullptr};
  if (P.band_offset) {
    KIRA_DBUF(b, int32_t, B_BAND_OFF, n);
    KIRA_CUDA(cudaMemcpyAsync(b, P.band_offset, 4ull * n, cudaMemcpyHostToDevice, st));
    D.band_offset = b;
  }
  if (P.abort_score) {
    KIRA_DBUF(b, int32_t, B_ABORT, n);
    KIRA_CUDA(cudaMemcpyAsync(b, P.abort_score, 4ull * n, cudaMemcpyHostToDevice, st));
    D.abort_score = b;
  }
  if (P.bandwidth) {
    KIRA_DBUF(b, int32_t, B_BANDW, n);
    KIRA_CUDA(cudaMemcpyAsync(b, P.bandwidth, 4ull * n, cudaMemcpyHostToDevice, st));
    D.bandwidth = b;
  }
  return KIRA_OK;
}

// Plane arenas of the batch's reads and windows (the resident reference keeps
// the planes built at upload).
int build_planes(kira_ctx* ctx, DevPairs& D, uint64_t read_bytes, uint64_t win_bytes,
                 bool resident, cudaStream_t st) {
  cudaError_t cerr = cudaSuccess;
  const uint64_t rb = plane_blocks(read_bytes);
  KIRA_DBUF(rp, uint4, B_READ_PLANES, rb);
  KIRA_CUDA(launch_pack_planes(D.read_seq, read_bytes, rp, rb, ctx->sms, st));
  D.read_planes = rp;
  if (resident) {
    if (!ctx->ref_planes) return fail(ctx, KIRA_ERR_INVALID, "no resident reference uploaded");
    D.win_planes = ctx->ref_planes;
  } else {
    const uint64_t wb = plane_blocks(win_bytes);
    KIRA_DBUF(wp, uint4, B_WIN_PLANES, wb);
    KIRA_CUDA(launch_pack_planes(D.win_seq, win_bytes, wp, wb, ctx->sms, st));
    D.win_planes = wp;
  }
  return KIRA_OK;
}

// Launch shape of the banded SW stage: the tuned choice for the band class if it
// covers the band, else the smallest shape that does.
int pick_shape(const kira_ctx* ctx, uint32_t max_band, uint32_t max_q, const SwParams& sp) {
  const int t = ctx->tuned_shape[band_class(max_band)];
  return shape_usable(t, max_band, max_q, sp) ? t : default_shape(max_band, max_q, sp);
}

// Bytes the banded-SW trace arena (trace slots + row metadata) may take: the
// context's override, else half of the free device memory plus what the arena
// already holds, between 64 MiB and 64 GiB.
uint64_t trace_budget(kira_ctx* ctx) {
  if (ctx->trace_budget) return ctx->trace_budget;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
  const uint64_t held = ctx->bufs[B_TRACE].bytes + ctx->bufs[B_META].bytes;
  return std::min<uint64_t>(std::max<uint64_t>((fr + held) / 2, 64ull << 20), 64ull << 30);
}

// Trace slot bytes of one item of a shape over reads of up to max_q bases.
uint64_t trace_slot_bytes(int shape, uint32_t max_q) {
  return shape_slot_bytes(kBswShapes[shape], max_q);
}

// True when the trace arena already holds `slot_bytes` of slots and `meta_words`
// of row metadata (no free-memory query is needed then).
bool trace_arena_holds(const kira_ctx* ctx, uint64_t slot_bytes, uint64_t meta_words) {
  return !ctx->trace_budget && ctx->bufs[B_TRACE].bytes >= slot_bytes + 16 &&
         ctx->bufs[B_META].bytes >= 4 * meta_words + 16;
}

// Items one trace round holds (>= 1, <= items).
uint32_t round_items(kira_ctx* ctx, uint32_t items, int shape, uint32_t max_q) {
  const uint64_t slot = trace_slot_bytes(shape, max_q);
  if (trace_arena_holds(ctx, slot * items, (uint64_t)(max_q + 1) * items)) return items;
  const uint64_t per = slot + 4ull * (max_q + 1);
  const uint64_t fit = trace_budget(ctx) / std::max<uint64_t>(per, 1);
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(items, fit));
}

// Scratch of the banded SW stage for up to `items` items, trace slots and row
// metadata for `trace_items` of them (one round).
int prepare_bsw(kira_ctx* ctx, uint32_t n_pairs, uint32_t items, uint32_t trace_items,
                const Maxes& mx, int shape, BswLaunch& B) {
  cudaError_t cerr = cudaSuccess;
  const BswShapeInfo sh = kBswShapes[shape];
  const uint64_t slot = trace_slot_bytes(shape, mx.q);
  const uint32_t meta_stride = mx.q + 1;
  const uint32_t slot_cap = mx.q + mx.w + 2;
  KIRA_DBUF(trace, uint8_t, B_TRACE, slot * std::max<uint32_t>(trace_items, 1));
  KIRA_DBUF(meta, uint32_t, B_META, (uint64_t)meta_stride * std::max<uint32_t>(trace_items, 1));
  KIRA_DBUF(ends, DpEnd, B_ENDS, std::max<uint32_t>(items, 1));
  KIRA_DBUF(slots, uint32_t, B_CIG_SLOTS, (uint64_t)slot_cap * std::max<uint32_t>(items, 1));
  KIRA_DBUF(iop, uint32_t, B_ITEM_OF_PAIR, std::max<uint32_t>(n_pairs, 1));
  B.tg = shape_trace_geom(sh, trace, meta, slot, meta_stride);
  B.ends = ends;
  B.cig_slots = slots;
  B.slot_cap = slot_cap;
  B.item_of_pair = iop;
  B.max_q = mx.q;
  return KIRA_OK;
}

// DP + traceback of `items` items in rounds of `per_round` (trace slots reused);
// `between` (profiling) is recorded after the first round's DP.
// With `work` (dynamic fetch) round r takes its items through counter work[r].
cudaError_t launch_bsw_rounds(int shape, const DevPairs& D, BswLaunch B, uint32_t items,
                              uint32_t per_round, int sms, cudaStream_t st, cudaEvent_t between,
                              uint32_t* work = nullptr) {
  const uint32_t rounds = (items + per_round - 1) / std::max<uint32_t>(per_round, 1);
  for (uint32_t r = 0; r < std::max<uint32_t>(rounds, 1); ++r) {
    B.item_lo = r * per_round;
    B.item_hi = rounds > 1 ? B.item_lo + per_round : 0u;
    B.work = work ? work + r : nullptr;
    cudaError_t e = launch_bsw(shape, D, B, per_round, sms, st, r == 0 ? between : nullptr);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// CIGAR scan + compaction over all pairs; writes the total op count to total_dev.
int finish_cigars(kira_ctx* ctx, uint32_t n, kira_sw_result* out, const uint32_t* ncig,
                  const BswLaunch& B, uint32_t* ops, uint64_t cap, uint64_t* total_dev,
                  cudaStream_t st, bool accumulate = false) {
  cudaError_t cerr = cudaSuccess;
  KIRA_DBUF(off, uint32_t, B_CIG_OFF, std::max<uint32_t>(n, 1));
  KIRA_DBUF(sums, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
  KIRA_CUDA(launch_cigar_scan(ncig, n, off, sums, total_dev, st, accumulate));
  CompactLaunch C{n, out, ncig, off, B.item_of_pair, B.cig_slots, B.slot_cap, ops, cap};
  KIRA_CUDA(launch_cigar_compact(C, ctx->sms, st));
  return KIRA_OK;
}

void mark(kira_ctx* ctx, int i, cudaStream_t st) {
  if (!ctx->profile) return;
  cudaEventRecord(ctx->ev[i], st);
  ctx->ev_recorded = i + 1;
}

// Batches of at least this many pairs split their banded-SW stage over two streams.
constexpr uint32_t kSplitPairs = 1u << 16;

// How one call of the composed path fits into a chunked batch: planes already
// built by the caller, whether the flag word is reset, and whether CIGAR offsets
// continue from the running total in total_dev.
struct ChunkMode {
  bool planes_ready = false;
  bool first = true;
  bool accumulate = false;
  cudaEvent_t before_scan = nullptr;  // the CIGAR scan waits for it (the previous chunk's)
  cudaEvent_t after_scan = nullptr;   // recorded once this chunk's CIGARs are placed
};

// The banded-SW stage of a chunk deferred to a launch over several chunks' items:
// the batch-wide per-pair arrays the front stages write, and the item list (with
// its count word) the Myers stage appends the chunk's SW pairs to as batch indices.
struct DeferSw {
  uint32_t* ncig;   // batch-wide, pair index = base + the chunk's pair
  int32_t* swoff;   // batch-wide band offsets
  uint32_t* slist;  // item list of the chunk's group
  uint32_t* count;  // its count word
  uint32_t base;    // batch index of the chunk's pair 0
};

// The composed path on device buffers, enqueued on `st`. With `df` only the stages
// up to Myers run (sieve, certificate, Myers; the SW pairs are listed in df).
int verify_pipeline(kira_ctx* ctx, DevPairs D, const Maxes& mx, const kira_verify_params& p,
                    uint64_t read_bytes, uint64_t win_bytes, bool resident, kira_sw_result* out,
                    uint32_t* ops, uint64_t cap, uint64_t* total_dev, kira_verify_detail* detail,
                    unsigned long long* cells_dev, cudaStream_t st, ChunkMode cm = ChunkMode(),
                    const DeferSw* df = nullptr) {
  cudaError_t cerr = cudaSuccess;
  const uint32_t n = D.n;
  if (n == 0) return KIRA_OK;
  int rc = check_sw_cfg(ctx, p.sw, mx.q, mx.band);
  if (rc) return rc;
  if (mx.q > 512) return fail(ctx, KIRA_ERR_READ_TOO_LONG, "read of %u bases > 512", mx.q);
  const SwParams sp = resolve(p.sw);
  const int shape = pick_shape(ctx, mx.band, mx.q, sp);
  if (shape < 0) return fail(ctx, KIRA_ERR_INVALID, "no banded-SW shape for band %u", mx.band);
  uint32_t* ncig = df ? df->ncig + df->base : nullptr;
  int32_t* swoff = df ? df->swoff + df->base : nullptr;
  uint32_t* slist = df ? df->slist : nullptr;
  if (!df) {
    KIRA_DBUF(a, uint32_t, B_NCIG, n);
    KIRA_DBUF(b, int32_t, B_SW_OFFSET, n);
    KIRA_DBUF(c, uint32_t, B_SW_LIST, n);
    ncig = a;
    swoff = b;
    slist = c;
  }
  KIRA_DBUF(mlist, uint32_t, B_MYERS_LIST, n);
  KIRA_DBUF(counters, uint32_t, B_COUNTERS, 4);
  KIRA_CUDA(cudaMemsetAsync(counters, 0, cm.first ? 16 : 8, st));
  VerifyDev V{p.sieve_threshold, p.cert_strict, sp,       out,       detail, ncig,
              swoff,             mlist,         counters, p.myers_k, (p.flags & KIRA_VERIFY_NO_QGRAM) ? 0 : 1,
              nullptr,           nullptr};
  if (!detail && V.qgram) {  // filter-first sieve: survivor list after its count word
    KIRA_DBUF(sl, uint32_t, B_SIEVE_LIST, (uint64_t)n + 1);
    V.sieve_count = sl;
    V.sieve_list = sl + 1;
  }
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);
  if (!cm.planes_ready) {
    rc = build_planes(ctx, D, read_bytes, win_bytes, resident, st);
    if (rc) return rc;
  }
  KIRA_CUDA(launch_verify_sieve(D, V, mx.q, ctx->sms, st));
  mark(ctx, 1, st);
  MyersLaunch M{};
  M.list = mlist;
  M.count_dev = counters + 0;
  M.k = p.myers_k;
  M.per_pair_k = 1;
  M.tw = std::max<uint32_t>((mx.w + 31) / 32, 1);
  M.lmax = std::max<uint32_t>((mx.q + 31) / 32, 1);
  M.cascade = 1;
  M.out = out;
  M.detail = detail;
  M.ncig = ncig;
  M.sw_list = slist;
  M.counters = counters;
  M.flags = counters + 2;
  if (df) {
    M.sw_count = df->count;
    M.sw_base = df->base;
  }
  KIRA_CUDA(launch_myers(D, M, n, ctx->sms, st));
  if (df) return KIRA_OK;  // the SW stage runs over the group's items later
  BswLaunch B{};
  const uint32_t per_round = round_items(ctx, n, shape, mx.q);
  rc = prepare_bsw(ctx, n, n, per_round, mx, shape, B);
  mark(ctx, 2, st);
  if (rc) return rc;
  B.list = slist;
  B.count_dev = counters + 1;
  B.sp = sp;
  B.bias = packed_bias(kBswShapes[shape], sp);
  B.offset = swoff;
  B.cells = cells_dev;
  B.out = out;
  B.ncig = ncig;
  B.flags = counters + 2;
  if (per_round >= n && n >= kSplitPairs && !ctx->profile) {
    // One trace round: the two halves of the banded-SW items (split on the device
    // by the Myers stage's count) run on two streams, so one half's DP fills the
    // SMs the other's last wave leaves idle and its traceback overlaps that DP.
    if (!ctx->aux) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking));
    if (!ctx->ev_fork) KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    if (!ctx->ev_join) KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
    KIRA_CUDA(cudaEventRecord(ctx->ev_fork, st));
    KIRA_CUDA(cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
    BswLaunch B1 = B, B2 = B;
    B1.split = 1u;
    B2.split = 2u;
    KIRA_CUDA(launch_bsw(shape, D, B1, n, ctx->sms, st));
    KIRA_CUDA(launch_bsw(shape, D, B2, n, ctx->sms, ctx->aux));
    KIRA_CUDA(cudaEventRecord(ctx->ev_join, ctx->aux));
    KIRA_CUDA(cudaStreamWaitEvent(st, ctx->ev_join, 0));
  } else {
    KIRA_CUDA(launch_bsw_rounds(shape, D, B, n, per_round, ctx->sms, st,
                                ctx->profile ? ctx->ev[3] : nullptr));
  }
  if (ctx->profile) ctx->ev_recorded = 4;
  mark(ctx, 4, st);
  if (cm.before_scan) KIRA_CUDA(cudaStreamWaitEvent(st, cm.before_scan, 0));
  rc = finish_cigars(ctx, n, out, ncig, B, ops, cap, total_dev, st, cm.accumulate);
  if (!rc && cm.after_scan) KIRA_CUDA(cudaEventRecord(cm.after_scan, st));
  mark(ctx, 5, st);
  return rc;
}

// Banded SW over a host batch already uploaded to D: pairs are bucketed by band
// class (each class gets the launch shape tuned for it and a trace geometry sized
// for its longest read), sorted longest-first inside a class, and fetched
// dynamically by the DP kernel's groups. One DP + one traceback launch per class.
// Device launches of one bucketed banded-SW call (everything after the host-side
// ordering and the work-list upload): value-initialised so its bytes are a key.
struct BucketRun {
  int shape[kBandClasses];
  uint32_t cnt[kBandClasses], per_round[kBandClasses];
  uint32_t one_round, nwork;
  uint32_t* work;
  BswLaunch L[kBandClasses];
};

// Enqueues the launches of a planned bucketed call on `st` (capturable).
cudaError_t enqueue_bucketed(kira_ctx* ctx, const DevPairs& D, const BucketRun& R,
                             cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(R.work, 0, 4ull * R.nwork, st);
  if (e != cudaSuccess) return e;
  mark(ctx, 2, st);
  int classes = 0;
  for (int c = 0; c < kBandClasses; ++c) classes += R.cnt[c] ? 1 : 0;
  if (R.one_round && !ctx->profile && classes > 1) {
    // Every class on its own stream, widest first on the context's stream: the
    // classes' DP sweeps fill each other's last partial waves, and each class's
    // traceback overlaps the others' sweeps. (Their trace slots, ends, CIGAR slots
    // and work counters are disjoint.) Stage timing keeps the serial form below.
    if ((e = cudaEventRecord(ctx->ev_cls_fork, st)) != cudaSuccess) return e;
    bool first = true;
    for (int c = kBandClasses - 1; c >= 0; --c) {
      if (!R.cnt[c]) continue;
      cudaStream_t s = first ? st : ctx->cls_st[c];
      if (!first && (e = cudaStreamWaitEvent(s, ctx->ev_cls_fork, 0)) != cudaSuccess) return e;
      if ((e = launch_bsw(R.shape[c], D, R.L[c], R.cnt[c], ctx->sms, s)) != cudaSuccess) return e;
      if (!first && (e = cudaEventRecord(ctx->ev_cls_join[c], s)) != cudaSuccess) return e;
      first = false;
    }
    first = true;
    for (int c = kBandClasses - 1; c >= 0; --c) {
      if (!R.cnt[c]) continue;
      if (!first && (e = cudaStreamWaitEvent(st, ctx->ev_cls_join[c], 0)) != cudaSuccess) return e;
      first = false;
    }
    return cudaSuccess;
  }
  if (R.one_round) {
    // Widest class first (longest rows), then the narrower ones fill in behind it.
    for (int c = kBandClasses - 1; c >= 0; --c)
      if (R.cnt[c] && (e = launch_bsw(R.shape[c], D, R.L[c], R.cnt[c], ctx->sms, st, nullptr,
                                      kBswPartDp)) != cudaSuccess)
        return e;
    mark(ctx, 3, st);
    for (int c = kBandClasses - 1; c >= 0; --c)
      if (R.cnt[c] && (e = launch_bsw(R.shape[c], D, R.L[c], R.cnt[c], ctx->sms, st, nullptr,
                                      kBswPartTb)) != cudaSuccess)
        return e;
  } else {
    for (int c = kBandClasses - 1; c >= 0; --c)
      if (R.cnt[c] && (e = launch_bsw_rounds(R.shape[c], D, R.L[c], R.cnt[c], R.per_round[c],
                                             ctx->sms, st, nullptr, R.L[c].work)) != cudaSuccess)
        return e;
    mark(ctx, 3, st);
  }
  mark(ctx, 4, st);
  return cudaSuccess;
}

// Host side of the bucketed call: band classes, ordering, shapes, trace rounds,
// scratch and the work-list upload. Fills R (launched by enqueue_bucketed).
int plan_bucketed(kira_ctx* ctx, const kira_pairs& P, const DevPairs& D, const kira_sw_cfg& cfg,
                  kira_sw_result* dout, uint32_t* ncig, uint32_t* flags_dev,
                  unsigned long long* cells_dev, BswLaunch& G, BucketRun& R, cudaStream_t st) {
  cudaError_t cerr = cudaSuccess;
  const uint32_t n = P.n;
  std::vector<uint8_t> cls(n);
  // Classes and per-class maxima, part by part on the context's host threads.
  struct ClassPart {
    uint32_t cnt[kBandClasses], qmax[kBandClasses], bmax[kBandClasses], q, w;
  };
  const uint32_t nparts = host_parts(n);
  std::vector<ClassPart> cp(nparts);
  host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    ClassPart x{};
    for (uint32_t i = lo; i < hi; ++i) {
      const uint32_t b = (uint32_t)std::max(P.bandwidth ? P.bandwidth[i] : cfg.bandwidth, 1);
      const int c = band_class(b);
      cls[i] = (uint8_t)c;
      ++x.cnt[c];
      x.qmax[c] = std::max(x.qmax[c], P.read_len[i]);
      x.bmax[c] = std::max(x.bmax[c], b);
      x.q = std::max(x.q, P.read_len[i]);
      x.w = std::max(x.w, P.win_len[i]);
    }
    cp[k] = x;
  });
  uint32_t cnt[kBandClasses] = {}, qmax[kBandClasses] = {}, bmax[kBandClasses] = {};
  uint32_t qall = 0, wall = 0;
  for (const ClassPart& x : cp) {
    for (int c = 0; c < kBandClasses; ++c) {
      cnt[c] += x.cnt[c];
      qmax[c] = std::max(qmax[c], x.qmax[c]);
      bmax[c] = std::max(bmax[c], x.bmax[c]);
    }
    qall = std::max(qall, x.q);
    wall = std::max(wall, x.w);
  }
  uint32_t base[kBandClasses + 1] = {};
  for (int c = 0; c < kBandClasses; ++c) base[c + 1] = base[c] + cnt[c];
  // Order: band class, then read length descending (the tail of a launch is
  // short), stable. Counting sort on (class, qall - q) when the key range is
  // modest (per-part histograms, then each part scatters from its own offsets,
  // which keeps the order stable), else a comparison sort.
  std::vector<uint32_t> list(n);
  const uint64_t nkeys = (uint64_t)kBandClasses * (qall + 1);
  if (nkeys <= 4ull * n + (1u << 16) && nkeys * nparts <= (64ull << 20)) {
    std::vector<uint32_t> at(nkeys * nparts, 0);  // [part][key]: counts, then offsets
    auto key = [&](uint32_t i) { return (uint64_t)cls[i] * (qall + 1) + (qall - P.read_len[i]); };
    host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
      uint32_t* h = at.data() + (uint64_t)k * nkeys;
      for (uint32_t i = lo; i < hi; ++i) ++h[key(i)];
    });
    uint32_t run = 0;
    for (uint64_t kk = 0; kk < nkeys; ++kk)
      for (uint32_t part = 0; part < nparts; ++part) {
        uint32_t& v = at[(uint64_t)part * nkeys + kk];
        const uint32_t c = v;
        v = run;
        run += c;
      }
    host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
      uint32_t* h = at.data() + (uint64_t)k * nkeys;
      for (uint32_t i = lo; i < hi; ++i) list[h[key(i)]++] = i;
    });
  } else {
    uint32_t at[kBandClasses];
    for (int c = 0; c < kBandClasses; ++c) at[c] = base[c];
    for (uint32_t i = 0; i < n; ++i) list[at[cls[i]]++] = i;
    for (int c = 0; c < kBandClasses; ++c)
      std::stable_sort(list.begin() + base[c], list.begin() + base[c + 1],
                       [&](uint32_t a, uint32_t b) { return P.read_len[a] > P.read_len[b]; });
  }
  const SwParams sp = resolve(cfg);
  int shape[kBandClasses];
  uint64_t slot[kBandClasses] = {}, per[kBandClasses] = {};
  uint64_t total = 0;
  for (int c = 0; c < kBandClasses; ++c) {
    shape[c] = cnt[c] ? pick_shape(ctx, bmax[c], qmax[c], sp) : -1;
    if (cnt[c] && shape[c] < 0) return fail(ctx, KIRA_ERR_INVALID, "no shape for band %u", bmax[c]);
    if (!cnt[c]) continue;
    slot[c] = trace_slot_bytes(shape[c], qmax[c]);
    per[c] = slot[c] + 4ull * (qmax[c] + 1);
    total += per[c] * cnt[c];
  }
  // One round: every class's traces live at once (all DP sweeps, then all
  // tracebacks). Otherwise each class runs in rounds over a shared arena.
  uint64_t tneed = 0, mneed = 0;
  for (int c = 0; c < kBandClasses; ++c) {
    tneed += slot[c] * cnt[c];
    mneed += (uint64_t)(qmax[c] + 1) * cnt[c];
  }
  const bool held = trace_arena_holds(ctx, tneed, mneed);
  const uint64_t budget = held ? total : trace_budget(ctx);
  const bool one_round = total <= budget;
  uint32_t per_round[kBandClasses] = {}, rounds_before[kBandClasses + 1] = {};
  uint64_t tbase[kBandClasses + 1] = {}, mbase[kBandClasses + 1] = {};
  uint64_t tbytes = 16, mwords = 1;
  for (int c = 0; c < kBandClasses; ++c) {
    uint32_t r = 0;
    if (cnt[c]) {
      per_round[c] = one_round ? cnt[c]
                               : (uint32_t)std::max<uint64_t>(
                                     1, std::min<uint64_t>(cnt[c], budget / per[c]));
      r = (cnt[c] + per_round[c] - 1) / per_round[c];
      tbytes = one_round ? tbytes : std::max(tbytes, slot[c] * per_round[c]);
      mwords = one_round ? mwords : std::max(mwords, (uint64_t)(qmax[c] + 1) * per_round[c]);
    }
    rounds_before[c + 1] = rounds_before[c] + r;
    tbase[c + 1] = tbase[c] + (one_round ? slot[c] * cnt[c] : 0);
    mbase[c + 1] = mbase[c] + (one_round ? (uint64_t)(qmax[c] + 1) * cnt[c] : 0);
  }
  if (one_round) {
    tbytes = std::max<uint64_t>(tbase[kBandClasses], 16);
    mwords = std::max<uint64_t>(mbase[kBandClasses], 1);
  }
  const uint32_t nwork = std::max<uint32_t>(rounds_before[kBandClasses], 1);
  ctx->last_rounds = rounds_before[kBandClasses];
  if (one_round) {  // the class streams of enqueue_bucketed (created outside any capture)
    if (!ctx->ev_cls_fork)
      KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_cls_fork, cudaEventDisableTiming));
    for (int c = 0; c < kBandClasses; ++c) {
      if (!cnt[c]) continue;
      if (!ctx->cls_st[c])
        KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->cls_st[c], cudaStreamNonBlocking));
      if (!ctx->ev_cls_join[c])
        KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_cls_join[c], cudaEventDisableTiming));
    }
  }
  const uint32_t cap = qall + wall + 2;
  KIRA_DBUF(dlist, uint32_t, B_SW_LIST, n);
  KIRA_DBUF(trace, uint8_t, B_TRACE, tbytes);
  KIRA_DBUF(meta, uint32_t, B_META, mwords);
  KIRA_DBUF(ends, DpEnd, B_ENDS, n);
  KIRA_DBUF(slots, uint32_t, B_CIG_SLOTS, (uint64_t)cap * n);
  KIRA_DBUF(iop, uint32_t, B_ITEM_OF_PAIR, n);
  KIRA_DBUF(work, uint32_t, B_WORK, nwork);
  KIRA_CUDA(cudaMemcpyAsync(dlist, list.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  R = BucketRun{};
  R.one_round = one_round ? 1u : 0u;
  R.nwork = nwork;
  R.work = work;
  for (int c = 0; c < kBandClasses; ++c) {
    R.shape[c] = shape[c];
    R.cnt[c] = cnt[c];
    R.per_round[c] = per_round[c];
    if (!cnt[c]) continue;
    const BswShapeInfo sh = kBswShapes[shape[c]];
    BswLaunch& B = R.L[c];
    B.list = dlist + base[c];
    B.count = cnt[c];
    B.sp = sp;
    B.bias = packed_bias(sh, sp);
    B.offset = D.band_offset;
    B.tg = shape_trace_geom(sh, trace + tbase[c], meta + mbase[c], slot[c], qmax[c] + 1);
    B.ends = ends + base[c];
    B.cells = cells_dev;
    B.cig_slots = slots + (uint64_t)base[c] * cap;
    B.slot_cap = cap;
    B.out = dout;
    B.ncig = ncig;
    B.item_of_pair = iop;
    B.flags = flags_dev;
    B.max_q = qmax[c];
    B.work = work + rounds_before[c];
    B.item_base = base[c];
  }
  G = BswLaunch{};
  G.item_of_pair = iop;
  G.cig_slots = slots;
  G.slot_cap = cap;
  return KIRA_OK;
}

// kira_gpu_verify_batch for large host batches: chunks of `chunk` pairs flow
// through three streams -- copies in (h2d), the composed path (the context's
// stream), results out (d2h) -- so the upload of chunk c+1, the kernels of chunk
// c and the download of chunk c-1 overlap. The host checks of all chunks run
// first, on parallel host threads. The read (and host window) arena is uploaded
// as far as each chunk needs it and its planes are packed for the new range
// only; CIGAR offsets stay global through the running total in total_dev.
// Results are identical to the one-shot path.
// Compact result form (kira_gpu_verify_batch_compact): host outputs.
struct CompactOut {
  uint8_t* status;       // n bytes
  kira_sw_result* rows;  // rows_cap rows: the pairs with an alignment, in pair order
  uint64_t rows_cap;
  uint64_t* rows_used;
};

// Device side of the compact form after every pair's row is final (stream `st`):
// scan of the keep flags, kept rows to their slots, row count to rows_total_dev.
int compact_rows_tail(kira_ctx* ctx, const kira_sw_result* dout, uint32_t n, const uint32_t* keep,
                      kira_sw_result** rows_dev, uint64_t** rows_total_dev, uint64_t cap,
                      cudaStream_t st) {
  cudaError_t cerr = cudaSuccess;
  KIRA_DBUF(off, uint32_t, B_ROW_OFF, std::max<uint32_t>(n, 1));
  KIRA_DBUF(sums, uint32_t, B_ROW_SUMS, n / 4096 + 2);
  KIRA_DBUF(total, uint64_t, B_ROW_TOTAL, 1);
  KIRA_DBUF(rows, kira_sw_result, B_ROWS, std::max<uint64_t>(std::min<uint64_t>(cap, n), 1));
  KIRA_CUDA(launch_cigar_scan(keep, n, off, sums, total, st));
  KIRA_CUDA(launch_compact_rows(dout, n, keep, off, rows, std::min<uint64_t>(cap, n), ctx->sms,
                                st));
  *rows_dev = rows;
  *rows_total_dev = total;
  return KIRA_OK;
}

// Last copies of a composed host call once the counts are known: the CIGAR ops and,
// in the compact form, the kept rows (as many as fit); the capacity checks.
int finish_host_outputs(kira_ctx* ctx, kira_cigar_buf* cigar, const uint32_t* ops, uint64_t total,
                        const CompactOut* co, const kira_sw_result* rows_dev, uint64_t rows_total,
                        cudaStream_t st) {
  if (co) *co->rows_used = rows_total;
  const uint64_t nrows = co ? std::min(rows_total, co->rows_cap) : 0;
  const uint64_t nops = std::min(total, cigar->cap);
  if (nrows)
    KIRA_CUDA(cudaMemcpyAsync(co->rows, rows_dev, sizeof(kira_sw_result) * nrows,
                              cudaMemcpyDeviceToHost, st));
  if (total <= cigar->cap && nops)
    KIRA_CUDA(cudaMemcpyAsync(cigar->ops, ops, 4ull * nops, cudaMemcpyDeviceToHost, st));
  if (nrows || (total <= cigar->cap && nops)) KIRA_CUDA(cudaStreamSynchronize(st));
  if (total > cigar->cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "CIGAR buffer holds %llu ops, %llu needed",
                (unsigned long long)cigar->cap, (unsigned long long)total);
  if (co && rows_total > co->rows_cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "row buffer holds %llu rows, %llu needed",
                (unsigned long long)co->rows_cap, (unsigned long long)rows_total);
  return KIRA_OK;
}

int verify_batch_chunked(kira_ctx* ctx, const kira_pairs& P, const kira_verify_params& p,
                         kira_sw_result* out, kira_cigar_buf* cigar, kira_verify_detail* detail,
                         uint64_t* cells, const std::vector<uint32_t>& bounds,
                         const CompactOut* co = nullptr) {
  cudaError_t cerr = cudaSuccess;
  const uint32_t n = P.n;
  const uint32_t nch = (uint32_t)bounds.size() - 1;  // chunk c: pairs [bounds[c], bounds[c + 1])
  cudaStream_t st = ctx->stream;
  const bool host_w = P.win_seq != nullptr;
  if (!host_w && !ctx->ref_dev) return fail(ctx, KIRA_ERR_INVALID, "no resident reference uploaded");
  const uint64_t wlim = host_w ? P.win_seq_bytes : ctx->ref_len;
  // Host checks (bounds as upload_pairs, maxes as host_maxes) of every chunk, in
  // sub-ranges of 2^14 pairs (about 50 us of reading each) spread over the
  // context's host threads in chunk order; this thread helps until the chunk it
  // needs next is checked, so the first chunk's copies start after a fraction of
  // the batch was read.
  struct Scan {
    Maxes mx;
    uint64_t rend = 0, wend = 0;
    int64_t bad = -1;  // first offending pair
    int kind = 0;      // 1: read outside read_seq, 2: window outside
  };
  const int32_t cfg_band = std::max(p.sw.bandwidth, 1);
  // Descriptors go up packed (12 bytes a pair instead of 24) when every offset that
  // passes the bounds check fits 32 bits; the check pass writes them to the
  // context's pinned staging buffer.
  PackedPair* stage = nullptr;
  if (P.read_seq_bytes <= UINT32_MAX && wlim <= UINT32_MAX) {
    if (ctx->stage_cap < n) {
      const uint64_t cap = std::max<uint64_t>(n, ctx->stage_cap + ctx->stage_cap / 4);
      if (ctx->stage) cudaFreeHost(ctx->stage);
      ctx->stage = nullptr;
      ctx->stage_cap = 0;
      if (cudaHostAlloc(reinterpret_cast<void**>(&ctx->stage), cap * sizeof(PackedPair),
                        cudaHostAllocDefault) == cudaSuccess) {
        ctx->stage_cap = cap;
      } else {  // no pinned staging: the descriptors go up unpacked
        cudaGetLastError();
        ctx->stage = nullptr;
      }
    }
    stage = ctx->stage;
  }
  auto scan_range = [&](uint32_t lo, uint32_t hi, Scan& sc) {
    uint64_t rend = 0, wend = 0;
    uint32_t q = 0, w = 0, band = 0;
    for (uint32_t i = lo; i < hi; ++i) {  // branch-free maxima
      const uint64_t re = P.read_off[i] + P.read_len[i], we = P.win_off[i] + P.win_len[i];
      rend = re > rend ? re : rend;
      wend = we > wend ? we : wend;
      q = P.read_len[i] > q ? P.read_len[i] : q;
      w = P.win_len[i] > w ? P.win_len[i] : w;
    }
    if (stage) {
      // Streaming stores: staging lines left dirty in the CPU caches make the
      // copy engine's reads of them several times slower (measured 5-12 GB/s
      // against 50 GB/s for the chunks written last).
      for (uint32_t i = lo; i < hi; ++i)
        stage_store(stage + i, PackedPair{(uint32_t)P.read_off[i], (uint32_t)P.win_off[i],
                                          (uint16_t)P.read_len[i], (uint16_t)P.win_len[i]});
      stage_fence();
    }
    if (P.bandwidth) {
      for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t b = (uint32_t)std::max(P.bandwidth[i], 1);
        band = b > band ? b : band;
      }
    } else {
      band = (uint32_t)cfg_band;
    }
    sc.rend = rend, sc.wend = wend, sc.mx.q = q, sc.mx.w = w, sc.mx.band = band;
    if (rend > P.read_seq_bytes || wend > wlim) {
      for (uint32_t i = lo; i < hi; ++i) {
        const uint64_t re = P.read_off[i] + P.read_len[i], we = P.win_off[i] + P.win_len[i];
        if (re > P.read_seq_bytes || we > wlim) {
          sc.bad = i;
          sc.kind = re > P.read_seq_bytes ? 1 : 2;
          break;
        }
      }
    }
  };
  constexpr uint32_t kSub = 1u << 14;
  std::vector<uint32_t> sub_lo, sub_chunk, first_sub(nch + 1);
  for (uint32_t c = 0; c < nch; ++c) {
    first_sub[c] = (uint32_t)sub_lo.size();
    const uint32_t lo = bounds[c], hi = bounds[c + 1];
    for (uint32_t x = lo; x < hi; x += kSub) sub_lo.push_back(x), sub_chunk.push_back(c);
  }
  first_sub[nch] = (uint32_t)sub_lo.size();
  const uint32_t nsub = (uint32_t)sub_lo.size();
  std::vector<Scan> subs(nsub);
  std::unique_ptr<std::atomic<uint32_t>[]> left(new std::atomic<uint32_t>[nch]);
  for (uint32_t c = 0; c < nch; ++c) left[c].store(first_sub[c + 1] - first_sub[c]);
  std::atomic<uint32_t> next{0};
  auto take_one = [&]() -> bool {
    const uint32_t sidx = next.fetch_add(1, std::memory_order_relaxed);
    if (sidx >= nsub) return false;
    const uint32_t c = sub_chunk[sidx];
    const uint32_t hi = std::min(bounds[c + 1], sub_lo[sidx] + kSub);
    scan_range(sub_lo[sidx], hi, subs[sidx]);
    left[c].fetch_sub(1, std::memory_order_release);
    return true;
  };
  host_pool(ctx)->run([&] {
    while (take_one()) {
    }
  });
  // Every host check finishes before this call returns, on every return path.
  struct JoinChecks {
    HostPool* pool;
    std::atomic<uint32_t>* next;
    uint32_t nsub;
    ~JoinChecks() {
      next->store(nsub);
      pool->wait();
    }
  } join_checks{ctx->pool.get(), &next, nsub};
  std::vector<Scan> scans(nch);
  auto checked = [&](uint32_t c) -> int {
    while (left[c].load(std::memory_order_acquire) != 0)
      if (!take_one()) std::this_thread::yield();
    Scan& sc = scans[c];
    for (uint32_t x = first_sub[c]; x < first_sub[c + 1]; ++x) {
      const Scan& u = subs[x];
      sc.rend = std::max(sc.rend, u.rend);
      sc.wend = std::max(sc.wend, u.wend);
      sc.mx.q = std::max(sc.mx.q, u.mx.q);
      sc.mx.w = std::max(sc.mx.w, u.mx.w);
      sc.mx.band = std::max(sc.mx.band, u.mx.band);
      if (sc.bad < 0 && u.bad >= 0) sc.bad = u.bad, sc.kind = u.kind;
    }
    if (sc.bad < 0) return KIRA_OK;
    return fail(ctx, KIRA_ERR_INVALID, "pair %lld: %s outside %s", (long long)sc.bad,
                sc.kind == 1 ? "read" : "window",
                sc.kind == 1 ? "read_seq" : (host_w ? "win_seq" : "the resident reference"));
  };
  if (!ctx->h2d) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
  if (!ctx->d2h) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
  while (ctx->ev_up.size() < nch + 1) {
    cudaEvent_t e[4] = {};
    for (auto& x : e) KIRA_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    ctx->ev_up.push_back(e[0]);
    ctx->ev_comp.push_back(e[1]);
    ctx->ev_pack.push_back(e[2]);
    ctx->ev_scan.push_back(e[3]);
  }
  // Consecutive chunks alternate between this context's stream and a twin's (own
  // stream and scratch, same reference and settings), so one chunk's row-serial
  // DP / traceback tail overlaps the next chunk's sieve and Myers. Planes are
  // packed in chunk order (each chunk waits for the previous chunk's packing) and
  // the CIGAR scans run in chunk order (the running total in total_dev).
  if (!ctx->twin) {
    int rc = kira_gpu_init(ctx->device, &ctx->twin);
    if (rc) return fail(ctx, rc, "second compute stream of the chunked path");
  }
  kira_ctx* twin = ctx->twin;
  std::copy(std::begin(ctx->tuned_shape), std::end(ctx->tuned_shape), twin->tuned_shape);
  twin->trace_budget = ctx->trace_budget;
  ctx_share_reference(twin, ctx);
  kira_ctx* const cxs[2] = {ctx, twin};
  // Full-size buffers first, on the compute stream; the copy stream starts after.
  KIRA_DBUF(rs, uint8_t, B_READ_SEQ, P.read_seq_bytes);
  KIRA_DBUF(rp, uint4, B_READ_PLANES, plane_blocks(P.read_seq_bytes));
  uint8_t* ws = ctx->ref_dev;
  uint4* wp = ctx->ref_planes;
  if (host_w) {
    KIRA_DBUF(w, uint8_t, B_WIN_SEQ, P.win_seq_bytes);
    KIRA_DBUF(wpl, uint4, B_WIN_PLANES, plane_blocks(P.win_seq_bytes));
    ws = w;
    wp = wpl;
  }
  KIRA_DBUF(ro, uint64_t, B_READ_OFF, n);
  KIRA_DBUF(rl, uint32_t, B_READ_LEN, n);
  KIRA_DBUF(wo, uint64_t, B_WIN_OFF, n);
  KIRA_DBUF(wl, uint32_t, B_WIN_LEN, n);
  PackedPair* dpk = nullptr;
  if (stage) {
    KIRA_DBUF(d, PackedPair, B_PACKED, n);
    dpk = d;
  }
  int32_t *bo = nullptr, *ab = nullptr, *bw = nullptr;
  if (P.band_offset) {
    KIRA_DBUF(b, int32_t, B_BAND_OFF, n);
    bo = b;
  }
  if (P.abort_score) {
    KIRA_DBUF(b, int32_t, B_ABORT, n);
    ab = b;
  }
  if (P.bandwidth) {
    KIRA_DBUF(b, int32_t, B_BANDW, n);
    bw = b;
  }
  KIRA_DBUF(dout, kira_sw_result, B_OUT, n);
  kira_verify_detail* ddet = nullptr;
  if (detail) {
    KIRA_DBUF(dd, kira_verify_detail, B_DETAIL, n);
    ddet = dd;
  }
  uint8_t* dstat = nullptr;
  uint32_t* keep = nullptr;
  if (co) {
    KIRA_DBUF(a, uint8_t, B_STATUS, n);
    KIRA_DBUF(b, uint32_t, B_KEEP, n);
    dstat = a;
    keep = b;
  }
  KIRA_DBUF(cells_dev, unsigned long long, B_CELLS, 1);
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  KIRA_DBUF(ops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(cigar->cap, 1));
  KIRA_CUDA(cudaMemsetAsync(cells_dev, 0, 8, st));
  KIRA_CUDA(cudaMemsetAsync(total_dev, 0, 8, st));
  KIRA_CUDA(cudaEventRecord(ctx->ev_up[nch], st));
  KIRA_CUDA(cudaStreamWaitEvent(ctx->h2d, ctx->ev_up[nch], 0));
  KIRA_CUDA(cudaStreamWaitEvent(twin->stream, ctx->ev_up[nch], 0));
  // Enqueue order: each chunk's uploads (as soon as its host checks pass) and then
  // its kernels, chunk by chunk, then every chunk's downloads. A chunk's kernels
  // start as soon as its uploads land instead of after the last chunk's host checks
  // (measured: the 2M-pair compact call 3.8 -> 3.6 ms); on the copy, compute and
  // download streams of this path the later uploads were not held up behind the
  // kernels' waits.
  // Grouped banded SW (three or more chunks): each chunk runs only the stages up to
  // Myers, which list its SW pairs (batch indices) in its group's item list; the
  // chunks form two groups (the first ending at about 55 % of the pairs), and each
  // group's DP + traceback run once over the group's items on two side streams
  // while the later chunks' uploads and front stages go on. One SW launch per chunk
  // was a small partial wave each (a chunk of 250k-500k pairs has 12k-25k items
  // against 38k resident one-lane groups). Scratch: group 0 in this context, group
  // 1 in the twin; the CIGAR scan and compaction run once over the batch.
  const bool grouped = nch >= 3;
  uint32_t gsplit = nch;  // first chunk of group 1
  DeferSw dfs{};
  if (grouped) {
    gsplit = 1;
    while (gsplit + 1 < nch && (uint64_t)bounds[gsplit] * 100 < (uint64_t)n * 55) ++gsplit;
    KIRA_DBUF(gn, uint32_t, B_NCIG, n);
    KIRA_DBUF(gs, int32_t, B_SW_OFFSET, n);
    KIRA_DBUF(gl, uint32_t, B_SW_LIST, n);
    KIRA_DBUF(gc, uint32_t, B_SW_GROUPS, 2);
    KIRA_CUDA(cudaMemsetAsync(gc, 0, 8, st));
    dfs = DeferSw{gn, gs, gl, gc, 0};
    for (int k = 0; k < 4; ++k)
      if (!ctx->cls_st[k]) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->cls_st[k], cudaStreamNonBlocking));
    for (int k = 0; k < kBandClasses; ++k)
      if (!ctx->ev_cls_join[k])
        KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_cls_join[k], cudaEventDisableTiming));
    if (!ctx->ev_cls_fork)
      KIRA_CUDA(cudaEventCreateWithFlags(&ctx->ev_cls_fork, cudaEventDisableTiming));
  }
  const SwParams gsp = resolve(p.sw);
  BswLaunch gB[2] = {};
  // DP + traceback of group g (chunks [c0, c1)) on side streams 2g and 2g + 1,
  // behind the group's front stages; ev_cls_join[g] marks the end.
  auto run_group_sw = [&](int g, uint32_t c0, uint32_t c1) -> int {
    kira_ctx* gx = g == 0 ? ctx : twin;
    cudaStream_t s1 = ctx->cls_st[2 * g], s2 = ctx->cls_st[2 * g + 1];
    Maxes gm;
    for (uint32_t c = c0; c < c1; ++c) {
      gm.q = std::max(gm.q, scans[c].mx.q);
      gm.w = std::max(gm.w, scans[c].mx.w);
      gm.band = std::max(gm.band, scans[c].mx.band);
    }
    const int shape = pick_shape(ctx, gm.band, gm.q, gsp);
    if (shape < 0) return fail(ctx, KIRA_ERR_INVALID, "no banded-SW shape for band %u", gm.band);
    const uint32_t lo = bounds[c0], ng = bounds[c1] - lo;
    const uint32_t per_round = round_items(gx, ng, shape, gm.q);
    BswLaunch& B = gB[g];
    int rc = prepare_bsw(gx, n, ng, per_round, gm, shape, B);
    if (rc) {
      if (gx != ctx) ctx->last_error = gx->last_error;
      return rc;
    }
    B.list = dfs.slist + lo;
    B.count_dev = dfs.count + g;
    B.sp = gsp;
    B.bias = packed_bias(kBswShapes[shape], gsp);
    B.offset = dfs.swoff;
    B.cells = cells_dev;
    B.out = dout;
    B.ncig = dfs.ncig;
    B.flags = static_cast<uint32_t*>(gx->bufs[B_COUNTERS].p) + 2;
    // The group's scratch was (re)sized on gx's stream; its chunks' fronts ran on
    // both compute streams.
    KIRA_CUDA(cudaEventRecord(ctx->ev_cls_join[2 + g], gx->stream));
    KIRA_CUDA(cudaStreamWaitEvent(s1, ctx->ev_cls_join[2 + g], 0));
    for (uint32_t c = c0; c < c1; ++c) KIRA_CUDA(cudaStreamWaitEvent(s1, ctx->ev_comp[c], 0));
    const DevPairs Dg{n,  rs, ro, rl, ws, wo, wl, bo, ab, bw, rp, wp};
    if (per_round >= ng && ng >= kSplitPairs) {
      KIRA_CUDA(cudaEventRecord(ctx->ev_cls_join[4 + g], s1));
      KIRA_CUDA(cudaStreamWaitEvent(s2, ctx->ev_cls_join[4 + g], 0));
      BswLaunch B1 = B, B2 = B;
      B1.split = 1u;
      B2.split = 2u;
      KIRA_CUDA(launch_bsw(shape, Dg, B1, ng, ctx->sms, s1));
      KIRA_CUDA(launch_bsw(shape, Dg, B2, ng, ctx->sms, s2));
      KIRA_CUDA(cudaEventRecord(ctx->ev_cls_join[4 + g], s2));
      KIRA_CUDA(cudaStreamWaitEvent(s1, ctx->ev_cls_join[4 + g], 0));
    } else {
      KIRA_CUDA(launch_bsw_rounds(shape, Dg, B, ng, per_round, ctx->sms, s1, nullptr));
    }
    KIRA_CUDA(cudaEventRecord(ctx->ev_cls_join[g], s1));
    return KIRA_OK;
  };
  std::vector<uint64_t> r_from(nch), r_to(nch), w_from(nch), w_to(nch);
  uint64_t rdone = 0, wdone = 0;
  cudaStream_t up = ctx->h2d;
  for (uint32_t c = 0; c < nch; ++c) {
    if (int rc = checked(c)) {
      // Earlier chunks' uploads and kernels are enqueued; let them finish first.
      cudaStreamSynchronize(up);
      cudaStreamSynchronize(st);
      cudaStreamSynchronize(twin->stream);
      return rc;
    }
    const uint32_t lo = bounds[c], hi = bounds[c + 1], m = hi - lo;
    const uint64_t rneed = std::max(rdone, scans[c].rend), wneed = std::max(wdone, scans[c].wend);
    const bool short_lens = scans[c].mx.q <= UINT16_MAX && scans[c].mx.w <= UINT16_MAX;
    if (dpk) {
      KIRA_CUDA(cudaMemcpyAsync(dpk + lo, stage + lo, sizeof(PackedPair) * m,
                                cudaMemcpyHostToDevice, up));
    } else {
      KIRA_CUDA(cudaMemcpyAsync(ro + lo, P.read_off + lo, 8ull * m, cudaMemcpyHostToDevice, up));
      KIRA_CUDA(cudaMemcpyAsync(wo + lo, P.win_off + lo, 8ull * m, cudaMemcpyHostToDevice, up));
    }
    if (!dpk || !short_lens) {
      KIRA_CUDA(cudaMemcpyAsync(rl + lo, P.read_len + lo, 4ull * m, cudaMemcpyHostToDevice, up));
      KIRA_CUDA(cudaMemcpyAsync(wl + lo, P.win_len + lo, 4ull * m, cudaMemcpyHostToDevice, up));
    }
    if (bo) KIRA_CUDA(cudaMemcpyAsync(bo + lo, P.band_offset + lo, 4ull * m, cudaMemcpyHostToDevice, up));
    if (ab) KIRA_CUDA(cudaMemcpyAsync(ab + lo, P.abort_score + lo, 4ull * m, cudaMemcpyHostToDevice, up));
    if (bw) KIRA_CUDA(cudaMemcpyAsync(bw + lo, P.bandwidth + lo, 4ull * m, cudaMemcpyHostToDevice, up));
    if (rneed > rdone)
      KIRA_CUDA(cudaMemcpyAsync(rs + rdone, P.read_seq + rdone, rneed - rdone,
                                cudaMemcpyHostToDevice, up));
    if (host_w && wneed > wdone)
      KIRA_CUDA(cudaMemcpyAsync(ws + wdone, P.win_seq + wdone, wneed - wdone,
                                cudaMemcpyHostToDevice, up));
    KIRA_CUDA(cudaEventRecord(ctx->ev_up[c], up));
    r_from[c] = rdone, r_to[c] = rneed, w_from[c] = wdone, w_to[c] = wneed;
    rdone = rneed, wdone = wneed;
    // This chunk's kernels, on its compute stream behind its uploads.
    kira_ctx* const cx = cxs[c & 1];
    cudaStream_t cs = cx->stream;
    KIRA_CUDA(cudaStreamWaitEvent(cs, ctx->ev_up[c], 0));
    if (dpk) {
      const bool short_lens = scans[c].mx.q <= UINT16_MAX && scans[c].mx.w <= UINT16_MAX;
      KIRA_CUDA(launch_unpack_pairs(dpk + lo, m, ro + lo, rl + lo, wo + lo, wl + lo, short_lens,
                                    ctx->sms, cs));
    }
    if (c) KIRA_CUDA(cudaStreamWaitEvent(cs, ctx->ev_pack[c - 1], 0));
    // Planes of the newly arrived range, from its first (possibly partial) block.
    if (r_to[c] > r_from[c]) {
      const uint64_t b0 = r_from[c] / 32, nb = plane_blocks(r_to[c]);
      KIRA_CUDA(launch_pack_planes(rs + b0 * 32, r_to[c] - b0 * 32, rp + b0, nb - b0, ctx->sms, cs));
    }
    if (host_w && w_to[c] > w_from[c]) {
      const uint64_t b0 = w_from[c] / 32, nb = plane_blocks(w_to[c]);
      KIRA_CUDA(launch_pack_planes(ws + b0 * 32, w_to[c] - b0 * 32, wp + b0, nb - b0, ctx->sms, cs));
    }
    KIRA_CUDA(cudaEventRecord(ctx->ev_pack[c], cs));
    DevPairs D{m,       rs,      ro + lo, rl + lo, ws,
               wo + lo, wl + lo, bo ? bo + lo : nullptr, ab ? ab + lo : nullptr,
               bw ? bw + lo : nullptr, rp, wp};
    ChunkMode cm;
    cm.planes_ready = true;
    cm.first = c < 2;  // each context's first chunk resets its flag word
    cm.accumulate = true;
    cm.before_scan = c ? ctx->ev_scan[c - 1] : nullptr;
    cm.after_scan = ctx->ev_scan[c];
    DeferSw df = dfs;
    df.slist = dfs.slist + bounds[c < gsplit ? 0 : gsplit];
    df.count = dfs.count + (c < gsplit ? 0 : 1);
    df.base = lo;
    int rc = verify_pipeline(cx, D, scans[c].mx, p, P.read_seq_bytes, P.win_seq_bytes, !host_w,
                             dout + lo, ops, cigar->cap, total_dev, ddet ? ddet + lo : nullptr,
                             cells_dev, cs, cm, grouped ? &df : nullptr);
    if (!rc && co && !grouped)
      rc = launch_status_keep(dout + lo, m, dstat + lo, keep + lo, ctx->sms, cs) == cudaSuccess
               ? KIRA_OK
               : cuda_fail(ctx, cudaGetLastError(), "status bytes");
    if (!rc) KIRA_CUDA(cudaEventRecord(ctx->ev_comp[c], cs));
    if (!rc && grouped && c + 1 == gsplit) {
      // Group 0's SW needs its chunks' maxima (checked) and their fronts (enqueued).
      rc = run_group_sw(0, 0, gsplit);
    }
    if (!rc && grouped && c + 1 == nch) rc = run_group_sw(1, gsplit, nch);
    if (rc) {
      if (cx != ctx && cx->last_error.size()) ctx->last_error = cx->last_error;
      cudaStreamSynchronize(up);
      cudaStreamSynchronize(st);
      cudaStreamSynchronize(twin->stream);
      for (int k = 0; k < 4; ++k)
        if (ctx->cls_st[k]) cudaStreamSynchronize(ctx->cls_st[k]);
      return rc;
    }
  }
  if (grouped) {
    // Both groups' SW done: one CIGAR scan over the batch, then each group's
    // compaction from its own slots, then the status bytes.
    KIRA_CUDA(cudaStreamWaitEvent(st, ctx->ev_cls_join[0], 0));
    KIRA_CUDA(cudaStreamWaitEvent(st, ctx->ev_cls_join[1], 0));
    KIRA_DBUF(off, uint32_t, B_CIG_OFF, n);
    KIRA_DBUF(sums, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
    KIRA_CUDA(launch_cigar_scan(dfs.ncig, n, off, sums, total_dev, st));
    for (int g = 0; g < 2; ++g) {
      const uint32_t lo = bounds[g ? gsplit : 0], hi = bounds[g ? nch : gsplit];
      CompactLaunch CL{hi - lo, dout + lo, dfs.ncig + lo, off + lo, gB[g].item_of_pair + lo,
                       gB[g].cig_slots, gB[g].slot_cap, ops, cigar->cap};
      KIRA_CUDA(launch_cigar_compact(CL, ctx->sms, st));
    }
    if (co) KIRA_CUDA(launch_status_keep(dout, n, dstat, keep, ctx->sms, st));
    for (uint32_t c = 0; c < nch; ++c) KIRA_CUDA(cudaEventRecord(ctx->ev_comp[c], st));
  }
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t lo = bounds[c], m = bounds[c + 1] - lo;
    KIRA_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->ev_comp[c], 0));
    if (co)
      KIRA_CUDA(cudaMemcpyAsync(co->status + lo, dstat + lo, m, cudaMemcpyDeviceToHost, ctx->d2h));
    else
      KIRA_CUDA(cudaMemcpyAsync(out + lo, dout + lo, sizeof(kira_sw_result) * m,
                                cudaMemcpyDeviceToHost, ctx->d2h));
    if (detail)
      KIRA_CUDA(cudaMemcpyAsync(detail + lo, ddet + lo, sizeof(kira_verify_detail) * m,
                                cudaMemcpyDeviceToHost, ctx->d2h));
  }
  kira_sw_result* rows_dev = nullptr;
  uint64_t* rows_total_dev = nullptr;
  uint64_t rows_total = 0;
  if (co) {  // after every chunk's rows (the copy stream waited for all of them)
    int rc = compact_rows_tail(ctx, dout, n, keep, &rows_dev, &rows_total_dev, co->rows_cap,
                               ctx->d2h);
    if (rc) return rc;
    KIRA_CUDA(cudaMemcpyAsync(&rows_total, rows_total_dev, 8, cudaMemcpyDeviceToHost, ctx->d2h));
  }
  uint64_t total = 0;
  unsigned long long hcells = 0;
  uint32_t flags[4] = {}, flags2[4] = {};
  KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, ctx->d2h));
  KIRA_CUDA(cudaMemcpyAsync(&hcells, cells_dev, 8, cudaMemcpyDeviceToHost, ctx->d2h));
  KIRA_CUDA(cudaMemcpyAsync(flags, ctx->bufs[B_COUNTERS].p, 16, cudaMemcpyDeviceToHost, ctx->d2h));
  if (nch > 1)
    KIRA_CUDA(cudaMemcpyAsync(flags2, twin->bufs[B_COUNTERS].p, 16, cudaMemcpyDeviceToHost,
                              ctx->d2h));
  KIRA_CUDA(cudaStreamSynchronize(ctx->d2h));
  cigar->used = total;
  if (cells) *cells = hcells;
  flags[2] |= flags2[2];
  if (flags[2] & 1u) return fail(ctx, KIRA_ERR_RUNTIME, "CIGAR slot overflow");
  if (flags[2] & 6u) return fail(ctx, KIRA_ERR_INVALID, "a pair exceeded the launch's length bounds");
  return finish_host_outputs(ctx, cigar, ops, total, co, rows_dev, rows_total, ctx->d2h);
}

// Runs `enqueue` on `st` through a CUDA graph: replays the cached executable
// graph when every launch parameter matches the one it was captured with,
// otherwise captures anew (updating the executable in place when the topology
// allows). Any capture failure falls back to plain launches.
template <class F>
cudaError_t run_as_graph(kira_ctx* ctx, const DevPairs& D, const BucketRun& R,
                         const CompactLaunch& CL, const uint64_t* total_dev, cudaStream_t st,
                         F&& enqueue) {
  // Key: every value the launches read, field by field (struct padding excluded).
  std::vector<uint8_t> key;
  auto put = [&key](const auto& v) {
    const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
    key.insert(key.end(), b, b + sizeof(v));
  };
  put(D.n), put(D.read_seq), put(D.read_off), put(D.read_len), put(D.win_seq);
  put(D.win_off), put(D.win_len), put(D.band_offset), put(D.abort_score), put(D.bandwidth);
  put(R.one_round), put(R.nwork), put(R.work), put(ctx->sms);
  for (int c = 0; c < kBandClasses; ++c) {
    put(R.shape[c]), put(R.cnt[c]), put(R.per_round[c]);
    if (!R.cnt[c]) continue;
    const BswLaunch& B = R.L[c];
    put(B.list), put(B.count), put(B.sp), put(B.offset), put(B.bias), put(B.max_q);
    put(B.tg.trace), put(B.tg.meta), put(B.tg.slot_bytes), put(B.tg.row_stride);
    put(B.tg.lane_bytes), put(B.tg.k_cells), put(B.tg.meta_stride), put(B.tg.half);
    put(B.ends), put(B.cells), put(B.cig_slots), put(B.slot_cap), put(B.out), put(B.ncig);
    put(B.item_of_pair), put(B.flags), put(B.work), put(B.item_base);
  }
  put(CL.n), put(CL.out), put(CL.ncig), put(CL.off), put(CL.item_of_pair), put(CL.slots);
  put(CL.slot_cap), put(CL.ops), put(CL.cap), put(total_dev);
  if (ctx->graph_exec && key == ctx->graph_key) {
    ++ctx->graph_replays;
    count_launch(ctx->graph_kernels);
    return cudaGraphLaunch(ctx->graph_exec, st);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return enqueue();
  const unsigned long long launched = launch_count();
  cudaError_t ee = enqueue();
  ctx->graph_kernels = launch_count() - launched;  // counted once here, run by the launch below
  e = cudaStreamEndCapture(st, &g);
  if (ee != cudaSuccess || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    ctx->graph_key.clear();
    return enqueue();
  }
  if (ctx->graph_exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(ctx->graph_exec, g, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(ctx->graph_exec);
      ctx->graph_exec = nullptr;
    }
  }
  if (!ctx->graph_exec && cudaGraphInstantiate(&ctx->graph_exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    ctx->graph_exec = nullptr;
    cudaGraphDestroy(g);
    ctx->graph_key.clear();
    return enqueue();
  }
  cudaGraphDestroy(g);
  ctx->graph_key = std::move(key);
  ++ctx->graph_captures;
  return cudaGraphLaunch(ctx->graph_exec, st);
}

}  // namespace

// ---------------------------------------------------------------------------
namespace {

// Chunked host input of the WFA and prefilter entry points: the pair arrays and
// the read / window arenas go up chunk by chunk on the copy-in stream (the arenas
// as far as each chunk needs them), and each chunk's kernels wait for its own
// copies, so uploads, kernels and result downloads of consecutive chunks overlap.
// Every chunk's uploads are enqueued before any chunk's kernels, and the downloads
// after all kernels: streams can share a hardware work queue, where a command that
// waits (kernels waiting for their upload, a download for its kernels) holds up
// what was enqueued after it.
struct ChunkedInput {
  uint32_t chunk = 0, nch = 0;
  std::vector<uint64_t> rend, wend;  // per chunk: arena bytes needed up to it
  DevPairs D{};                      // full-size device buffers
  uint64_t rdone = 0, wdone = 0;
};

// Checks every pair's bounds (as upload_pairs) and plans the arena ranges; chunk is
// rounded up to a multiple of the host pass's part size.
int chunked_plan(kira_ctx* ctx, const kira_pairs& P, uint64_t want, ChunkedInput& ci) {
  const uint32_t n = P.n;
  ci.chunk = (uint32_t)std::min<uint64_t>(n, (want + kHostPart - 1) / kHostPart * kHostPart);
  ci.nch = (n + ci.chunk - 1) / ci.chunk;
  const uint64_t wlim = P.win_seq ? P.win_seq_bytes : ctx->ref_len;
  const uint32_t parts = host_parts(n);
  std::vector<uint64_t> rend(parts, 0), wend(parts, 0);
  std::vector<int64_t> bad(parts, -1);
  host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    uint64_t re_max = 0, we_max = 0;
    for (uint32_t i = lo; i < hi; ++i) {
      const uint64_t re = P.read_off[i] + P.read_len[i], we = P.win_off[i] + P.win_len[i];
      re_max = re > re_max ? re : re_max;
      we_max = we > we_max ? we : we_max;
    }
    rend[k] = re_max;
    wend[k] = we_max;
    if (re_max <= P.read_seq_bytes && we_max <= wlim) return;
    for (uint32_t i = lo; i < hi; ++i)
      if (P.read_off[i] + P.read_len[i] > P.read_seq_bytes || P.win_off[i] + P.win_len[i] > wlim) {
        bad[k] = i;
        return;
      }
  });
  for (const int64_t i : bad) {
    if (i < 0) continue;
    if (P.read_off[i] + P.read_len[i] > P.read_seq_bytes)
      return fail(ctx, KIRA_ERR_INVALID, "pair %u: read outside read_seq", (uint32_t)i);
    return fail(ctx, KIRA_ERR_INVALID, "pair %u: window outside %s", (uint32_t)i,
                P.win_seq ? "win_seq" : "the resident reference");
  }
  ci.rend.assign(ci.nch, 0);
  ci.wend.assign(ci.nch, 0);
  uint64_t r = 0, w = 0;
  for (uint32_t c = 0; c < ci.nch; ++c) {  // cumulative: later chunks never shrink the range
    const uint32_t k0 = c * (ci.chunk / kHostPart), k1 = std::min(parts, k0 + ci.chunk / kHostPart);
    for (uint32_t k = k0; k < k1; ++k) r = std::max(r, rend[k]), w = std::max(w, wend[k]);
    ci.rend[c] = r;
    ci.wend[c] = w;
  }
  cudaError_t cerr = cudaSuccess;
  KIRA_DBUF(rs, uint8_t, B_READ_SEQ, P.read_seq_bytes);
  KIRA_DBUF(ro, uint64_t, B_READ_OFF, n);
  KIRA_DBUF(rl, uint32_t, B_READ_LEN, n);
  KIRA_DBUF(wo, uint64_t, B_WIN_OFF, n);
  KIRA_DBUF(wl, uint32_t, B_WIN_LEN, n);
  const uint8_t* ws = ctx->ref_dev;
  if (P.win_seq) {
    KIRA_DBUF(wb, uint8_t, B_WIN_SEQ, P.win_seq_bytes);
    ws = wb;
  }
  ci.D = DevPairs{n, rs, ro, rl, ws, wo, wl, nullptr, nullptr, nullptr, nullptr, nullptr};
  if (!ctx->h2d) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
  if (!ctx->d2h) KIRA_CUDA(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
  while (ctx->ev_up.size() < ci.nch + 1) {
    cudaEvent_t e[4] = {};
    for (auto& x : e) KIRA_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    ctx->ev_up.push_back(e[0]);
    ctx->ev_comp.push_back(e[1]);
    ctx->ev_pack.push_back(e[2]);
    ctx->ev_scan.push_back(e[3]);
  }
  return KIRA_OK;
}

// Enqueues chunk c's copies on the copy-in stream (extra copies the caller adds
// through `extra(lo, m, stream)`) and records ev_up[c] after them.
template <class F>
int chunked_upload(kira_ctx* ctx, const kira_pairs& P, ChunkedInput& ci, uint32_t c, F&& extra) {
  const uint32_t lo = c * ci.chunk, m = std::min(P.n, lo + ci.chunk) - lo;
  cudaStream_t up = ctx->h2d;
  const DevPairs& D = ci.D;
  KIRA_CUDA(cudaMemcpyAsync((uint64_t*)D.read_off + lo, P.read_off + lo, 8ull * m,
                            cudaMemcpyHostToDevice, up));
  KIRA_CUDA(cudaMemcpyAsync((uint32_t*)D.read_len + lo, P.read_len + lo, 4ull * m,
                            cudaMemcpyHostToDevice, up));
  KIRA_CUDA(cudaMemcpyAsync((uint64_t*)D.win_off + lo, P.win_off + lo, 8ull * m,
                            cudaMemcpyHostToDevice, up));
  KIRA_CUDA(cudaMemcpyAsync((uint32_t*)D.win_len + lo, P.win_len + lo, 4ull * m,
                            cudaMemcpyHostToDevice, up));
  if (ci.rend[c] > ci.rdone) {
    KIRA_CUDA(cudaMemcpyAsync((uint8_t*)D.read_seq + ci.rdone, P.read_seq + ci.rdone,
                              ci.rend[c] - ci.rdone, cudaMemcpyHostToDevice, up));
    ci.rdone = ci.rend[c];
  }
  if (P.win_seq && ci.wend[c] > ci.wdone) {
    KIRA_CUDA(cudaMemcpyAsync((uint8_t*)D.win_seq + ci.wdone, P.win_seq + ci.wdone,
                              ci.wend[c] - ci.wdone, cudaMemcpyHostToDevice, up));
    ci.wdone = ci.wend[c];
  }
  const int rc = extra(lo, m, up);
  if (rc) return rc;
  KIRA_CUDA(cudaEventRecord(ctx->ev_up[c], up));
  return KIRA_OK;
}

// Device view of chunk [lo, lo + m) of a chunked input.
DevPairs chunk_view(const DevPairs& D, uint32_t lo, uint32_t m) {
  DevPairs v = D;
  v.n = m;
  v.read_off += lo;
  v.read_len += lo;
  v.win_off += lo;
  v.win_len += lo;
  return v;
}

// Chunk size of a host batch: the context's setting (-1: a quarter of the batch,
// at least 2^18 pairs; 0: one shot); chunking needs at least two chunks and no
// stage profiling.
uint64_t host_chunk(const kira_ctx* ctx, uint32_t n) {
  if (ctx->profile) return 0;
  const uint64_t chunk = ctx->chunk_pairs < 0 ? std::max<uint64_t>(1u << 18, (n + 3ull) / 4)
                                              : (uint64_t)ctx->chunk_pairs;
  return chunk && n >= 2 * chunk ? chunk : 0;
}

}  // namespace

namespace {

// The composed path on host buffers: full rows (`out`) or the compact form (`co`).
int verify_host(kira_ctx* ctx, const kira_pairs& P, const kira_verify_params& prm,
                kira_sw_result* out, kira_cigar_buf* cigar, kira_verify_detail* detail,
                uint64_t* cells, const CompactOut* co) {
  const kira_verify_params* p = &prm;
  cigar->used = 0;
  if (cells) *cells = 0;
  if (P.n == 0) return KIRA_OK;
  cudaSetDevice(ctx->device);
  // Chunks alternate between two compute streams so each chunk's row-serial DP and
  // traceback tail overlaps the next chunk; a few large chunks still do best
  // (each pays some fixed launch and tail cost). Automatic: batches of at least
  // 2^20 pairs in chunks of 1/8, 1/4, 1/4, 1/4, 1/8 of the batch (a small first
  // chunk starts the GPU sooner, a small last one drains sooner), smaller ones in
  // quarters of at least 2^18 pairs; chunk_pairs > 0: equal chunks of that size.
  std::vector<uint32_t> bounds;
  if (!ctx->profile) {
    const uint64_t n = P.n;
    if (ctx->chunk_pairs < 0 && n >= (1u << 20)) {
      bounds = {0u, (uint32_t)(n / 8), (uint32_t)(3 * n / 8), (uint32_t)(5 * n / 8),
                (uint32_t)(n - n / 8), (uint32_t)n};
    } else {
      const uint64_t chunk = ctx->chunk_pairs < 0 ? std::max<uint64_t>(1u << 18, (n + 3) / 4)
                                                  : (uint64_t)ctx->chunk_pairs;
      if (chunk && n >= 2 * chunk)
        for (uint64_t lo = 0; lo <= n; lo += chunk) bounds.push_back((uint32_t)std::min(lo, n));
      if (!bounds.empty() && bounds.back() != n) bounds.push_back((uint32_t)n);
    }
  }
  if (bounds.size() >= 3)
    return verify_batch_chunked(ctx, P, *p, out, cigar, detail, cells, bounds, co);
  const Maxes mx = host_maxes(ctx, P, p->sw.bandwidth);
  DevPairs D;
  int rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  cudaError_t cerr = cudaSuccess;
  cudaStream_t st = ctx->stream;
  const uint32_t n = P.n;
  KIRA_DBUF(dout, kira_sw_result, B_OUT, n);
  kira_verify_detail* ddet = nullptr;
  if (detail) {
    KIRA_DBUF(dd, kira_verify_detail, B_DETAIL, n);
    ddet = dd;
  }
  KIRA_DBUF(cells_dev, unsigned long long, B_CELLS, 1);
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  KIRA_DBUF(ops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(cigar->cap, 1));
  KIRA_CUDA(cudaMemsetAsync(cells_dev, 0, 8, st));
  rc = verify_pipeline(ctx, D, mx, *p, P.read_seq_bytes, P.win_seq_bytes, P.win_seq == nullptr,
                       dout, ops, cigar->cap, total_dev, ddet, cells_dev, st);
  if (rc) return rc;
  uint64_t total = 0, rows_total = 0;
  unsigned long long hcells = 0;
  uint32_t flags[4];
  kira_sw_result* rows_dev = nullptr;
  if (co) {
    KIRA_DBUF(dstat, uint8_t, B_STATUS, n);
    KIRA_DBUF(keep, uint32_t, B_KEEP, n);
    KIRA_CUDA(launch_status_keep(dout, n, dstat, keep, ctx->sms, st));
    uint64_t* rows_total_dev = nullptr;
    rc = compact_rows_tail(ctx, dout, n, keep, &rows_dev, &rows_total_dev, co->rows_cap, st);
    if (rc) return rc;
    KIRA_CUDA(cudaMemcpyAsync(co->status, dstat, n, cudaMemcpyDeviceToHost, st));
    KIRA_CUDA(cudaMemcpyAsync(&rows_total, rows_total_dev, 8, cudaMemcpyDeviceToHost, st));
  } else {
    KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_sw_result) * n, cudaMemcpyDeviceToHost, st));
  }
  if (detail)
    KIRA_CUDA(cudaMemcpyAsync(detail, ddet, sizeof(kira_verify_detail) * n,
                              cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&hcells, cells_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(flags, ctx->bufs[B_COUNTERS].p, 16, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  cigar->used = total;
  if (cells) *cells = hcells;
  if (flags[2] & 1u) return fail(ctx, KIRA_ERR_RUNTIME, "CIGAR slot overflow");
  if (flags[2] & 6u) return fail(ctx, KIRA_ERR_INVALID, "a pair exceeded the launch's length bounds");
  return finish_host_outputs(ctx, cigar, ops, total, co, rows_dev, rows_total, st);
}

}  // namespace

extern "C" {

int kira_gpu_is_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n > 0 ? 1 : 0;
}

int kira_gpu_init(int device, kira_ctx** out) {
  if (!out) return KIRA_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return KIRA_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return KIRA_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return KIRA_ERR_DRIVER;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return KIRA_ERR_DRIVER;
  if (prop.major < 10) return KIRA_ERR_NO_DEVICE;  // sm_100a binary only
  // Freed arena blocks stay in the device's default pool for reuse instead of
  // going back to the driver at every synchronisation.
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  kira_ctx* ctx = new kira_ctx();
  ctx->device = device;
  ctx->sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return KIRA_ERR_DRIVER;
  }
  *out = ctx;
  return KIRA_OK;
}

void kira_gpu_destroy(kira_ctx* ctx) {
  if (!ctx) return;
  if (ctx->twin) kira_gpu_destroy(ctx->twin);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& b : ctx->bufs)
    if (b.p) cudaFreeAsync(b.p, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  ctx->ref_owner.reset();
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  for (auto e : ctx->ev_up) cudaEventDestroy(e);
  for (auto e : ctx->ev_comp) cudaEventDestroy(e);
  for (auto e : ctx->ev_pack) cudaEventDestroy(e);
  for (auto e : ctx->ev_scan) cudaEventDestroy(e);
  if (ctx->h2d) cudaStreamDestroy(ctx->h2d);
  if (ctx->d2h) cudaStreamDestroy(ctx->d2h);
  if (ctx->aux) {
    cudaStreamSynchronize(ctx->aux);
    cudaStreamDestroy(ctx->aux);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  for (int c = 0; c < kBandClasses; ++c) {
    if (ctx->cls_st[c]) {
      cudaStreamSynchronize(ctx->cls_st[c]);
      cudaStreamDestroy(ctx->cls_st[c]);
    }
    if (ctx->ev_cls_join[c]) cudaEventDestroy(ctx->ev_cls_join[c]);
  }
  if (ctx->ev_cls_fork) cudaEventDestroy(ctx->ev_cls_fork);
  if (ctx->stage) cudaFreeHost(ctx->stage);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int kira_gpu_last_error(const kira_ctx* ctx, char* buf, size_t len) {
  const std::string& s = ctx ? ctx->last_error : std::string();
  if (buf && len) {
    const size_t k = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return (int)s.size();
}

uint64_t kira_gpu_arena_bytes(const kira_ctx* ctx) {
  uint64_t t = 0;
  if (!ctx) return 0;
  for (const auto& b : ctx->bufs) t += b.bytes;
  return t + ctx->ref_len;
}

int kira_gpu_sieve_batch(kira_ctx* ctx, const kira_sieve_job* jobs, uint32_t n,
                         kira_sieve_result* out) {
  if (!ctx) return KIRA_ERR_INVALID;
  if (n == 0) return KIRA_OK;
  if (!jobs || !out) return fail(ctx, KIRA_ERR_INVALID, "null jobs/out");
  cudaSetDevice(ctx->device);
  // backend.rs:101-116: per-job validation before any device work.
  uint64_t rbytes = 0, wbytes = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const kira_sieve_job& j = jobs[i];
    if (j.read_bytes > KIRA_READ_BYTES_MAX)
      return fail(ctx, KIRA_ERR_READ_TOO_LONG,
                  "read too long for the CUDA backend (%u > %d bytes packed)", j.read_bytes,
                  KIRA_READ_BYTES_MAX);
    if ((uint64_t)j.read_bytes * 4 < j.read_nucs || (uint64_t)j.ref_bytes * 4 < j.ref_nucs)
      return fail(ctx, KIRA_ERR_INVALID, "job %u: packed buffer shorter than its length", i);
    if (j.ref_nucs >= (1u << 20) + j.read_nucs)
      return fail(ctx, KIRA_ERR_INVALID, "job %u: window longer than 2^20 shifts", i);
    rbytes += j.read_bytes;
    wbytes += j.ref_bytes;
  }
  std::vector<uint8_t> hr(rbytes + 1), hw(wbytes + 1);
  std::vector<uint64_t> ro(n), wo(n);
  std::vector<uint32_t> rn(n), wn(n), mm(n);
  uint64_t a = 0, b = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const kira_sieve_job& j = jobs[i];
    if (j.read_bytes) std::memcpy(hr.data() + a, j.read_packed, j.read_bytes);
    if (j.ref_bytes) std::memcpy(hw.data() + b, j.ref_packed, j.ref_bytes);
    ro[i] = a;
    wo[i] = b;
    a += j.read_bytes;
    b += j.ref_bytes;
    rn[i] = j.read_nucs;
    wn[i] = j.ref_nucs;
    mm[i] = j.max_mismatches;
  }
  cudaError_t cerr = cudaSuccess;
  cudaStream_t st = ctx->stream;
  KIRA_DBUF(drs, uint8_t, B_READ_SEQ, rbytes + 1);
  KIRA_DBUF(dws, uint8_t, B_WIN_SEQ, wbytes + 1);
  KIRA_DBUF(dro, uint64_t, B_READ_OFF, n);
  KIRA_DBUF(dwo, uint64_t, B_WIN_OFF, n);
  KIRA_DBUF(drn, uint32_t, B_READ_LEN, n);
  KIRA_DBUF(dwn, uint32_t, B_WIN_LEN, n);
  KIRA_DBUF(dmm, uint32_t, B_BAND_OFF, n);
  KIRA_DBUF(dout, kira_sieve_result, B_SIEVE_OUT, n);
  KIRA_CUDA(cudaMemcpyAsync(drs, hr.data(), rbytes + 1, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(dws, hw.data(), wbytes + 1, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(dro, ro.data(), 8ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(dwo, wo.data(), 8ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(drn, rn.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(dwn, wn.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemcpyAsync(dmm, mm.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  SieveJobsDev J{n, drs, dro, drn, dws, dwo, dwn, dmm};
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);  // stage 0 of kira_gpu_stage_times: the sieve kernel alone
  KIRA_CUDA(launch_sieve_dropin(J, dout, ctx->sms, st));
  mark(ctx, 1, st);
  KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_sieve_result) * n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  return KIRA_OK;
}

int kira_gpu_set_bsw_shape(kira_ctx* ctx, uint32_t band, int shape) {
  if (!ctx) return KIRA_ERR_INVALID;
  if (shape >= 0 && !shape_fits(shape, band))
    return fail(ctx, KIRA_ERR_INVALID, "shape %d does not cover band %u", shape, band);
  ctx->tuned_shape[band_class(band)] = shape;
  return KIRA_OK;
}

int kira_gpu_set_plain(kira_ctx* ctx, int plain) {
  if (!ctx) return KIRA_ERR_INVALID;
  ctx->plain = plain != 0;
  return KIRA_OK;
}

int kira_gpu_set_graphs(kira_ctx* ctx, int enable, uint64_t* captures, uint64_t* replays) {
  if (!ctx) return KIRA_ERR_INVALID;
  if (enable >= 0) ctx->graphs = enable != 0;
  if (captures) *captures = ctx->graph_captures;
  if (replays) *replays = ctx->graph_replays;
  return KIRA_OK;
}

int kira_gpu_nm_md(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_result* results,
                   const uint32_t* cigar_ops, uint64_t n_ops, uint32_t* nm, uint32_t* md_off,
                   char* md, uint64_t md_cap, uint64_t* md_used) {
  if (!ctx || !pairs || !results || !nm || !md_off || !md_used) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  *md_used = 0;
  md_off[0] = 0;
  if (P.n == 0) return KIRA_OK;
  if (n_ops && !cigar_ops) return KIRA_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);
  DevPairs D;
  int rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  cudaError_t cerr = cudaSuccess;
  const uint32_t n = P.n;
  KIRA_DBUF(dres, kira_sw_result, B_NMMD_RES, n);
  KIRA_DBUF(dops, uint32_t, B_NMMD_OPS, std::max<uint64_t>(n_ops, 1));
  KIRA_DBUF(dnm, uint32_t, B_NMMD_NM, n);
  KIRA_DBUF(dlen, uint32_t, B_NMMD_LEN, n);
  KIRA_DBUF(doff, uint32_t, B_NMMD_OFF, n);
  KIRA_DBUF(sums, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  KIRA_DBUF(flags, uint32_t, B_NMMD_FLAGS, 1);
  KIRA_CUDA(cudaMemcpyAsync(dres, results, sizeof(kira_sw_result) * n, cudaMemcpyHostToDevice, st));
  if (n_ops)
    KIRA_CUDA(cudaMemcpyAsync(dops, cigar_ops, 4ull * n_ops, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(cudaMemsetAsync(flags, 0, 4, st));
  mark(ctx, 1, st);
  NmMdLaunch L{n, dres, dops, n_ops, dnm, dlen, doff, nullptr, flags};
  KIRA_CUDA(launch_nm_md(D, L, false, ctx->sms, st));
  KIRA_CUDA(launch_cigar_scan(dlen, n, doff, sums, total_dev, st));
  mark(ctx, 2, st);
  uint64_t total = 0;
  uint32_t hflags = 0;
  KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&hflags, flags, 4, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(nm, dnm, 4ull * n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(md_off, doff, 4ull * n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  if (hflags & 1u) return fail(ctx, KIRA_ERR_INVALID, "a result's CIGAR lies outside cigar_ops");
  if (total > UINT32_MAX) return fail(ctx, KIRA_ERR_INVALID, "MD text above 4 GiB: split the batch");
  md_off[n] = (uint32_t)total;
  *md_used = total;
  if (total > md_cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "MD buffer holds %llu bytes, %llu needed",
                (unsigned long long)md_cap, (unsigned long long)total);
  KIRA_DBUF(dmd, char, B_NMMD_OUT, std::max<uint64_t>(total, 1));
  L.md = dmd;
  mark(ctx, 3, st);
  KIRA_CUDA(launch_nm_md(D, L, true, ctx->sms, st));
  mark(ctx, 4, st);
  if (total) KIRA_CUDA(cudaMemcpyAsync(md, dmd, total, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  return KIRA_OK;
}

namespace {

// router::wfa_score_budget (src/alignment/router.rs:160-165) on the host.
int64_t wfa_budget_host(int64_t read_len, int64_t pct, int64_t x, int64_t o, int64_t e) {
  return std::max(read_len * pct / 100 * x, (o + e * 4) * 3);
}

constexpr uint64_t kWfaScratchBudget = 4ull << 30;  // per-call warp history, bytes

}  // namespace

int kira_gpu_wfa_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_wfa_params* prm,
                       const int32_t* max_score, const int32_t* text_begin_free,
                       kira_wfa_result* out, kira_cigar_buf* cigar) {
  if (!ctx || !pairs || !prm || !out) return KIRA_ERR_INVALID;
  const bool tb = prm->traceback != 0;
  if (tb && !cigar) return fail(ctx, KIRA_ERR_INVALID, "traceback needs a CIGAR buffer");
  if (cigar) cigar->used = 0;
  const kira_pairs& P = *pairs;
  const uint32_t n = P.n;
  if (n == 0) return KIRA_OK;
  if (tb && cigar->cap && !cigar->ops) return KIRA_ERR_INVALID;
  WfaLaunch L{};
  L.n = n;
  L.valid = 1;
  const int64_t kCostMax = 1 << 20;
  if (prm->scored) {
    // WfaCosts::scored (wfa.rs:41-52): refused costs give None for every pair.
    const int64_t a = prm->match_score, b = prm->mismatch, o = prm->gap_open, e = prm->gap_extend;
    if (a <= 0 || b <= 0 || o < 0 || e <= 0) {
      L.valid = 0;
    } else {
      if (a + b > kCostMax || o > kCostMax || a + e > kCostMax)
        return fail(ctx, KIRA_ERR_INVALID, "WFA costs above 2^20");
      L.x = (int32_t)(a + b), L.o = (int32_t)o, L.ei = (int32_t)(a + e), L.ed = (int32_t)e;
    }
  } else {
    if (prm->mismatch < 1 || prm->gap_open < 0 || prm->gap_extend < 1)
      return fail(ctx, KIRA_ERR_INVALID, "WFA penalties need mismatch >= 1, gap_open >= 0, "
                  "gap_extend >= 1");
    if (prm->mismatch > kCostMax || prm->gap_open > kCostMax || prm->gap_extend > kCostMax)
      return fail(ctx, KIRA_ERR_INVALID, "WFA costs above 2^20");
    L.x = prm->mismatch, L.o = prm->gap_open, L.ei = prm->gap_extend, L.ed = prm->gap_extend;
  }
  if (!L.valid) {
    for (uint32_t i = 0; i < n; ++i) {
      out[i] = kira_wfa_result{};
      out[i].cost = -1;
    }
    return KIRA_OK;
  }
  L.lookback = std::max(L.x, std::max(L.o + L.ei, L.o + L.ed));
  L.scored = prm->scored ? 1 : 0;
  L.match = prm->match_score;
  L.max_score = prm->max_score;
  L.budget_pct = prm->budget_pct < 0 ? 25 : prm->budget_pct;
  L.budget_x = L.x, L.budget_o = L.o, L.budget_e = L.ei;
  L.tbf = prm->text_begin_free;
  L.drop = prm->adaptive_drop < 0 ? -1 : prm->adaptive_drop;

  // Batch bounds that size the per-warp history.
  struct WfaMax {
    uint32_t m = 0, n = 0;
    int64_t s = INT64_MIN, tbf = INT64_MIN;
  };
  std::vector<WfaMax> wm(host_parts(n));
  host_for(ctx, n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    WfaMax x;
    for (uint32_t i = lo; i < hi; ++i) {
      x.m = P.read_len[i] > x.m ? P.read_len[i] : x.m;
      x.n = P.win_len[i] > x.n ? P.win_len[i] : x.n;
    }
    if (max_score)
      for (uint32_t i = lo; i < hi; ++i) x.s = std::max<int64_t>(x.s, max_score[i]);
    if (text_begin_free)
      for (uint32_t i = lo; i < hi; ++i) x.tbf = std::max<int64_t>(x.tbf, text_begin_free[i]);
    wm[k] = x;
  });
  uint32_t m_max = 0, n_max = 0;
  int64_t s_max = INT64_MIN, tbf_max = INT64_MIN;
  for (const WfaMax& x : wm) {
    m_max = std::max(m_max, x.m);
    n_max = std::max(n_max, x.n);
    s_max = std::max(s_max, x.s);
    tbf_max = std::max(tbf_max, x.tbf);
  }
  if (m_max > (uint32_t)kWfaMaxLen || n_max > (uint32_t)kWfaMaxLen)
    return fail(ctx, KIRA_ERR_READ_TOO_LONG, "WFA reads and windows up to %d bases", kWfaMaxLen);
  if (!max_score)
    s_max = prm->max_score >= 0 ? prm->max_score
                                : wfa_budget_host(m_max, L.budget_pct, L.x, L.o, L.ei);
  if (!text_begin_free) tbf_max = prm->text_begin_free;
  tbf_max = std::min<int64_t>(std::max<int64_t>(tbf_max, 0), std::max<int64_t>(n_max - 1, 0));
  const int64_t cost_cap = L.drop < 0 ? (int64_t)L.o + (int64_t)L.ei * m_max
                                      : (int64_t)std::max(L.x, L.o + L.ei) * (2 * m_max + n_max + 2);
  const int64_t S = std::max<int64_t>(0, std::min(s_max, cost_cap));
  auto width = [&](int64_t s) {
    return std::min<int64_t>(tbf_max + 1 + s / L.ei + s / L.ed, (int64_t)m_max + n_max + 3);
  };
  // Lanes per pair: short reads keep their fronts narrow, so several pairs share a
  // warp; long reads take a warp each.
  L.group = ctx->wfa_lanes ? ctx->wfa_lanes : (m_max <= 512 ? 8 : 32);
  const uint64_t R = (uint64_t)L.lookback + 1;
  uint64_t hist = 0, meta_slots = 0, ring_width = 0;
  if (tb) {
    for (int64_t s = 0; s <= S; ++s) hist += 3ull * (uint64_t)width(s);
    meta_slots = (uint64_t)S + 1;
  } else {
    ring_width = (uint64_t)width(S);
    hist = R * 3ull * ring_width;
  }
  if (hist >= (1ull << 31) || meta_slots >= (1ull << 26) || R > (1u << 20))
    return fail(ctx, KIRA_ERR_OOM, "WFA history of %llu entries per pair: lower max_score",
                (unsigned long long)hist);
  const uint64_t ring_sz = (R * 3ull * sizeof(int2) + 15) & ~15ull;
  const bool ring_shared = ring_sz <= 512;
  const uint64_t meta_bytes = (meta_slots * 3ull * sizeof(int2) + 255) & ~255ull;
  const uint64_t ring_goff = meta_bytes;
  const uint64_t hist_off = ring_goff + (ring_shared ? 0 : ((ring_sz + 255) & ~255ull));
  const uint64_t group_bytes = hist_off + ((hist * 2ull + 255) & ~255ull);
  L.meta_slots = (uint32_t)meta_slots;
  L.hist_cap = (uint32_t)hist;
  L.ring_len = (uint32_t)R;
  L.ring_width = (uint32_t)ring_width;
  L.ring_bytes = ring_shared ? (uint32_t)ring_sz : 0u;
  L.ring_goff = (uint32_t)ring_goff;
  L.hist_off = (uint32_t)hist_off;
  L.group_bytes = group_bytes;
  L.pat_region = 32u + ((m_max + 15u) & ~15u);
  L.smem_group = L.ring_bytes + L.pat_region + 32u + ((n_max + 15u) & ~15u);
  const uint32_t min_cost = (uint32_t)(L.o + std::min(L.ei, L.ed));
  L.slot_cap = (uint32_t)(2 * (S / min_cost) + 2);
  L.max_score_pp = nullptr;
  L.tbf_pp = nullptr;
  // Fixed-window fast path: 64 diagonals per pair (128 when 64 cover fewer than 32
  // scores), placed so every cell of the highest score stays inside for this
  // batch's leading free text; pairs still open at that score fall back to the
  // general kernel with a warp per pair (their fronts are the wide ones).
  // ctx->wfa_lanes != 0 forces the general kernel alone.
  auto place = [&](int width, int* base) {
    int best = -1;
    for (int b = -(width - 1 - (int)tbf_max); b <= 0; ++b) {
      const int64_t lo_s = (int64_t)L.o + (int64_t)L.ei * (1 - b) - 1;
      const int64_t hi_s = (int64_t)L.o + (int64_t)L.ed * (b + width - tbf_max) - 1;
      const int64_t sm = std::min<int64_t>(std::min(lo_s, hi_s), 1 << 20);
      if (sm > best) best = (int)sm, *base = b;
    }
    return best;
  };
  int win_base = 0, win_segments = 2;
  int win_smax = tbf_max <= 63 ? place(64, &win_base) : -1;
  if (win_smax < std::min<int64_t>(S, 32) && tbf_max <= 127) {
    int b4 = 0;
    const int s4 = place(128, &b4);
    if (s4 > win_smax) win_smax = s4, win_base = b4, win_segments = 4;
  }
  const bool use_window = ctx->wfa_lanes == 0 && win_smax >= 16 && L.ring_len <= 64;
  if (use_window) {
    win_smax = (int)std::min<int64_t>(win_smax, S);
    L.win_base = win_base;
    L.win_smax = win_smax;
    L.win_segments = win_segments;
    L.win_ring_bytes =
        (uint32_t)((L.ring_len * 3u * (32u * (uint32_t)win_segments + 2u) * 2u + 15u) & ~15u);
  }

  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);
  cudaError_t cerr = cudaSuccess;
  int32_t *dms = nullptr, *dtbf = nullptr;
  if (max_score) {
    KIRA_DBUF(b, int32_t, B_WFA_MAXS, n);
    dms = b;
  }
  if (text_begin_free) {
    KIRA_DBUF(b, int32_t, B_WFA_TBF, n);
    dtbf = b;
  }
  // Large host batches go chunk by chunk (uploads, kernels and downloads of
  // consecutive chunks overlap); CIGAR offsets continue through the running total.
  const uint64_t chunked = host_chunk(ctx, n);
  ChunkedInput ci;
  DevPairs D;
  int rc = chunked ? chunked_plan(ctx, P, chunked, ci) : upload_pairs(ctx, P, D);
  if (rc) return rc;
  if (chunked) {
    D = ci.D;
  } else {
    if (dms) KIRA_CUDA(cudaMemcpyAsync(dms, max_score, 4ull * n, cudaMemcpyHostToDevice, st));
    if (dtbf)
      KIRA_CUDA(cudaMemcpyAsync(dtbf, text_begin_free, 4ull * n, cudaMemcpyHostToDevice, st));
  }
  // Launch shape: four warps per block while their staged bytes fit comfortably.
  const uint32_t groups_per_warp = 32u / (uint32_t)L.group;
  uint32_t wpb = 4;
  while (wpb > 1 && (uint64_t)wpb * groups_per_warp * L.smem_group > (160u << 10)) wpb >>= 1;
  const uint32_t gpb = wpb * groups_per_warp;
  const size_t smem = (size_t)gpb * L.smem_group;
  int per_sm = 0;
  KIRA_CUDA(wfa_blocks_per_sm(L.group, tb, smem, (int)(32 * wpb), &per_sm));
  if (per_sm < 1) return fail(ctx, KIRA_ERR_INVALID, "WFA: %zu shared bytes per block", smem);
  const uint32_t csz = chunked ? ci.chunk : n, nch = chunked ? ci.nch : 1;
  uint64_t blocks = std::min<uint64_t>((csz + gpb - 1) / gpb, (uint64_t)ctx->sms * per_sm);
  blocks = std::min<uint64_t>(blocks,
                              std::max<uint64_t>(1, kWfaScratchBudget / (gpb * group_bytes)));
  KIRA_DBUF(scratch, uint8_t, B_WFA_SCRATCH, blocks * gpb * group_bytes);
  KIRA_DBUF(dout, kira_wfa_result, B_WFA_OUT, n);
  KIRA_DBUF(work, uint32_t, B_WORK, 4);  // window fetch, flags, general fetch, fallbacks
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  L.scratch = scratch;
  L.flags = work + 1;
  uint64_t wblocks = 0;
  uint32_t fwpb = 4;
  if (use_window) {
    const size_t wsmem = (size_t)4 * (L.win_ring_bytes + L.smem_group - L.ring_bytes);
    int wper = 0;
    KIRA_CUDA(wfa_window_blocks_per_sm(win_segments, tb, wsmem, &wper));
    if (wper < 1) return fail(ctx, KIRA_ERR_INVALID, "WFA window: %zu shared bytes", wsmem);
    wblocks = std::min<uint64_t>((csz + 3) / 4, (uint64_t)ctx->sms * wper);
    KIRA_DBUF(fb, uint32_t, B_WFA_FB, csz);
    L.fb_list = fb;
    // Fallback launch shape: 32 lanes per pair, up to 4 warps (pairs) per block; it
    // uses no more groups than the scratch above holds.
    while (fwpb > 1 && (uint64_t)fwpb * L.smem_group > (160u << 10)) fwpb >>= 1;
    int fper = 0;
    KIRA_CUDA(wfa_blocks_per_sm(32, tb, (size_t)fwpb * L.smem_group, (int)(32 * fwpb), &fper));
    if (fper < 1) return fail(ctx, KIRA_ERR_INVALID, "WFA fallback: %u shared bytes", L.smem_group);
    L.fb_count = work + 3;
    if (tb) {
      KIRA_DBUF(wh, int16_t, B_WFA_WHIST,
                wblocks * 4 * (uint64_t)(win_smax + 1) * 3 * 32 * win_segments);
      L.win_hist = wh;
    }
  }
  uint32_t *ncig = nullptr, *off = nullptr, *sums = nullptr, *ops = nullptr;
  if (tb) {
    KIRA_DBUF(nc, uint32_t, B_WFA_NCIG, n);
    KIRA_DBUF(sl, uint32_t, B_WFA_SLOTS, (uint64_t)n * L.slot_cap);
    KIRA_DBUF(of, uint32_t, B_CIG_OFF, n);
    KIRA_DBUF(su, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
    KIRA_DBUF(dops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(cigar->cap, 1));
    ncig = nc, off = of, sums = su, ops = dops;
    L.slots = sl;
  }
  KIRA_CUDA(cudaMemsetAsync(work, 0, 16, st));
  KIRA_CUDA(cudaMemsetAsync(total_dev, 0, 8, st));
  if (chunked) {  // copies start once the buffers exist and the counters are reset
    KIRA_CUDA(cudaEventRecord(ctx->ev_up[nch], st));
    KIRA_CUDA(cudaStreamWaitEvent(ctx->h2d, ctx->ev_up[nch], 0));
  }
  mark(ctx, 1, st);
  for (uint32_t c = 0; chunked && c < nch; ++c) {
    rc = chunked_upload(ctx, P, ci, c, [&](uint32_t l, uint32_t k, cudaStream_t up) -> int {
      if (dms) KIRA_CUDA(cudaMemcpyAsync(dms + l, max_score + l, 4ull * k, cudaMemcpyHostToDevice, up));
      if (dtbf)
        KIRA_CUDA(cudaMemcpyAsync(dtbf + l, text_begin_free + l, 4ull * k, cudaMemcpyHostToDevice, up));
      return KIRA_OK;
    });
    if (rc) return rc;
  }
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t lo = c * csz, m = std::min(n, lo + csz) - lo;
    if (chunked) KIRA_CUDA(cudaStreamWaitEvent(st, ctx->ev_up[c], 0));
    if (c) {  // fetch counters of both kernels and the fallback count
      KIRA_CUDA(cudaMemsetAsync(work, 0, 4, st));
      KIRA_CUDA(cudaMemsetAsync(work + 2, 0, 8, st));
    }
    WfaLaunch Lc = L;
    Lc.n = m;
    Lc.out = dout + lo;
    Lc.max_score_pp = dms ? dms + lo : nullptr;
    Lc.tbf_pp = dtbf ? dtbf + lo : nullptr;
    if (tb) {
      Lc.ncig = ncig + lo;
      Lc.slots = L.slots + (size_t)lo * L.slot_cap;
    }
    const DevPairs Dc = chunk_view(D, lo, m);
    if (use_window) {
      // Window kernel first; its fallbacks (pairs still open at win_smax) run
      // through the general kernel over the fallback list.
      Lc.work = work;
      KIRA_CUDA(launch_wfa_window(Dc, Lc, (uint32_t)std::min<uint64_t>(wblocks, (m + 3) / 4), tb,
                                  st));
      Lc.list = L.fb_list;
      Lc.list_count = L.fb_count;
      Lc.group = 32;
      Lc.work = work + 2;
      KIRA_CUDA(launch_wfa(Dc, Lc,
                           (uint32_t)std::max<uint64_t>(
                               1, std::min<uint64_t>(blocks * gpb / fwpb, (m + fwpb - 1) / fwpb)),
                           fwpb, tb, st));
    } else {
      Lc.work = work + 2;
      const uint32_t bl = (uint32_t)std::min<uint64_t>(blocks, (m + gpb - 1) / gpb);
      KIRA_CUDA(launch_wfa(Dc, Lc, bl, wpb, tb, st));
    }
    mark(ctx, 2, st);
    if (tb) {
      KIRA_CUDA(launch_cigar_scan(ncig + lo, m, off + lo, sums, total_dev, st, true));
      WfaCompact C{m, dout + lo, ncig + lo, off + lo, Lc.slots, L.slot_cap, ops, cigar->cap};
      KIRA_CUDA(launch_wfa_compact(C, ctx->sms, st));
    }
    if (chunked) KIRA_CUDA(cudaEventRecord(ctx->ev_comp[c], st));
  }
  for (uint32_t c = 0; chunked && c < nch; ++c) {
    const uint32_t lo = c * csz, m = std::min(n, lo + csz) - lo;
    KIRA_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->ev_comp[c], 0));
    KIRA_CUDA(cudaMemcpyAsync(out + lo, dout + lo, sizeof(kira_wfa_result) * m,
                              cudaMemcpyDeviceToHost, ctx->d2h));
  }
  mark(ctx, 3, st);
  cudaStream_t dn = chunked ? ctx->d2h : st;
  uint64_t total = 0;
  uint32_t flags = 0;
  KIRA_CUDA(cudaMemcpyAsync(&flags, work + 1, 4, cudaMemcpyDeviceToHost, dn));
  if (tb) KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, dn));
  if (!chunked)
    KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_wfa_result) * n, cudaMemcpyDeviceToHost, dn));
  KIRA_CUDA(cudaStreamSynchronize(dn));
  if (flags & 2u) return fail(ctx, KIRA_ERR_RUNTIME, "WFA history above its computed bound");
  if (flags & 1u) return fail(ctx, KIRA_ERR_RUNTIME, "WFA CIGAR above its computed bound");
  if (!tb) {
    mark(ctx, 4, st);
    return KIRA_OK;
  }
  cigar->used = total;
  if (total > cigar->cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "CIGAR buffer holds %llu ops, %llu needed",
                (unsigned long long)cigar->cap, (unsigned long long)total);
  if (total) KIRA_CUDA(cudaMemcpyAsync(cigar->ops, ops, 4ull * total, cudaMemcpyDeviceToHost, dn));
  mark(ctx, 4, st);
  KIRA_CUDA(cudaStreamSynchronize(dn));
  return KIRA_OK;
}

namespace {

// Chains that reach ungapped_extend must lie inside their read and window: the
// reference's u32 subtractions and slices panic otherwise (prefilter.rs:362-364).
int check_chains(kira_ctx* ctx, const kira_pairs& P, const kira_chain* chains,
                 uint32_t* max_read_len) {
  std::vector<int64_t> bad(host_parts(P.n), -1);
  std::vector<int> kind(host_parts(P.n), 0);
  std::vector<uint32_t> qmax(host_parts(P.n), 0);
  host_for(ctx, P.n, [&](uint32_t lo, uint32_t hi, uint32_t k) {
    uint32_t q = 0;
    for (uint32_t i = lo; i < hi; ++i) q = P.read_len[i] > q ? P.read_len[i] : q;
    qmax[k] = q;
    for (uint32_t i = lo; i < hi; ++i) {
      const kira_chain& c = chains[i];
      const bool extends = P.read_len[i] > 0 && c.read_start <= c.read_end &&
                           c.ref_start <= c.ref_end && c.read_end > c.read_start;
      const bool outside = extends && (c.read_end > P.read_len[i] || c.ref_end > P.win_len[i]);
      if (P.read_len[i] > 65535u || outside) {
        bad[k] = i;
        kind[k] = P.read_len[i] > 65535u ? 1 : 2;
        return;
      }
    }
  });
  *max_read_len = 0;
  for (const uint32_t q : qmax) *max_read_len = std::max(*max_read_len, q);
  for (size_t k = 0; k < bad.size(); ++k) {
    if (bad[k] < 0) continue;
    if (kind[k] == 1)
      return fail(ctx, KIRA_ERR_READ_TOO_LONG, "pair %u: reads up to 65535 bases", (uint32_t)bad[k]);
    return fail(ctx, KIRA_ERR_INVALID, "chain %u ends outside its read or window", (uint32_t)bad[k]);
  }
  return KIRA_OK;
}

// (accept_min_identity * 100.0).round() as u16 (prefilter.rs:266): f32 product,
// rounding half away from zero, saturating cast (NaN -> 0).
int32_t identity_floor(float pct) {
  const float v = pct * 100.0f;
  if (!(v == v)) return 0;
  const float r = std::round(v);
  return r <= 0.0f ? 0 : (r >= 65535.0f ? 65535 : (int32_t)r);
}

}  // namespace

int kira_gpu_prefilter_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_chain* chains,
                             const uint8_t* is_top1, const int32_t* score_margin,
                             const kira_prefilter_cfg* cfg, kira_prefilter_result* out,
                             kira_cigar_buf* cigar, char* md, uint64_t md_cap,
                             uint64_t* md_used) {
  if (!ctx || !pairs || !chains || !cfg || !out || !cigar || !md_used) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  const uint32_t n = P.n;
  cigar->used = 0;
  *md_used = 0;
  if (n == 0) return KIRA_OK;
  if ((cigar->cap && !cigar->ops) || (md_cap && !md)) return KIRA_ERR_INVALID;
  uint32_t q_max = 0;
  int rc = check_chains(ctx, P, chains, &q_max);
  if (rc) return rc;
  PrefilterLaunch L{};
  L.match = cfg->match_score;
  L.mismatch = cfg->mismatch;
  L.xdrop = cfg->xdrop;
  L.accept_enable = cfg->accept_enable != 0;
  L.only_top1 = cfg->accept_only_top1 != 0;
  L.multi = cfg->multi_alignments_enabled != 0;
  L.tail = cfg->tail != 0;
  L.exact_first = cfg->exact_first != 0;
  L.span_slack = cfg->accept_span_slack;
  L.max_mismatches = cfg->accept_max_mismatches;
  L.long_read_threshold = cfg->long_read_threshold;
  L.require_margin = cfg->accept_require_score_margin;
  L.identity_floor = cfg->min_identity_x10000 >= 0 ? cfg->min_identity_x10000
                                                   : identity_floor(cfg->accept_min_identity);
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);
  cudaError_t cerr = cudaSuccess;
  // Large host batches go chunk by chunk (uploads, kernels and downloads overlap);
  // CIGAR and MD offsets continue through running totals, and pass 2 writes only
  // what fits the caller's buffers, so no chunk waits for the host.
  const uint64_t chunked = host_chunk(ctx, n);
  ChunkedInput ci;
  DevPairs D;
  rc = chunked ? chunked_plan(ctx, P, chunked, ci) : upload_pairs(ctx, P, D);
  if (rc) return rc;
  if (chunked) D = ci.D;
  KIRA_DBUF(dch, kira_chain, B_PF_CHAINS, n);
  uint8_t* dtop = nullptr;
  int32_t* dmar = nullptr;
  if (is_top1) {
    KIRA_DBUF(b, uint8_t, B_PF_TOP1, n);
    dtop = b;
  }
  if (score_margin) {
    KIRA_DBUF(b, int32_t, B_PF_MARGIN, n);
    dmar = b;
  }
  if (!chunked) {
    KIRA_CUDA(cudaMemcpyAsync(dch, chains, sizeof(kira_chain) * n, cudaMemcpyHostToDevice, st));
    if (dtop) KIRA_CUDA(cudaMemcpyAsync(dtop, is_top1, n, cudaMemcpyHostToDevice, st));
    if (dmar) KIRA_CUDA(cudaMemcpyAsync(dmar, score_margin, 4ull * n, cudaMemcpyHostToDevice, st));
  }
  KIRA_DBUF(dout, kira_prefilter_result, B_PF_OUT, n);
  KIRA_DBUF(ncig, uint32_t, B_PF_NCIG, n);
  KIRA_DBUF(mdlen, uint32_t, B_PF_MDLEN, n);
  KIRA_DBUF(cig_off, uint32_t, B_CIG_OFF, n);
  KIRA_DBUF(md_off, uint32_t, B_PF_MDOFF, n);
  KIRA_DBUF(sums, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
  KIRA_DBUF(totals, uint64_t, B_TOTAL, 2);
  KIRA_DBUF(flags, uint32_t, B_WORK, 1);
  const uint64_t ops_cap = std::min<uint64_t>(cigar->cap, 3ull * n);
  KIRA_DBUF(ops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(ops_cap, 1));
  // An ungapped span of L columns has at most 2L + 1 MD bytes (all mismatches).
  const uint64_t md_dev = std::min<uint64_t>(md_cap, (uint64_t)n * (2ull * q_max + 8));
  KIRA_DBUF(dmd, char, B_PF_MD, std::max<uint64_t>(md_dev, 1));
  L.ncig = ncig;
  L.mdlen = mdlen;
  L.flags = flags;
  L.ops = ops;
  L.cigar_cap = ops_cap;
  L.md = dmd;
  L.md_cap = md_dev;
  KIRA_CUDA(cudaMemsetAsync(flags, 0, 4, st));
  KIRA_CUDA(cudaMemsetAsync(totals, 0, 16, st));
  const uint32_t csz = chunked ? ci.chunk : n, nch = chunked ? ci.nch : 1;
  if (chunked) {
    KIRA_CUDA(cudaEventRecord(ctx->ev_up[nch], st));
    KIRA_CUDA(cudaStreamWaitEvent(ctx->h2d, ctx->ev_up[nch], 0));
  }
  mark(ctx, 1, st);
  for (uint32_t c = 0; chunked && c < nch; ++c) {
    rc = chunked_upload(ctx, P, ci, c, [&](uint32_t l, uint32_t k, cudaStream_t up) -> int {
      KIRA_CUDA(cudaMemcpyAsync(dch + l, chains + l, sizeof(kira_chain) * k,
                                cudaMemcpyHostToDevice, up));
      if (dtop) KIRA_CUDA(cudaMemcpyAsync(dtop + l, is_top1 + l, k, cudaMemcpyHostToDevice, up));
      if (dmar)
        KIRA_CUDA(cudaMemcpyAsync(dmar + l, score_margin + l, 4ull * k, cudaMemcpyHostToDevice, up));
      return KIRA_OK;
    });
    if (rc) return rc;
  }
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t lo = c * csz, m = std::min(n, lo + csz) - lo;
    if (chunked) KIRA_CUDA(cudaStreamWaitEvent(st, ctx->ev_up[c], 0));
    const DevPairs Dc = chunk_view(D, lo, m);
    PrefilterLaunch Lc = L;
    Lc.chains = dch + lo;
    Lc.is_top1 = dtop ? dtop + lo : nullptr;
    Lc.score_margin = dmar ? dmar + lo : nullptr;
    Lc.out = dout + lo;
    Lc.ncig = ncig + lo;
    Lc.mdlen = mdlen + lo;
    KIRA_CUDA(launch_prefilter(Dc, Lc, false, ctx->sms, st));
    mark(ctx, 2, st);
    KIRA_CUDA(launch_cigar_scan(ncig + lo, m, cig_off + lo, sums, totals, st, true));
    KIRA_CUDA(launch_cigar_scan(mdlen + lo, m, md_off + lo, sums, totals + 1, st, true));
    KIRA_CUDA(launch_prefilter_offsets(m, dout + lo, cig_off + lo, md_off + lo, ctx->sms, st));
    mark(ctx, 3, st);
    KIRA_CUDA(launch_prefilter(Dc, Lc, true, ctx->sms, st));
    mark(ctx, 4, st);
    if (chunked) KIRA_CUDA(cudaEventRecord(ctx->ev_comp[c], st));
  }
  for (uint32_t c = 0; chunked && c < nch; ++c) {
    const uint32_t lo = c * csz, m = std::min(n, lo + csz) - lo;
    KIRA_CUDA(cudaStreamWaitEvent(ctx->d2h, ctx->ev_comp[c], 0));
    KIRA_CUDA(cudaMemcpyAsync(out + lo, dout + lo, sizeof(kira_prefilter_result) * m,
                              cudaMemcpyDeviceToHost, ctx->d2h));
  }
  cudaStream_t dn = chunked ? ctx->d2h : st;
  uint64_t tot[2] = {0, 0};
  uint32_t hflags = 0;
  KIRA_CUDA(cudaMemcpyAsync(tot, totals, 16, cudaMemcpyDeviceToHost, dn));
  KIRA_CUDA(cudaMemcpyAsync(&hflags, flags, 4, cudaMemcpyDeviceToHost, dn));
  if (!chunked)
    KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_prefilter_result) * n,
                              cudaMemcpyDeviceToHost, dn));
  KIRA_CUDA(cudaStreamSynchronize(dn));
  if (hflags & 1u) return fail(ctx, KIRA_ERR_RUNTIME, "a chain ended outside its read or window");
  cigar->used = tot[0];
  *md_used = tot[1];
  if (tot[0] > cigar->cap || tot[1] > md_cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "CIGAR / MD buffers hold %llu ops / %llu bytes; "
                "%llu / %llu needed", (unsigned long long)cigar->cap,
                (unsigned long long)md_cap, (unsigned long long)tot[0],
                (unsigned long long)tot[1]);
  if (tot[0])
    KIRA_CUDA(cudaMemcpyAsync(cigar->ops, ops, 4ull * tot[0], cudaMemcpyDeviceToHost, dn));
  if (tot[1]) KIRA_CUDA(cudaMemcpyAsync(md, dmd, tot[1], cudaMemcpyDeviceToHost, dn));
  mark(ctx, 5, st);
  KIRA_CUDA(cudaStreamSynchronize(dn));
  return KIRA_OK;
}

int kira_gpu_exact_match_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_chain* chains,
                               uint8_t* out) {
  if (!ctx || !pairs || !chains || !out) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  const uint32_t n = P.n;
  if (n == 0) return KIRA_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  DevPairs D;
  int rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  cudaError_t cerr = cudaSuccess;
  KIRA_DBUF(dch, kira_chain, B_PF_CHAINS, n);
  KIRA_DBUF(dout, uint8_t, B_PF_EXACT, n);
  KIRA_CUDA(cudaMemcpyAsync(dch, chains, sizeof(kira_chain) * n, cudaMemcpyHostToDevice, st));
  KIRA_CUDA(launch_exact_match(D, dch, dout, ctx->sms, st));
  KIRA_CUDA(cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  return KIRA_OK;
}

int kira_gpu_set_wfa_lanes(kira_ctx* ctx, int lanes) {
  if (!ctx || (lanes != 0 && lanes != 8 && lanes != 16 && lanes != 32)) return KIRA_ERR_INVALID;
  ctx->wfa_lanes = lanes;
  return KIRA_OK;
}

int kira_gpu_set_chunk_pairs(kira_ctx* ctx, int64_t pairs) {
  if (!ctx || pairs > UINT32_MAX) return KIRA_ERR_INVALID;
  ctx->chunk_pairs = pairs < 0 ? -1 : pairs;
  return KIRA_OK;
}

uint32_t kira_gpu_bsw_rounds(const kira_ctx* ctx) { return ctx ? ctx->last_rounds : 0; }

int kira_gpu_set_trace_budget(kira_ctx* ctx, uint64_t bytes) {
  if (!ctx) return KIRA_ERR_INVALID;
  ctx->trace_budget = bytes;
  return KIRA_OK;
}

int kira_gpu_bsw_shapes(int* lanes, int* cells, int* packed, int max_shapes) {
  const int n = std::min(max_shapes, kNumBswShapes);
  for (int i = 0; i < n; ++i) {
    if (lanes) lanes[i] = kBswShapes[i].g;
    if (cells) cells[i] = shape_cap(kBswShapes[i]) / kBswShapes[i].g;
    if (packed) packed[i] = kBswShapes[i].packed;
  }
  return kNumBswShapes;
}

int kira_gpu_profile(kira_ctx* ctx, int enable) {
  if (!ctx) return KIRA_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (enable && !ctx->ev[0])
    for (auto& e : ctx->ev) KIRA_CUDA(cudaEventCreate(&e));
  ctx->profile = enable != 0;
  ctx->ev_recorded = 0;
  return KIRA_OK;
}

int kira_gpu_stage_times(kira_ctx* ctx, float* ms, int max_stages) {
  if (!ctx || !ms) return -KIRA_ERR_INVALID;
  if (!ctx->profile || ctx->ev_recorded < 2) return 0;
  const int n = std::min(ctx->ev_recorded - 1, max_stages);
  for (int i = 0; i < n; ++i) {
    if (cudaEventSynchronize(ctx->ev[i + 1]) != cudaSuccess) return -KIRA_ERR_RUNTIME;
    if (cudaEventElapsedTime(ms + i, ctx->ev[i], ctx->ev[i + 1]) != cudaSuccess) ms[i] = -1.0f;
  }
  return n;
}

int kira_gpu_ref_upload(kira_ctx* ctx, const uint8_t* seq, uint64_t len) {
  if (!ctx) return KIRA_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->ref_owner.reset();
  ctx->ref_dev = nullptr;
  ctx->ref_planes = nullptr;
  ctx->ref_len = 0;
  if (len == 0) return KIRA_OK;
  uint8_t* dev = nullptr;
  uint4* planes = nullptr;
  const int device = ctx->device;
  KIRA_CUDA(cudaMalloc(&dev, len + 16));
  const uint64_t nb = plane_blocks(len);
  cudaError_t e = cudaMalloc(&planes, nb * sizeof(uint4));
  if (e != cudaSuccess) {
    cudaFree(dev);
    return cuda_fail(ctx, e, "cudaMalloc(reference planes)");
  }
  // One holder frees both arrays when the last context sharing them lets go.
  ctx->ref_owner = std::shared_ptr<void>(dev, [device, planes](void* p) {
    cudaSetDevice(device);
    cudaFree(p);
    cudaFree(planes);
  });
  ctx->ref_dev = dev;
  ctx->ref_planes = planes;
  KIRA_CUDA(cudaMemcpy(ctx->ref_dev, seq, len, cudaMemcpyHostToDevice));
  KIRA_CUDA(cudaMemsetAsync(ctx->ref_dev + len, 0, 16, ctx->stream));
  KIRA_CUDA(launch_pack_planes(ctx->ref_dev, len, ctx->ref_planes, nb, ctx->sms, ctx->stream));
  KIRA_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->ref_len = len;
  return KIRA_OK;
}

int kira_gpu_myers_batch(kira_ctx* ctx, const kira_pairs* pairs, uint32_t max_k, int32_t* dist,
                         int32_t* end_pos) {
  if (!ctx || !pairs) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  if (P.n == 0) return KIRA_OK;
  cudaSetDevice(ctx->device);
  const Maxes mx = host_maxes(ctx, P, 1);
  if (mx.q > 512) return fail(ctx, KIRA_ERR_INVALID, "pattern of %u bases > 512", mx.q);
  DevPairs D;
  int rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  cudaError_t cerr = cudaSuccess;
  KIRA_DBUF(dd, int32_t, B_DIST, P.n);
  KIRA_DBUF(de, int32_t, B_END, P.n);
  KIRA_DBUF(counters, uint32_t, B_COUNTERS, 4);
  KIRA_CUDA(cudaMemsetAsync(counters, 0, 16, ctx->stream));
  rc = build_planes(ctx, D, P.read_seq_bytes, P.win_seq_bytes, P.win_seq == nullptr, ctx->stream);
  if (rc) return rc;
  MyersLaunch M{};
  M.flags = counters + 2;
  M.count = P.n;
  M.k = (int32_t)max_k;
  M.per_pair_k = 0;
  M.tw = std::max<uint32_t>((mx.w + 31) / 32, 1);
  M.lmax = std::max<uint32_t>((mx.q + 31) / 32, 1);
  M.dist = dd;
  M.end = de;
  cudaStream_t st = ctx->stream;
  KIRA_CUDA(launch_myers(D, M, P.n, ctx->sms, st));
  KIRA_CUDA(cudaMemcpyAsync(dist, dd, 4ull * P.n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(end_pos, de, 4ull * P.n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  return KIRA_OK;
}

int kira_gpu_bsw_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                       kira_sw_result* out, kira_cigar_buf* cigar, uint64_t* cells) {
  if (!ctx || !pairs || !cfg || !out || !cigar) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  cigar->used = 0;
  if (cells) *cells = 0;
  if (P.n == 0) return KIRA_OK;
  cudaSetDevice(ctx->device);
  const Maxes mx = host_maxes(ctx, P, cfg->bandwidth);
  int rc = check_sw_cfg(ctx, *cfg, mx.q, mx.band);
  if (rc) return rc;
  DevPairs D;
  cudaStream_t st = ctx->stream;
  ctx->ev_recorded = 0;
  mark(ctx, 0, st);
  rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  mark(ctx, 1, st);
  cudaError_t cerr = cudaSuccess;
  const uint32_t n = P.n;
  KIRA_DBUF(dout, kira_sw_result, B_OUT, n);
  KIRA_DBUF(ncig, uint32_t, B_NCIG, n);
  KIRA_DBUF(counters, uint32_t, B_COUNTERS, 4);
  KIRA_DBUF(cells_dev, unsigned long long, B_CELLS, 1);
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  KIRA_DBUF(ops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(cigar->cap, 1));
  KIRA_CUDA(cudaMemsetAsync(counters, 0, 16, st));
  KIRA_CUDA(cudaMemsetAsync(cells_dev, 0, 8, st));
  BswLaunch B{};
  if (ctx->plain) {
    // The one-launch comparator: the same kernel choice the bucketed path makes for
    // the batch's widest band (the tuned shape of its class when the batch fits it,
    // packed int16 wherever the scores fit, else int32), one launch over every pair
    // in input order; only the bucketing, dynamic fetch and graph replay differ.
    const SwParams sp = resolve(*cfg);
    const int shape = pick_shape(ctx, mx.band, mx.q, sp);
    if (shape < 0)
      return fail(ctx, KIRA_ERR_INVALID, "band %u above the one-launch maximum", mx.band);
    const uint32_t per_round = round_items(ctx, n, shape, mx.q);
    ctx->last_rounds = (n + per_round - 1) / per_round;
    rc = prepare_bsw(ctx, n, n, per_round, mx, shape, B);
    if (rc) return rc;
    B.count = n;
    B.sp = sp;
    B.bias = packed_bias(kBswShapes[shape], sp);
    B.offset = D.band_offset;
    B.cells = cells_dev;
    B.out = dout;
    B.ncig = ncig;
    B.flags = counters + 2;
    mark(ctx, 2, st);
    KIRA_CUDA(launch_bsw_rounds(shape, D, B, n, per_round, ctx->sms, st,
                                ctx->profile ? ctx->ev[3] : nullptr));
    if (ctx->profile) ctx->ev_recorded = 4;
    mark(ctx, 4, st);
    rc = finish_cigars(ctx, n, dout, ncig, B, ops, cigar->cap, total_dev, st);
    if (rc) return rc;
  } else {
    BucketRun R;
    rc = plan_bucketed(ctx, P, D, *cfg, dout, ncig, counters + 2, cells_dev, B, R, st);
    if (rc) return rc;
    KIRA_DBUF(off, uint32_t, B_CIG_OFF, std::max<uint32_t>(n, 1));
    KIRA_DBUF(sums, uint32_t, B_CHUNK_SUMS, n / 4096 + 2);
    CompactLaunch CL{n, dout, ncig, off, B.item_of_pair, B.cig_slots, B.slot_cap, ops, cigar->cap};
    auto enqueue_all = [&]() -> cudaError_t {
      cudaError_t e = enqueue_bucketed(ctx, D, R, st);
      if (e == cudaSuccess) e = launch_cigar_scan(ncig, n, off, sums, total_dev, st);
      if (e == cudaSuccess) e = launch_cigar_compact(CL, ctx->sms, st);
      return e;
    };
    if (ctx->graphs && !ctx->profile) {
      KIRA_CUDA(run_as_graph(ctx, D, R, CL, total_dev, st, enqueue_all));
    } else {
      KIRA_CUDA(enqueue_all());
    }
  }
  mark(ctx, 5, st);
  uint64_t total = 0;
  unsigned long long hcells = 0;
  uint32_t flags[4];
  KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_sw_result) * n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&hcells, cells_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(flags, counters, 16, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  cigar->used = total;
  if (cells) *cells = hcells;
  if (flags[2] & 1u) return fail(ctx, KIRA_ERR_RUNTIME, "CIGAR slot overflow");
  if (flags[2] & 6u) return fail(ctx, KIRA_ERR_INVALID, "a pair exceeded the launch's length bounds");
  if (total > cigar->cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "CIGAR buffer holds %llu ops, %llu needed",
                (unsigned long long)cigar->cap, (unsigned long long)total);
  if (total) {
    KIRA_CUDA(cudaMemcpyAsync(cigar->ops, ops, 4ull * total, cudaMemcpyDeviceToHost, st));
    KIRA_CUDA(cudaStreamSynchronize(st));
  }
  return KIRA_OK;
}

// i16 fit check of sw_batch_avx2 (src/alignment/mod.rs:1854-1868).
static bool i16_fits(uint32_t q, uint32_t r, const kira_sw_cfg& c) {
  const int64_t mx = 32767;
  const bool costs = c.match_score >= 0 && c.match_score <= mx && c.mismatch >= 0 &&
                     c.mismatch <= mx && c.gap_open >= 0 && c.gap_extend >= 0 &&
                     (int64_t)c.gap_open + c.gap_extend <= mx;
  if (!costs || q > mx || r > mx) return false;
  return (int64_t)std::min(q, r) * c.match_score <= mx;
}

// int8_path_viable (src/alignment/sw_int8_vnni.rs:47-55).
static bool int8_viable(uint32_t q, const kira_sw_cfg& c) {
  const int64_t ms = std::max(c.match_score, 1);
  auto in = [](int32_t v) { return v >= 0 && v <= 32; };
  return (int64_t)q * ms < 120 && in(c.match_score) && in(c.mismatch) && in(c.gap_open) &&
         in(c.gap_extend);
}

int kira_gpu_align_batch_simd(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                              int mode, int detected, kira_sw_result* out, kira_cigar_buf* cigar) {
  if (!ctx || !pairs || !cfg || !out || !cigar) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  cigar->used = 0;
  if (P.n == 0) return KIRA_OK;  // mod.rs:1116-1118
  cudaSetDevice(ctx->device);
  const uint32_t n = P.n;
  const uint32_t q0 = P.read_len[0], r0 = P.win_len[0];
  bool mixed = false;
  for (uint32_t i = 0; i < n && !mixed; ++i) mixed = P.read_len[i] != q0 || P.win_len[i] != r0;
  // Which kernel the reference dispatch (mod.rs:1131-1149, 1824-1841) would run.
  uint32_t group = 0;  // 0: scalar banded for every input
  if (!mixed) {
    if (mode == KIRA_SIMD_AVX_VNNI && detected == KIRA_SIMD_AVX_VNNI) {
      group = (int8_viable(q0, *cfg) && n <= 32) ? 32u : 16u;
    } else if (mode == KIRA_SIMD_AVX2 &&
               (detected == KIRA_SIMD_AVX2 || detected == KIRA_SIMD_AVX_VNNI)) {
      group = 16u;
    }
    if (group == 16u && !i16_fits(q0, r0, *cfg)) group = 0;  // per-chunk scalar fallback
  }
  if (group == 0) return kira_gpu_bsw_batch(ctx, pairs, cfg, out, cigar, nullptr);
  // Full-window kernel.
  const int cap_need = (int)r0;
  int shape = -1;
  for (int s = 0; s < kNumBswShapes; ++s)
    if (!kBswShapes[s].packed && shape_cap(kBswShapes[s]) >= cap_need) {
      shape = s;
      break;
    }
  if (shape < 0)
    return fail(ctx, KIRA_ERR_INVALID, "full-window batch: window of %u > supported 544", r0);
  if (cfg->gap_open < 0 || cfg->gap_extend < 0)
    return fail(ctx, KIRA_ERR_INVALID, "gap costs must be >= 0");
  DevPairs D;
  int rc = upload_pairs(ctx, P, D);
  if (rc) return rc;
  cudaError_t cerr = cudaSuccess;
  cudaStream_t st = ctx->stream;
  Maxes mx;
  mx.q = q0;
  mx.w = r0;
  mx.band = 1;
  KIRA_DBUF(dout, kira_sw_result, B_OUT, n);
  KIRA_DBUF(ncig, uint32_t, B_NCIG, n);
  KIRA_DBUF(counters, uint32_t, B_COUNTERS, 4);
  KIRA_DBUF(total_dev, uint64_t, B_TOTAL, 1);
  KIRA_DBUF(ops, uint32_t, B_CIGAR_OUT, std::max<uint64_t>(cigar->cap, 1));
  KIRA_CUDA(cudaMemsetAsync(counters, 0, 16, st));
  BswLaunch B{};
  rc = prepare_bsw(ctx, n, n, n, mx, shape, B);
  if (rc) return rc;
  bool any_abort = false;
  if (P.abort_score)
    for (uint32_t i = 0; i < n && !any_abort; ++i) any_abort = P.abort_score[i] > kAbortOff;
  B.count = n;
  B.sp = resolve(*cfg);
  B.out = dout;
  B.ncig = ncig;
  B.flags = counters + 2;
  B.full = 1;
  B.group = group;
  if (any_abort) {
    KIRA_DBUF(keys, uint32_t, B_ROWKEYS, (uint64_t)(mx.q + 1) * n);
    KIRA_DBUF(done, uint32_t, B_DONE_ROW, n);
    B.rowkeys = keys;
    B.done_row = done;
  }
  KIRA_CUDA(launch_bsw(shape, D, B, n, ctx->sms, st));
  rc = finish_cigars(ctx, n, dout, ncig, B, ops, cigar->cap, total_dev, st);
  if (rc) return rc;
  uint64_t total = 0;
  uint32_t flags[4];
  KIRA_CUDA(cudaMemcpyAsync(out, dout, sizeof(kira_sw_result) * n, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(&total, total_dev, 8, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaMemcpyAsync(flags, counters, 16, cudaMemcpyDeviceToHost, st));
  KIRA_CUDA(cudaStreamSynchronize(st));
  cigar->used = total;
  if (flags[2]) return fail(ctx, KIRA_ERR_RUNTIME, "full-window batch outside its launch shape");
  if (total > cigar->cap)
    return fail(ctx, KIRA_ERR_CAPACITY, "CIGAR buffer holds %llu ops, %llu needed",
                (unsigned long long)cigar->cap, (unsigned long long)total);
  if (total) {
    KIRA_CUDA(cudaMemcpyAsync(cigar->ops, ops, 4ull * total, cudaMemcpyDeviceToHost, st));
    KIRA_CUDA(cudaStreamSynchronize(st));
  }
  return KIRA_OK;
}

int kira_gpu_verify_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_verify_params* p,
                          kira_sw_result* out, kira_cigar_buf* cigar, kira_verify_detail* detail,
                          uint64_t* cells) {
  if (!ctx || !pairs || !p || !out || !cigar) return KIRA_ERR_INVALID;
  return verify_host(ctx, *pairs, *p, out, cigar, detail, cells, nullptr);
}

int kira_gpu_verify_batch_compact(kira_ctx* ctx, const kira_pairs* pairs,
                                  const kira_verify_params* p, uint8_t* status,
                                  kira_sw_result* rows, uint64_t rows_cap, uint64_t* rows_used,
                                  kira_cigar_buf* cigar, uint64_t* cells) {
  if (!ctx || !pairs || !p || !status || (!rows && rows_cap) || !rows_used || !cigar)
    return KIRA_ERR_INVALID;
  *rows_used = 0;
  const CompactOut co{status, rows, rows_cap, rows_used};
  return verify_host(ctx, *pairs, *p, nullptr, cigar, nullptr, cells, &co);
}

int kira_gpu_verify_dev(kira_ctx* ctx, const kira_pairs* pairs, const kira_verify_params* p,
                        kira_sw_result* out, uint32_t* cigar_ops, uint64_t cigar_cap,
                        uint64_t* cigar_used_dev, kira_verify_detail* detail,
                        unsigned long long* cells_dev, void* stream) {
  if (!ctx || !pairs || !p || !out || !cigar_used_dev) return KIRA_ERR_INVALID;
  const kira_pairs& P = *pairs;
  if (P.n == 0) return KIRA_OK;
  if (!P.max_read_len || !P.max_win_len)
    return fail(ctx, KIRA_ERR_INVALID, "device batches need max_read_len and max_win_len");
  cudaSetDevice(ctx->device);
  Maxes mx;
  mx.q = P.max_read_len;
  mx.w = P.max_win_len;
  mx.band = P.bandwidth ? P.max_bandwidth : (uint32_t)std::max(p->sw.bandwidth, 1);
  if (!mx.band) return fail(ctx, KIRA_ERR_INVALID, "per-pair bandwidth needs max_bandwidth");
  DevPairs D{P.n, P.read_seq, P.read_off, P.read_len,
             P.win_seq ? P.win_seq : ctx->ref_dev, P.win_off, P.win_len,
             P.band_offset, P.abort_score, P.bandwidth, nullptr, nullptr};
  return verify_pipeline(ctx, D, mx, *p, P.read_seq_bytes, P.win_seq_bytes, P.win_seq == nullptr,
                         out, cigar_ops, cigar_cap, cigar_used_dev, detail, cells_dev,
                         (cudaStream_t)stream);
}

}  // extern "C"

namespace kira {
// Makes `dst` use `src`'s resident reference (shared, freed with the last holder).
int ctx_share_reference(kira_ctx* dst, const kira_ctx* src) {
  if (!dst || !src || dst->device != src->device) return KIRA_ERR_INVALID;
  dst->ref_owner = src->ref_owner;
  dst->ref_dev = src->ref_dev;
  dst->ref_planes = src->ref_planes;
  dst->ref_len = src->ref_len;
  return KIRA_OK;
}
}  // namespace kira
