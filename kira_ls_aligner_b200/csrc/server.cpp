// server.cpp -- continuous-batching request server over libkira_gpu contexts.
//
// Requests (a batch of short read x window pairs for the composed verification,
// or of long gap-fill segments for banded SW) are submitted from any host thread
// and answered asynchronously through tickets. The server owns `slots` worker
// threads, each with its own kira_ctx (stream + grow-only device arena); all
// contexts share one device-resident reference. A free slot takes the oldest
// queued request plus every later queued request of the same kind and the same
// parameters, up to max_batch_pairs, concatenates them into one batch, runs the
// library's pipeline on its stream and scatters each request's results into the
// caller's buffers. Requests that arrive while other batches are on the GPU are
// picked up by the next free slot, and the slots' streams overlap on the device.
//
// Admission: a batch starts only when its device-memory estimate fits in
// mem_fraction of the currently free device memory plus what the slot already
// holds; otherwise the batch is cut to the requests that fit, and a single
// request that does not fit waits (bounded, re-checked) while other slots are
// busy. Each slot's banded-SW trace arena is capped at its share of the budget,
// so longer batches run in trace rounds instead of failing.
//
// A pair's result does not depend on which other pairs share its batch, so a
// request's results are identical alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kira_gpu.h"

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace kira {
int ctx_share_reference(kira_ctx* dst, const kira_ctx* src);  // api.cu
}

namespace {

// Copies into pinned staging memory with streaming stores where the host has them
// (x86 SSE2): the copy engine reads lines the CPU left dirty in its caches several
// times slower than lines in memory. stage_fence() orders the stores before the
// staged arrays are handed to the upload.
void stage_copy(void* dst, const void* src, size_t n) {
#if defined(__SSE2__)
  auto* d = static_cast<uint8_t*>(dst);
  auto* s = static_cast<const uint8_t*>(src);
  const size_t head = std::min(n, (size_t)((16 - ((uintptr_t)d & 15)) & 15));
  std::memcpy(d, s, head);
  size_t i = head;
  for (; i + 16 <= n; i += 16)
    _mm_stream_si128(reinterpret_cast<__m128i*>(d + i),
                     _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i)));
  std::memcpy(d + i, s + i, n - i);
#else
  std::memcpy(dst, src, n);
#endif
}

inline void stage_u64(uint64_t* dst, uint64_t v) {
#if defined(__SSE2__) && defined(__x86_64__)
  _mm_stream_si64(reinterpret_cast<long long*>(dst), (long long)v);
#else
  *dst = v;
#endif
}

inline void stage_fence() {
#if defined(__SSE2__)
  _mm_sfence();
#endif
}

}  // namespace

namespace {

using Clock = std::chrono::steady_clock;

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now().time_since_epoch())
      .count();
}

enum Kind { KIND_VERIFY = 0, KIND_BSW = 1 };

struct Request {
  uint64_t ticket = 0;
  int kind = KIND_VERIFY;
  kira_pairs pairs{};
  kira_verify_params vp{};
  kira_sw_cfg cfg{};
  kira_sw_result* out = nullptr;
  uint32_t* cigar_ops = nullptr;
  uint64_t cigar_cap = 0;
  uint32_t max_q = 0, max_w = 0;
  uint64_t cost = 0;  // pair-equivalents for the batch cap (see submit)
  int status = KIRA_PENDING;
  uint64_t cigar_used = 0;
  int64_t t_submit = 0, t_start = 0, t_done = 0;
  uint64_t batch = 0;
  uint32_t batch_requests = 0;
};

// Pinned host staging, grown on demand.
struct Pinned {
  void* p = nullptr;
  size_t bytes = 0;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
  template <class T>
  T* get(size_t count) {
    const size_t need = std::max<size_t>(count, 1) * sizeof(T);
    if (need > bytes) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      bytes = 0;
      const size_t cap = std::max(need, 2 * bytes);  // doubling: regrowth is rare
      if (cudaHostAlloc(&p, cap, cudaHostAllocDefault) != cudaSuccess) return nullptr;
      bytes = cap;
    }
    return static_cast<T*>(p);
  }
};

struct Slot {
  kira_ctx* ctx = nullptr;
  std::thread th;
  Pinned reads, roff, rlen, wins, woff, wlen, boff, abrt, band, out, cig;
  uint64_t held = 0;  // device bytes this slot's last batch was estimated at
};

}  // namespace

struct kira_server {
  int device = 0;
  uint32_t max_batch_pairs = 1u << 20;
  double mem_fraction = 0.5;
  uint64_t trace_budget = 0;
  kira_ctx* owner = nullptr;  // holds the resident reference
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_ticket = 1, next_batch = 1;
  uint32_t busy = 0;
  bool stop = false;
  uint64_t batches = 0, pairs_done = 0;
  double ms_stage = 0, ms_run = 0, ms_scatter = 0, ms_admit = 0;  // host time per phase
  int64_t free_at = 0;      // when free_bytes was last read
  uint64_t free_bytes = 0;  // cached cudaMemGetInfo
  std::string last_error;
};

namespace {

bool same_params(const Request& a, const Request& b) {
  if (a.kind != b.kind) return false;
  if ((a.pairs.win_seq == nullptr) != (b.pairs.win_seq == nullptr)) return false;
  if ((a.pairs.band_offset == nullptr) != (b.pairs.band_offset == nullptr)) return false;
  if ((a.pairs.abort_score == nullptr) != (b.pairs.abort_score == nullptr)) return false;
  if ((a.pairs.bandwidth == nullptr) != (b.pairs.bandwidth == nullptr)) return false;
  return a.kind == KIND_VERIFY ? std::memcmp(&a.vp, &b.vp, sizeof(a.vp)) == 0
                               : std::memcmp(&a.cfg, &b.cfg, sizeof(a.cfg)) == 0;
}

// Device bytes a batch needs outside the (capped) trace arena.
uint64_t estimate(const std::vector<Request*>& b, uint64_t trace_budget) {
  uint64_t e = trace_budget;
  for (const Request* r : b) {
    const uint64_t n = r->pairs.n;
    e += r->pairs.read_seq_bytes + (r->pairs.win_seq ? r->pairs.win_seq_bytes : 0);
    e += n * (96ull + 4ull * (r->max_q + r->max_w + 2));
  }
  return e;
}

// Runs one batch on a slot; fills every request's outputs and status.
void run_batch(kira_server* S, Slot& sl, std::vector<Request*>& b) {
  const int64_t t_in = now_ns();
  uint64_t n = 0, rbytes = 0, wbytes = 0;
  for (Request* r : b) {
    n += r->pairs.n;
    rbytes += r->pairs.read_seq_bytes;
    wbytes += r->pairs.win_seq ? r->pairs.win_seq_bytes : 0;
  }
  const Request& r0 = *b.front();
  const bool host_w = r0.pairs.win_seq != nullptr;
  uint8_t* reads = sl.reads.get<uint8_t>(rbytes + 16);
  uint64_t* roff = sl.roff.get<uint64_t>(n);
  uint32_t* rlen = sl.rlen.get<uint32_t>(n);
  uint8_t* wins = host_w ? sl.wins.get<uint8_t>(wbytes + 16) : nullptr;
  uint64_t* woff = sl.woff.get<uint64_t>(n);
  uint32_t* wlen = sl.wlen.get<uint32_t>(n);
  int32_t* boff = r0.pairs.band_offset ? sl.boff.get<int32_t>(n) : nullptr;
  int32_t* abrt = r0.pairs.abort_score ? sl.abrt.get<int32_t>(n) : nullptr;
  int32_t* band = r0.pairs.bandwidth ? sl.band.get<int32_t>(n) : nullptr;
  kira_sw_result* out = sl.out.get<kira_sw_result>(n);
  int rc = KIRA_OK;
  if (!reads || !roff || !rlen || !woff || !wlen || !out || (host_w && !wins) ||
      (r0.pairs.band_offset && !boff) || (r0.pairs.abort_score && !abrt) ||
      (r0.pairs.bandwidth && !band))
    rc = KIRA_ERR_OOM;
  kira_pairs P{};
  uint64_t at = 0, rb = 0, wb = 0;
  if (rc == KIRA_OK) {
    for (Request* r : b) {
      const kira_pairs& q = r->pairs;
      stage_copy(reads + rb, q.read_seq, q.read_seq_bytes);
      if (host_w) stage_copy(wins + wb, q.win_seq, q.win_seq_bytes);
      for (uint32_t i = 0; i < q.n; ++i) {
        stage_u64(roff + at + i, q.read_off[i] + rb);
        stage_u64(woff + at + i, q.win_off[i] + (host_w ? wb : 0));
      }
      stage_copy(rlen + at, q.read_len, 4ull * q.n);
      stage_copy(wlen + at, q.win_len, 4ull * q.n);
      if (boff) stage_copy(boff + at, q.band_offset, 4ull * q.n);
      if (abrt) stage_copy(abrt + at, q.abort_score, 4ull * q.n);
      if (band) stage_copy(band + at, q.bandwidth, 4ull * q.n);
      P.max_read_len = std::max(P.max_read_len, q.max_read_len);
      P.max_win_len = std::max(P.max_win_len, q.max_win_len);
      P.max_bandwidth = std::max(P.max_bandwidth, q.max_bandwidth);
      at += q.n;
      rb += q.read_seq_bytes;
      wb += host_w ? q.win_seq_bytes : 0;
    }
    std::memset(reads + rb, 0, 16);
    if (host_w) std::memset(wins + wb, 0, 16);
    stage_fence();
    P.n = (uint32_t)n;
    P.read_seq = reads;
    P.read_seq_bytes = rb;
    P.read_off = roff;
    P.read_len = rlen;
    P.win_seq = wins;
    P.win_seq_bytes = wb;
    P.win_off = woff;
    P.win_len = wlen;
    P.band_offset = boff;
    P.abort_score = abrt;
    P.bandwidth = band;
  }
  const int64_t t_staged = now_ns();
  uint64_t cap = 0;
  for (Request* r : b) cap += std::max<uint64_t>(r->cigar_cap, 4ull * r->pairs.n);
  uint32_t* ops = rc == KIRA_OK ? sl.cig.get<uint32_t>(cap) : nullptr;
  if (rc == KIRA_OK && !ops) rc = KIRA_ERR_OOM;
  for (int attempt = 0; rc == KIRA_OK && attempt < 2; ++attempt) {
    kira_cigar_buf cb{ops, cap, 0};
    rc = r0.kind == KIND_VERIFY
             ? kira_gpu_verify_batch(sl.ctx, &P, &r0.vp, out, &cb, nullptr, nullptr)
             : kira_gpu_bsw_batch(sl.ctx, &P, &r0.cfg, out, &cb, nullptr);
    if (rc == KIRA_ERR_CAPACITY && attempt == 0) {  // grow to the reported need, once
      cap = cb.used;
      ops = sl.cig.get<uint32_t>(cap);
      rc = ops ? KIRA_OK : KIRA_ERR_OOM;
      continue;
    }
    break;
  }
  const int64_t t_ran = now_ns();
  std::string err;
  if (rc != KIRA_OK) {
    char buf[512];
    kira_gpu_last_error(sl.ctx, buf, sizeof(buf));
    err = buf;
  }
  // Scatter: a request's pairs and CIGAR ops are contiguous in the batch. The
  // result rows and ops are written without the lock; each request's status and
  // op count are published under it (with t_done), so a waiter that sees a final
  // status also sees its outputs.
  std::vector<int> fin(b.size());
  std::vector<uint64_t> fin_used(b.size());
  at = 0;
  for (size_t ri = 0; ri < b.size(); ++ri) {
    Request* r = b[ri];
    const uint32_t k = r->pairs.n;
    int st = rc;
    uint64_t used = 0;
    if (rc == KIRA_OK && k) {
      const uint64_t base = out[at].cigar_off;
      const uint64_t end = (uint64_t)out[at + k - 1].cigar_off + out[at + k - 1].n_cigar;
      used = end - base;
      for (uint32_t i = 0; i < k; ++i) {
        kira_sw_result x = out[at + i];
        x.cigar_off = (uint32_t)(x.cigar_off - base);
        r->out[i] = x;
      }
      if (used <= r->cigar_cap) {
        if (used) std::memcpy(r->cigar_ops, ops + base, 4ull * used);
      } else {
        st = KIRA_ERR_CAPACITY;
      }
    }
    fin[ri] = st;
    fin_used[ri] = used;
    at += k;
  }
  std::lock_guard<std::mutex> lk(S->mu);
  const int64_t t = now_ns();
  for (size_t ri = 0; ri < b.size(); ++ri) {
    b[ri]->cigar_used = fin_used[ri];
    b[ri]->t_done = t;
    b[ri]->status = fin[ri];
  }
  S->ms_stage += (t_staged - t_in) / 1e6;
  S->ms_run += (t_ran - t_staged) / 1e6;
  S->ms_scatter += (t - t_ran) / 1e6;
  S->batches += 1;
  S->pairs_done += n;
  if (!err.empty()) S->last_error = err;
  S->cv_done.notify_all();
}

void slot_loop(kira_server* S, Slot* sl) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
    if (S->stop) return;
    // Form a batch: the oldest request plus later compatible ones.
    std::vector<Request*> b;
    uint64_t pairs = 0;
    for (auto it = S->queue.begin(); it != S->queue.end();) {
      Request* r = *it;
      if (b.empty() || (same_params(*b.front(), *r) && pairs + r->cost <= S->max_batch_pairs)) {
        b.push_back(r);
        pairs += r->cost;
        it = S->queue.erase(it);
      } else {
        ++it;
      }
    }
    // Admission by free device memory (read outside the lock, at most every 50 ms).
    const int64_t t_adm = now_ns();
    if (t_adm - S->free_at > 50'000'000) {
      lk.unlock();
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
      lk.lock();
      S->free_bytes = fr;
      S->free_at = now_ns();
    }
    S->ms_admit += (now_ns() - t_adm) / 1e6;
    const uint64_t room = (uint64_t)((double)S->free_bytes * S->mem_fraction) + sl->held;
    while (b.size() > 1 && estimate(b, S->trace_budget) > room) {
      S->queue.push_front(b.back());  // back to the queue head, order kept
      b.pop_back();
    }
    if (estimate(b, S->trace_budget) > room && S->busy > 0) {
      for (auto it = b.rbegin(); it != b.rend(); ++it) S->queue.push_front(*it);
      S->cv_done.wait_for(lk, std::chrono::milliseconds(20));
      continue;
    }
    const uint64_t bid = S->next_batch++;
    const int64_t t = now_ns();
    for (Request* r : b) {
      r->t_start = t;
      r->batch = bid;
      r->batch_requests = (uint32_t)b.size();
    }
    sl->held = std::max(sl->held, estimate(b, S->trace_budget));
    S->busy += 1;
    lk.unlock();
    run_batch(S, *sl, b);
    lk.lock();
    S->busy -= 1;
    S->cv_work.notify_all();
  }
}

int submit(kira_server* S, Request* r, uint64_t* ticket) {
  const kira_pairs& P = r->pairs;
  if (P.n && (!P.read_seq || !P.read_off || !P.read_len || !P.win_off || !P.win_len))
    return KIRA_ERR_INVALID;
  if (P.n && !r->out) return KIRA_ERR_INVALID;
  // Batch cost in pair-equivalents: a verification pair counts 1; a banded-SW
  // pair counts its band cells over those of a 150-base read at band 33.
  uint64_t cells = 0;
  for (uint32_t i = 0; i < P.n; ++i) {
    r->max_q = std::max(r->max_q, P.read_len[i]);
    r->max_w = std::max(r->max_w, P.win_len[i]);
    if (r->kind == KIND_BSW) {
      const int32_t band = std::max(P.bandwidth ? P.bandwidth[i] : r->cfg.bandwidth, 1);
      cells += (uint64_t)P.read_len[i] * (2ull * (uint64_t)band + 1);
    }
  }
  r->cost = r->kind == KIND_BSW ? std::max<uint64_t>(P.n, cells / 10050) : P.n;
  r->pairs.max_read_len = r->max_q;
  r->pairs.max_win_len = r->max_w;
  std::unique_ptr<Request> own(r);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return KIRA_ERR_RUNTIME;
  r->ticket = S->next_ticket++;
  r->t_submit = now_ns();
  if (P.n == 0) {  // nothing to run
    r->status = KIRA_OK;
    r->t_start = r->t_done = r->t_submit;
  } else {
    S->queue.push_back(r);
    S->cv_work.notify_one();
  }
  *ticket = r->ticket;
  S->reqs.emplace(r->ticket, std::move(own));
  return KIRA_OK;
}

}  // namespace

extern "C" {

int kira_server_create(const kira_server_cfg* cfg, kira_server** out) {
  if (!cfg || !out || cfg->slots < 1 || cfg->slots > 64) return KIRA_ERR_INVALID;
  *out = nullptr;
  auto S = std::make_unique<kira_server>();
  S->device = cfg->device;
  S->max_batch_pairs = cfg->max_batch_pairs ? cfg->max_batch_pairs : (1u << 20);
  S->mem_fraction = cfg->mem_fraction > 0 && cfg->mem_fraction <= 1 ? cfg->mem_fraction : 0.5;
  int rc = kira_gpu_init(cfg->device, &S->owner);
  if (rc) return rc;
  size_t fr = 0, tot = 0;
  cudaSetDevice(cfg->device);
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 1ull << 30;
  S->trace_budget = std::max<uint64_t>(
      64ull << 20, (uint64_t)((double)fr * S->mem_fraction / (2.0 * cfg->slots)));
  for (int i = 0; i < cfg->slots; ++i) {
    auto sl = std::make_unique<Slot>();
    rc = kira_gpu_init(cfg->device, &sl->ctx);
    if (rc) {
      for (auto& s : S->slots) kira_gpu_destroy(s->ctx);
      kira_gpu_destroy(S->owner);
      return rc;
    }
    kira_gpu_set_trace_budget(sl->ctx, S->trace_budget);
    // Pinned staging for a full batch of 150-250 bp pairs up front: growing pinned
    // memory later (cudaFreeHost / cudaHostAlloc) stalls the device mid-stream.
    const size_t np = std::min<size_t>(S->max_batch_pairs, 1u << 21);
    sl->reads.get<uint8_t>(np * 64 + 16);
    sl->roff.get<uint64_t>(np);
    sl->rlen.get<uint32_t>(np);
    sl->woff.get<uint64_t>(np);
    sl->wlen.get<uint32_t>(np);
    sl->out.get<kira_sw_result>(np);
    sl->cig.get<uint32_t>(4 * np);
    S->slots.push_back(std::move(sl));
  }
  for (auto& sl : S->slots) sl->th = std::thread(slot_loop, S.get(), sl.get());
  *out = S.release();
  return KIRA_OK;
}

void kira_server_destroy(kira_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    for (Request* r : S->queue) {
      r->status = KIRA_ERR_RUNTIME;
      r->t_done = now_ns();
    }
    S->queue.clear();
    S->cv_work.notify_all();
    S->cv_done.notify_all();
  }
  for (auto& sl : S->slots)
    if (sl->th.joinable()) sl->th.join();
  for (auto& sl : S->slots) kira_gpu_destroy(sl->ctx);
  kira_gpu_destroy(S->owner);
  delete S;
}

int kira_server_ref_upload(kira_server* S, const uint8_t* seq, uint64_t len) {
  if (!S) return KIRA_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  // Only between batches: wait (bounded, re-checked) until no slot is running.
  for (int spins = 0; S->busy > 0 || !S->queue.empty(); ++spins) {
    if (spins > 3000) return KIRA_ERR_TIMEOUT;
    S->cv_done.wait_for(lk, std::chrono::milliseconds(10));
  }
  int rc = kira_gpu_ref_upload(S->owner, seq, len);
  if (rc) {
    char buf[512];
    kira_gpu_last_error(S->owner, buf, sizeof(buf));
    S->last_error = buf;
    return rc;
  }
  for (auto& sl : S->slots) kira::ctx_share_reference(sl->ctx, S->owner);
  return KIRA_OK;
}

int kira_server_submit_verify(kira_server* S, const kira_pairs* pairs,
                              const kira_verify_params* params, kira_sw_result* out,
                              uint32_t* cigar_ops, uint64_t cigar_cap, uint64_t* ticket) {
  if (!S || !pairs || !params || !ticket) return KIRA_ERR_INVALID;
  auto* r = new Request();
  r->kind = KIND_VERIFY;
  r->pairs = *pairs;
  r->vp = *params;
  r->out = out;
  r->cigar_ops = cigar_ops;
  r->cigar_cap = cigar_ops ? cigar_cap : 0;
  return submit(S, r, ticket);
}

int kira_server_submit_bsw(kira_server* S, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                           kira_sw_result* out, uint32_t* cigar_ops, uint64_t cigar_cap,
                           uint64_t* ticket) {
  if (!S || !pairs || !cfg || !ticket) return KIRA_ERR_INVALID;
  auto* r = new Request();
  r->kind = KIND_BSW;
  r->pairs = *pairs;
  r->cfg = *cfg;
  r->out = out;
  r->cigar_ops = cigar_ops;
  r->cigar_cap = cigar_ops ? cigar_cap : 0;
  return submit(S, r, ticket);
}

int kira_server_poll(kira_server* S, uint64_t ticket) {
  if (!S) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  return it == S->reqs.end() ? KIRA_ERR_INVALID : it->second->status;
}

int kira_server_wait(kira_server* S, uint64_t ticket, int64_t timeout_ms) {
  if (!S) return KIRA_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return KIRA_ERR_INVALID;
  Request* r = it->second.get();
  const auto deadline = Clock::now() + std::chrono::milliseconds(std::max<int64_t>(timeout_ms, 0));
  while (r->status == KIRA_PENDING) {
    if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        r->status == KIRA_PENDING)
      return KIRA_ERR_TIMEOUT;
  }
  return r->status;
}

int kira_server_info(kira_server* S, uint64_t ticket, kira_request_info* info) {
  if (!S || !info) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return KIRA_ERR_INVALID;
  const Request& r = *it->second;
  info->status = r.status;
  info->n_pairs = r.pairs.n;
  info->cigar_used = r.cigar_used;
  info->t_submit_ns = r.t_submit;
  info->t_start_ns = r.t_start;
  info->t_done_ns = r.t_done;
  info->batch_id = r.batch;
  info->batch_requests = r.batch_requests;
  return KIRA_OK;
}

int kira_server_release(kira_server* S, uint64_t ticket) {
  if (!S) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end() || it->second->status == KIRA_PENDING) return KIRA_ERR_INVALID;
  S->reqs.erase(it);
  return KIRA_OK;
}

int kira_server_stats(kira_server* S, uint64_t* batches, uint64_t* pairs, uint32_t* queued) {
  if (!S) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  if (batches) *batches = S->batches;
  if (pairs) *pairs = S->pairs_done;
  if (queued) *queued = (uint32_t)S->queue.size();
  return KIRA_OK;
}

int kira_server_profile(kira_server* S, double* ms4) {
  if (!S || !ms4) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  ms4[0] = S->ms_stage;
  ms4[1] = S->ms_run;
  ms4[2] = S->ms_scatter;
  ms4[3] = S->ms_admit;
  return KIRA_OK;
}

int kira_server_last_error(kira_server* S, char* buf, size_t len) {
  if (!S) return KIRA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  if (buf && len) {
    const size_t k = std::min(len - 1, S->last_error.size());
    std::memcpy(buf, S->last_error.data(), k);
    buf[k] = 0;
  }
  return KIRA_OK;
}

}  // extern "C"
