// kira_oracle.cpp -- CPU restatement of the kira-ls-aligner verification hot
// path. TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library and the
// timed CPU baseline. The product never links it.
//
// Parity status: pinned by the reference's own known-answer tests (ported in
// tests/test_oracle_*.py) and by naive restatements from those tests; the
// reference crate itself (Rust) cannot be compiled here (no cargo), and its CUDA
// sieve kernel is compiled from source into oracle/_ref/ for a second pin.
//
// Citations are file:line in kira-ls-aligner v0.8.3.

#include "kira_oracle.h"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr int32_t kI32Min = INT32_MIN;

inline int32_t sat_add_i32(int32_t a, int32_t b) {
  int64_t s = (int64_t)a + (int64_t)b;
  if (s > INT32_MAX) return INT32_MAX;
  if (s < INT32_MIN) return INT32_MIN;
  return (int32_t)s;
}

inline uint32_t cig(uint32_t len, uint32_t op) { return (len << 4) | op; }

// push_cigar (src/alignment/mod.rs:1756-1764): merge with the previous op when equal.
struct Cigar {
  std::vector<uint32_t> ops;
  void push(uint32_t op, uint32_t len) {
    if (!ops.empty() && (ops.back() & 0xF) == op) {
      ops.back() += len << 4;
      return;
    }
    ops.push_back(cig(len, op));
  }
};

// ---------------------------------------------------------------------------
// bitpacked.rs
// ---------------------------------------------------------------------------

// encode_base (bitpacked.rs:12-20): A/a=0, C/c=1, G/g=2, T/t=3, else 0.
inline uint8_t encode_base(uint8_t b) {
  switch (b) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 0;
  }
}

// is_acgt (bitpacked.rs:89-91).
inline bool is_acgt(uint8_t b) {
  switch (b) {
    case 'A': case 'a': case 'C': case 'c': case 'G': case 'g': case 'T': case 't': return true;
    default: return false;
  }
}

// pack_into (bitpacked.rs:57-86): four bases per byte, low bits first, tail zero.
bool pack_into(const uint8_t* seq, size_t n, std::vector<uint8_t>& bits) {
  const size_t bytes = (n + 3) / 4;
  bits.assign(bytes, 0);
  bool valid = true;
  const size_t chunks = n / 4;
  for (size_t c = 0; c < chunks; ++c) {
    const uint8_t* q = seq + 4 * c;
    valid = valid && is_acgt(q[0]) && is_acgt(q[1]) && is_acgt(q[2]) && is_acgt(q[3]);
    bits[c] = (uint8_t)(encode_base(q[0]) | (encode_base(q[1]) << 2) | (encode_base(q[2]) << 4) |
                        (encode_base(q[3]) << 6));
  }
  const size_t rest = chunks * 4;
  if (rest < n) {
    uint8_t byte = 0;
    for (size_t j = 0; rest + j < n; ++j) {
      valid = valid && is_acgt(seq[rest + j]);
      byte |= (uint8_t)(encode_base(seq[rest + j]) << (2 * j));
    }
    bits[chunks] = byte;
  }
  return valid;
}

// shift_bits_right_into (bitpacked.rs:102-119).
void shift_bits_right(const uint8_t* bits, size_t n, int off, uint8_t* out) {
  if (off == 0) {
    if (n) std::memcpy(out, bits, n);
    return;
  }
  for (size_t i = 0; i < n; ++i) {
    uint8_t lo = (uint8_t)(bits[i] >> off);
    uint8_t hi = (i + 1 < n) ? (uint8_t)(bits[i + 1] << (8 - off)) : 0;
    out[i] = (uint8_t)(lo | hi);
  }
}

// mismatch_count_u64 (bitpacked.rs:238-270): pair-OR popcount, tail pairs masked.
size_t mismatch_count_u64(const uint8_t* read, const uint8_t* ref, size_t n_bytes, size_t n_nucs) {
  const uint64_t kPairLow = 0x5555555555555555ull;
  const size_t full_bytes = n_nucs / 4;
  const size_t tail_pairs = n_nucs % 4;
  uint32_t total = 0;
  size_t i = 0;
  while (i + 8 <= full_bytes) {
    uint64_t a, b;
    std::memcpy(&a, read + i, 8);
    std::memcpy(&b, ref + i, 8);
    uint64_t x = a ^ b;
    total += (uint32_t)__builtin_popcountll((x | (x >> 1)) & kPairLow);
    i += 8;
  }
  while (i < full_bytes) {
    uint8_t x = read[i] ^ ref[i];
    total += (uint32_t)__builtin_popcount((uint8_t)((x | (x >> 1)) & 0x55));
    ++i;
  }
  if (tail_pairs != 0 && full_bytes < n_bytes) {
    uint8_t x = read[full_bytes] ^ ref[full_bytes];
    uint8_t pm = (uint8_t)((x | (x >> 1)) & 0x55);
    uint8_t keep = (uint8_t)(((1u << (tail_pairs * 2)) - 1) & 0x55);
    total += (uint32_t)__builtin_popcount((uint8_t)(pm & keep));
  }
  return total;
}

// mismatch_count_scalar (bitpacked.rs:272-296); the AVX2 variant
// (bitpacked.rs:300-354) counts the same pairs, so the byte loop stands for both.
size_t mismatch_count_scalar(const uint8_t* read, const uint8_t* ref, size_t n_bytes,
                             size_t n_nucs) {
  uint32_t total = 0;
  const size_t full_bytes = n_nucs / 4;
  const size_t tail_pairs = n_nucs % 4;
  for (size_t i = 0; i < full_bytes; ++i) {
    uint8_t x = read[i] ^ ref[i];
    total += (uint32_t)__builtin_popcount((uint8_t)((x | (x >> 1)) & 0x55));
  }
  if (tail_pairs != 0 && full_bytes < n_bytes) {
    uint8_t x = read[full_bytes] ^ ref[full_bytes];
    uint8_t pm = (uint8_t)((x | (x >> 1)) & 0x55);
    uint8_t keep = (uint8_t)(((1u << (tail_pairs * 2)) - 1) & 0x55);
    total += (uint32_t)__builtin_popcount((uint8_t)(pm & keep));
  }
  return total;
}

// mismatch_count dispatch (bitpacked.rs:215-233).
size_t mismatch_count(const uint8_t* read, const uint8_t* ref, size_t n_bytes, size_t n_nucs) {
  if (n_bytes <= 64) return mismatch_count_u64(read, ref, n_bytes, n_nucs);
  return mismatch_count_scalar(read, ref, n_bytes, n_nucs);
}

// scan_best_with_second_raw (bitpacked.rs:154-199). Returns false for None.
// Ties on the best count keep the lowest shift (strict <); ties with the best
// count at another shift become the second value.
bool scan_best_with_second_raw(const uint8_t* read_bits, size_t read_bytes, size_t read_len,
                               bool read_valid, const uint8_t* const phases[4],
                               size_t ref_bytes, size_t ref_len, size_t* best_shift_out,
                               size_t* best_mism_out, bool* has_second, size_t* second_out) {
  const size_t r = read_len;
  if (r == 0 || ref_len < r || !read_valid) return false;
  const size_t n_shifts = ref_len - r + 1;
  size_t best_shift = 0;
  size_t best = SIZE_MAX, second = SIZE_MAX;
  for (size_t t = 0; t < n_shifts; ++t) {
    const size_t phase = t % 4, byte_off = t / 4;
    if (byte_off + read_bytes > ref_bytes) continue;
    size_t m = mismatch_count(read_bits, phases[phase] + byte_off, read_bytes, r);
    if (m < best) {
      second = best;
      best = m;
      best_shift = t;
    } else if (m < second) {
      second = m;
    }
  }
  if (best == SIZE_MAX) return false;
  *best_shift_out = best_shift;
  *best_mism_out = best;
  *has_second = second != SIZE_MAX;
  *second_out = second;
  return true;
}

// packed_scan_scratch (mod.rs:594-621): pack both, reject either invalid, scan.
bool packed_scan(const uint8_t* read, size_t q, const uint8_t* text, size_t w, size_t* shift,
                 size_t* mism, bool* has_second, size_t* second) {
  std::vector<uint8_t> rb, tb;
  if (!pack_into(read, q, rb)) return false;
  if (!pack_into(text, w, tb)) return false;
  const size_t nb = tb.size();
  std::vector<uint8_t> ph(4 * nb);
  for (int p = 0; p < 4; ++p) shift_bits_right(tb.data(), nb, 2 * p, ph.data() + p * nb);
  const uint8_t* phases[4] = {ph.data(), ph.data() + nb, ph.data() + 2 * nb, ph.data() + 3 * nb};
  return scan_best_with_second_raw(rb.data(), rb.size(), q, true, phases, nb, w, shift, mism,
                                   has_second, second);
}

// ---------------------------------------------------------------------------
// myers.rs
// ---------------------------------------------------------------------------

// base_to_idx (myers.rs:8-16): -1 stands for None.
inline int base_to_idx(uint8_t b) {
  switch (b) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

constexpr size_t kBlockBits = 64;
constexpr size_t kFixedBlocks = 4;

// bounded_edit_distance_fixed (myers.rs:101-204).
bool myers_fixed(const uint8_t* pattern, size_t m, const uint8_t* text, size_t n, size_t max_k,
                 size_t* dist, size_t* pos) {
  const size_t blocks = (m + kBlockBits - 1) / kBlockBits;
  uint64_t peq[4][kFixedBlocks] = {};
  for (size_t i = 0; i < m; ++i) {
    int c = base_to_idx(pattern[i]);
    if (c >= 0) peq[c][i / kBlockBits] |= 1ull << (i % kBlockBits);
  }
  const size_t top_used = m - (blocks - 1) * kBlockBits;
  const uint64_t top_mask = top_used == kBlockBits ? ~0ull : ((1ull << top_used) - 1);
  const uint64_t high_bit = 1ull << (top_used - 1);
  uint64_t vp[kFixedBlocks] = {}, vn[kFixedBlocks] = {};
  for (size_t b = 0; b < blocks; ++b) vp[b] = ~0ull;
  vp[blocks - 1] &= top_mask;
  size_t err = m, best_score = m, best_pos = 0;
  const uint64_t zero_lane[kFixedBlocks] = {};
  for (size_t j = 0; j < n; ++j) {
    int ci = base_to_idx(text[j]);
    const uint64_t* peq_c = ci >= 0 ? peq[ci] : zero_lane;
    uint64_t hin_p = 0, hin_n = 0;
    bool add_carry = false;
    for (size_t b = 0; b < blocks; ++b) {
      const uint64_t eq = peq_c[b], vpb = vp[b], vnb = vn[b];
      const uint64_t x = eq | vnb;
      const uint64_t av = eq & vpb;
      uint64_t s1 = av + vpb;
      bool c1 = s1 < av;
      uint64_t sum_lo = s1 + (add_carry ? 1 : 0);
      bool c2 = sum_lo < s1;
      add_carry = c1 || c2;
      const uint64_t d0 = (sum_lo ^ vpb) | x;
      const uint64_t hp = vnb | ~(d0 | vpb);
      const uint64_t hn = d0 & vpb;
      const uint64_t hp_s = (hp << 1) | hin_p;
      const uint64_t hn_s = (hn << 1) | hin_n;
      hin_p = hp >> 63;
      hin_n = hn >> 63;
      const uint64_t nvp = hn_s | ~(d0 | hp_s);
      const uint64_t nvn = d0 & hp_s;
      const uint64_t mask = b == blocks - 1 ? top_mask : ~0ull;
      vp[b] = nvp & mask;
      vn[b] = nvn & mask;
      if (b == blocks - 1) {
        if (hp & high_bit) err += 1;
        if (hn & high_bit) err -= 1;
      }
    }
    if (err <= best_score) {
      best_score = err;
      best_pos = j + 1;
    }
    const size_t rem = n - 1 - j;
    const size_t sat = err > rem ? err - rem : 0;
    if (best_score > max_k && sat > max_k) return false;
  }
  if (best_score <= max_k) {
    *dist = best_score;
    *pos = best_pos;
    return true;
  }
  return false;
}

// bounded_edit_distance_inner (myers.rs:206-324): heap blocks, u128 carry.
bool myers_heap(const uint8_t* pattern, size_t m, const uint8_t* text, size_t n, size_t max_k,
                size_t* dist, size_t* pos) {
  const size_t blocks = (m + kBlockBits - 1) / kBlockBits;
  std::vector<uint64_t> peq[4];
  for (auto& l : peq) l.assign(blocks, 0);
  for (size_t i = 0; i < m; ++i) {
    int c = base_to_idx(pattern[i]);
    if (c >= 0) peq[c][i / kBlockBits] |= 1ull << (i % kBlockBits);
  }
  const size_t top_used = m - (blocks - 1) * kBlockBits;
  const uint64_t top_mask = top_used == kBlockBits ? ~0ull : ((1ull << top_used) - 1);
  const uint64_t high_bit = 1ull << (top_used - 1);
  std::vector<uint64_t> vp(blocks, ~0ull), vn(blocks, 0);
  vp[blocks - 1] &= top_mask;
  size_t err = m, best_score = m, best_pos = 0;
  for (size_t j = 0; j < n; ++j) {
    const int ci = base_to_idx(text[j]);
    const bool n_in_text = ci < 0;
    const std::vector<uint64_t>& peq_c = ci >= 0 ? peq[ci] : peq[0];
    uint64_t hin_p = 0, hin_n = 0;
    unsigned __int128 carry = 0;
    for (size_t b = 0; b < blocks; ++b) {
      const uint64_t eq = n_in_text ? 0 : peq_c[b];
      const uint64_t vpb = vp[b], vnb = vn[b];
      const uint64_t x = eq | vnb;
      const uint64_t av = eq & vpb;
      unsigned __int128 s = (unsigned __int128)av + vpb + carry;
      const uint64_t sum_lo = (uint64_t)s;
      carry = s >> 64;
      const uint64_t d0 = (sum_lo ^ vpb) | x;
      const uint64_t hp = vnb | ~(d0 | vpb);
      const uint64_t hn = d0 & vpb;
      const uint64_t hp_s = (hp << 1) | hin_p;
      const uint64_t hn_s = (hn << 1) | hin_n;
      const uint64_t nhp = hp >> 63, nhn = hn >> 63;
      const uint64_t nvp = hn_s | ~(d0 | hp_s);
      const uint64_t nvn = d0 & hp_s;
      const uint64_t mask = b == blocks - 1 ? top_mask : ~0ull;
      vp[b] = nvp & mask;
      vn[b] = nvn & mask;
      if (b == blocks - 1) {
        if (hp & high_bit) err += 1;
        if (hn & high_bit) err -= 1;
      }
      hin_p = nhp;
      hin_n = nhn;
    }
    if (err <= best_score) {
      best_score = err;
      best_pos = j + 1;
    }
    const size_t rem = n - 1 - j;
    const size_t sat = err > rem ? err - rem : 0;
    if (best_score > max_k && sat > max_k) return false;
  }
  if (best_score <= max_k) {
    *dist = best_score;
    *pos = best_pos;
    return true;
  }
  return false;
}

// bounded_edit_distance (myers.rs:47-70) with an optional forced storage path.
bool myers(const uint8_t* pat, size_t m, const uint8_t* text, size_t n, size_t max_k, int path,
           size_t* dist, size_t* pos) {
  if (m == 0) {
    *dist = 0;
    *pos = 0;
    return true;
  }
  if (n == 0) {
    if (m <= max_k) {
      *dist = m;
      *pos = 0;
      return true;
    }
    return false;
  }
  if (path == 2 || (path == 0 && m > kFixedBlocks * kBlockBits))
    return myers_heap(pat, m, text, n, max_k, dist, pos);
  if (path == 1 && m > kFixedBlocks * kBlockBits) return false;
  return myers_fixed(pat, m, text, n, max_k, dist, pos);
}

// ---------------------------------------------------------------------------
// Banded affine SW (mod.rs:1370-1650)
// ---------------------------------------------------------------------------

constexpr uint8_t TRACE_STOP = 0, TRACE_DIAG = 1, TRACE_E = 2, TRACE_F = 3;  // mod.rs:1652-1658
constexpr uint8_t TRACE_DIR_MASK = 0x03, TRACE_E_EXTEND = 0x04, TRACE_F_EXTEND = 0x08;
constexpr int32_t kNeg4 = kI32Min / 4;  // i32::MIN / 4 sentinel of the scalar kernel

struct SwOut {
  uint32_t ref_start = 0, ref_end = 0;
  int32_t read_start = 0, read_end = 0, score = 0;
  bool early_abort = false;
  uint64_t cells = 0;
  Cigar cigar;
  // Filled only on request (test of traceback forms): per row its band start and
  // every cell's H and trace byte (test infrastructure, not the reference's output).
  std::vector<int32_t> row_starts;
  std::vector<std::vector<int32_t>> h_rows;
  std::vector<std::vector<uint8_t>> trace_rows;
};

enum class TS { H, E, F };

SwOut banded_sw_with(const uint8_t* read, size_t q_len, const uint8_t* reference, size_t r_len,
                     int32_t offset, const orc_cfg& cfg, int32_t abort_score, bool adaptive,
                     int32_t drift_knob, int32_t dp_xdrop, bool keep_matrix = false) {
  SwOut res;
  if (keep_matrix) res.h_rows.resize(q_len + 1);
  const int32_t band = std::max(cfg.bandwidth, 1);
  std::vector<int32_t> prev_h, prev_e, cur_h, cur_e, cur_f;
  int32_t prev_start = 1;
  std::vector<std::vector<uint8_t>> trace_rows(q_len + 1);
  std::vector<int32_t> row_starts(q_len + 1, 1);
  int32_t best_score = 0;
  size_t best_i = 0, best_j = 0;
  int32_t best_qlen_score = 0;
  size_t best_qlen_j = 0;
  bool early_abort = false;
  const int32_t max_drift = adaptive ? drift_knob : 0;  // mod.rs:1425
  int32_t adaptive_center = 1 + offset;                  // mod.rs:1426
  const int32_t r_len_i = (int32_t)r_len;
  const int32_t gof = sat_add_i32(cfg.gap_open, cfg.gap_extend);  // mod.rs:1483

  for (size_t i = 1; i <= q_len; ++i) {
    const int32_t static_center = (int32_t)i + offset;
    const int32_t center =
        adaptive ? std::clamp(adaptive_center, static_center - max_drift, static_center + max_drift)
                 : static_center;
    const int32_t j_start = std::max(center - band, 1);
    const int32_t j_end = std::min(center + band, r_len_i);
    if (j_start > j_end) {  // mod.rs:1437-1444: band left the window; row skipped
      row_starts[i] = 1;
      trace_rows[i].clear();
      prev_h.clear();
      prev_e.clear();
      prev_start = 1;
      continue;
    }
    const size_t row_len = (size_t)(j_end - j_start + 1);
    row_starts[i] = j_start;
    res.cells += row_len;
    cur_h.assign(row_len, 0);
    cur_e.assign(row_len, kNeg4);
    cur_f.assign(row_len, kNeg4);
    std::vector<uint8_t>& trace = trace_rows[i];
    trace.assign(row_len, 0);
    int32_t row_best = 0;
    int32_t row_best_j = -1;
    const uint8_t qb = read[i - 1];
    for (int32_t j = j_start; j <= j_end; ++j) {
      const size_t idx = (size_t)(j - j_start);
      const uint8_t rb = reference[j - 1];
      const int32_t s = qb == rb ? cfg.match_score : -cfg.mismatch;
      // prev_diag (mod.rs:1732-1754): outside the previous band, H=0 but the pair scores.
      int32_t h_diag = 0;
      {
        const int32_t pidx = j - 1 - prev_start;
        if (pidx >= 0 && (size_t)pidx < prev_h.size()) h_diag = prev_h[(size_t)pidx];
      }
      const int32_t h_match = h_diag + s;
      // prev_cell (mod.rs:1723-1730).
      int32_t e_from_h = kNeg4, e_from_e = kNeg4;
      {
        const int32_t pidx = j - prev_start;
        if (pidx >= 0 && (size_t)pidx < prev_h.size()) {
          e_from_h = prev_h[(size_t)pidx] - gof;
          e_from_e = prev_e[(size_t)pidx] - cfg.gap_extend;
        }
      }
      const int32_t e = std::max(e_from_h, e_from_e);
      int32_t f_from_h = kNeg4, f_from_f = kNeg4;
      if (idx > 0) {
        f_from_h = cur_h[idx - 1] - gof;
        f_from_f = cur_f[idx - 1] - cfg.gap_extend;
      }
      const int32_t f = std::max(f_from_h, f_from_f);
      cur_e[idx] = e;
      cur_f[idx] = f;
      // Direction priority diag >= E >= F (mod.rs:1504-1516).
      int32_t h = 0;
      uint8_t tr = TRACE_STOP;
      if (h_match >= e && h_match >= f && h_match > 0) {
        h = h_match;
        tr = TRACE_DIAG;
      } else if (e >= f && e > 0) {
        h = e;
        tr = TRACE_E;
      } else if (f > 0) {
        h = f;
        tr = TRACE_F;
      }
      cur_h[idx] = h;
      if (e_from_e > e_from_h) tr |= TRACE_E_EXTEND;
      if (f_from_f > f_from_h) tr |= TRACE_F_EXTEND;
      trace[idx] = tr;
      if (h > row_best) {
        row_best = h;
        row_best_j = j;
      }
      if (h > best_score) {
        best_score = h;
        best_i = i;
        best_j = (size_t)j;
      }
      if (i == q_len && h > best_qlen_score) {
        best_qlen_score = h;
        best_qlen_j = (size_t)j;
      }
    }
    if (keep_matrix) res.h_rows[i] = cur_h;
    std::swap(prev_h, cur_h);
    std::swap(prev_e, cur_e);
    prev_start = j_start;
    if (adaptive) {  // mod.rs:1546-1559
      const int32_t raw = row_best_j >= 0 ? row_best_j + 1 : adaptive_center + 1;
      const int32_t static_next = (int32_t)i + 1 + offset;
      adaptive_center = std::clamp(raw, static_next - max_drift, static_next + max_drift);
    }
    if (dp_xdrop > 0 && best_score - row_best > dp_xdrop) {  // mod.rs:1561-1564
      early_abort = true;
      break;
    }
    if (abort_score > kI32Min / 8) {  // mod.rs:1565-1572
      const int32_t remaining = (int32_t)(q_len - i);
      const int32_t max_possible = best_score + remaining * cfg.match_score;
      if (max_possible < abort_score) {
        early_abort = true;
        break;
      }
    }
  }
  // Clip-penalty end preference (mod.rs:1575-1579).
  if (best_qlen_score > 0 && sat_add_i32(best_qlen_score, cfg.clip_penalty) > best_score) {
    best_score = best_qlen_score;
    best_i = q_len;
    best_j = best_qlen_j;
  }
  // Traceback state machine (mod.rs:1581-1627).
  int32_t i = (int32_t)best_i, j = (int32_t)best_j;
  const int32_t read_end = i;
  const uint32_t ref_end = (uint32_t)j;
  TS state = TS::H;
  std::vector<uint32_t> rev;
  Cigar cg;
  while (i > 0 && j > 0) {
    const int32_t row_start = row_starts[(size_t)i];
    const int64_t idx = (int64_t)j - row_start;
    if (idx < 0 || (size_t)idx >= trace_rows[(size_t)i].size()) break;
    const uint8_t tr = trace_rows[(size_t)i][(size_t)idx];
    if (state == TS::H) {
      const uint8_t d = tr & TRACE_DIR_MASK;
      if (d == TRACE_STOP) break;
      if (d == TRACE_DIAG) {
        cg.push(0, 1);
        --i;
        --j;
      } else if (d == TRACE_E) {
        state = TS::E;
      } else {
        state = TS::F;
      }
    } else if (state == TS::E) {
      cg.push(1, 1);
      --i;
      state = (tr & TRACE_E_EXTEND) ? TS::E : TS::H;
    } else {
      cg.push(2, 1);
      --j;
      state = (tr & TRACE_F_EXTEND) ? TS::F : TS::H;
    }
  }
  std::reverse(cg.ops.begin(), cg.ops.end());
  if (keep_matrix) {
    res.row_starts = row_starts;
    res.trace_rows = std::move(trace_rows);
  }
  res.ref_start = (uint32_t)j;
  res.ref_end = ref_end;
  res.read_start = i;
  res.read_end = read_end;
  res.score = best_score;
  res.early_abort = early_abort;
  res.cigar = std::move(cg);
  return res;
}

void emit(const SwOut& s, orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  out->ref_start = s.ref_start;
  out->ref_end = s.ref_end;
  out->read_start = s.read_start;
  out->read_end = s.read_end;
  out->score = s.score;
  out->n_cigar = (uint32_t)s.cigar.ops.size();
  out->early_abort = s.early_abort ? 1u : 0u;
  out->pad = 0;
  out->cells = s.cells;
  if (cigar) {
    const uint32_t n = std::min<uint32_t>(cap, (uint32_t)s.cigar.ops.size());
    for (uint32_t k = 0; k < n; ++k) cigar[k] = s.cigar.ops[k];
  }
}

// traceback_interleaved (mod.rs:1667-1716) over a lane-interleaved full matrix.
void traceback_interleaved(const uint8_t* trace, size_t trace_size, size_t trace_w,
                           size_t lane_stride, size_t lane, int32_t i, int32_t j, Cigar& cg,
                           int32_t* oi, int32_t* oj) {
  TS state = TS::H;
  while (i > 0 && j > 0) {
    const size_t idx = ((size_t)i * trace_w + (size_t)j) * lane_stride + lane;
    if (idx >= trace_size) break;
    const uint8_t tr = trace[idx];
    if (state == TS::H) {
      const uint8_t d = tr & TRACE_DIR_MASK;
      if (d == TRACE_STOP) break;
      if (d == TRACE_DIAG) {
        cg.push(0, 1);
        --i;
        --j;
      } else if (d == TRACE_E) {
        state = TS::E;
      } else {
        state = TS::F;
      }
    } else if (state == TS::E) {
      cg.push(1, 1);
      --i;
      state = (tr & TRACE_E_EXTEND) ? TS::E : TS::H;
    } else {
      cg.push(2, 1);
      --j;
      state = (tr & TRACE_F_EXTEND) ? TS::F : TS::H;
    }
  }
  std::reverse(cg.ops.begin(), cg.ops.end());
  *oi = i;
  *oj = j;
}

// ---------------------------------------------------------------------------
// Full-window batch SW: sw_batch_avx2_inner (mod.rs:1914-2135) restated with the
// same AVX2 intrinsics, and sw_batch_int8_inner (sw_int8_vnni.rs:141-370).
// ---------------------------------------------------------------------------

// Unaligned 256-bit row access inside the AVX2 kernels (macros: lambdas would not
// inherit the functions' target attribute).
#define LD(p) _mm256_loadu_si256((const __m256i*)(p))
#define ST(p, v) _mm256_storeu_si256((__m256i*)(p), (v))

// Lane-result assembly shared by both kernels (mod.rs:2104-2132).
void finish_lane(const uint8_t* trace, size_t trace_size, size_t trace_w, size_t lanes_stride,
                 size_t k, size_t q_len, int32_t local_score, int32_t best_i, int32_t best_j,
                 int32_t qlen_score, int32_t qlen_j, int32_t clip, bool done, SwOut& out) {
  int32_t si, sj, bs;
  if (qlen_score > 0 && sat_add_i32(qlen_score, clip) > local_score) {
    si = (int32_t)q_len;
    sj = qlen_j;
    bs = qlen_score;
  } else {
    si = best_i;
    sj = best_j;
    bs = local_score;
  }
  int32_t ei, ej;
  traceback_interleaved(trace, trace_size, trace_w, lanes_stride, k, si, sj, out.cigar, &ei, &ej);
  out.ref_start = (uint32_t)ej;
  out.ref_end = (uint32_t)sj;
  out.read_start = ei;
  out.read_end = si;
  out.score = bs;
  out.early_abort = done;
}

__attribute__((target("avx2"))) void sw_avx2_inner(int lanes, const uint8_t* const* reads,
                                                   const uint8_t* const* wins, size_t q_len,
                                                   size_t r_len, const int32_t* aborts,
                                                   const orc_cfg& cfg, SwOut* outs) {
  constexpr size_t L = 16;
  const __m256i v_zero = _mm256_setzero_si256();
  const __m256i v_go = _mm256_set1_epi16((int16_t)(-sat_add_i32(cfg.gap_open, cfg.gap_extend)));
  const __m256i v_ge = _mm256_set1_epi16((int16_t)(-cfg.gap_extend));
  const __m256i v_match = _mm256_set1_epi16((int16_t)cfg.match_score);
  const __m256i v_mism = _mm256_set1_epi16((int16_t)(-cfg.mismatch));
  const __m256i v_one = _mm256_set1_epi16(1), v_two = _mm256_set1_epi16(2),
                v_three = _mm256_set1_epi16(3);
  const __m256i v_four = _mm256_set1_epi16(TRACE_E_EXTEND), v_eight = _mm256_set1_epi16(TRACE_F_EXTEND);
  const __m256i v_neg = _mm256_set1_epi16(-16384);
  const size_t trace_w = r_len + 1;
  // One 16-lane i16 vector per column, kept as flat lane arrays.
  std::vector<int16_t> ph_buf((r_len + 1) * L, 0), pe_buf((r_len + 1) * L, -16384),
      ch_buf((r_len + 1) * L, 0), ce_buf((r_len + 1) * L, -16384);
  int16_t* prev_hp = ph_buf.data();
  int16_t* prev_ep = pe_buf.data();
  int16_t* cur_hp = ch_buf.data();
  int16_t* cur_ep = ce_buf.data();
  std::vector<uint8_t> trace((q_len + 1) * (r_len + 1) * L, 0);
  std::vector<uint8_t> read_cols((q_len + 1) * L, 0), ref_cols((r_len + 1) * L, 0);
  for (size_t i = 1; i <= q_len; ++i)
    for (int k = 0; k < lanes; ++k) read_cols[i * L + k] = reads[k][i - 1];
  for (size_t j = 1; j <= r_len; ++j)
    for (int k = 0; k < lanes; ++k) ref_cols[j * L + k] = wins[k][j - 1];
  __m256i best_v = v_zero, best_i_v = v_zero, best_j_v = v_zero, best_qlen_v = v_zero,
          best_qlen_j_v = v_zero;
  bool lane_done[L] = {};
  alignas(32) int16_t best_arr[L];
  for (size_t i = 1; i <= q_len; ++i) {
    ST(cur_hp, v_zero);
    ST(cur_ep, v_neg);
    __m256i cur_f = v_neg;
    const __m128i read_v = _mm_loadu_si128((const __m128i*)(read_cols.data() + i * L));
    const __m256i i_vec = _mm256_set1_epi16((int16_t)i);
    for (size_t j = 1; j <= r_len; ++j) {
      const __m128i ref_v = _mm_loadu_si128((const __m128i*)(ref_cols.data() + j * L));
      const __m256i eq16 = _mm256_cvtepi8_epi16(_mm_cmpeq_epi8(read_v, ref_v));
      const __m256i score = _mm256_blendv_epi8(v_mism, v_match, eq16);
      const __m256i h_match = _mm256_adds_epi16(LD(prev_hp + (j - 1) * L), score);
      const __m256i e_from_h = _mm256_adds_epi16(LD(prev_hp + j * L), v_go);
      const __m256i e_from_e = _mm256_adds_epi16(LD(prev_ep + j * L), v_ge);
      const __m256i e = _mm256_max_epi16(e_from_h, e_from_e);
      const __m256i e_ext = _mm256_cmpgt_epi16(e_from_e, e_from_h);
      const __m256i f_from_h = _mm256_adds_epi16(LD(cur_hp + (j - 1) * L), v_go);
      const __m256i f_from_f = _mm256_adds_epi16(cur_f, v_ge);
      const __m256i f = _mm256_max_epi16(f_from_h, f_from_f);
      const __m256i f_ext = _mm256_cmpgt_epi16(f_from_f, f_from_h);
      const __m256i h = _mm256_max_epi16(_mm256_max_epi16(_mm256_max_epi16(h_match, e), f), v_zero);
      ST(cur_hp + j * L, h);
      ST(cur_ep + j * L, e);
      cur_f = f;
      const __m256i is_zero = _mm256_cmpeq_epi16(h, v_zero);
      const __m256i eq_m = _mm256_cmpeq_epi16(h, h_match);
      const __m256i eq_e = _mm256_cmpeq_epi16(h, e);
      const __m256i is_match = _mm256_andnot_si256(is_zero, eq_m);
      const __m256i is_e = _mm256_andnot_si256(is_zero, _mm256_andnot_si256(eq_m, eq_e));
      __m256i tr = _mm256_blendv_epi8(v_three, v_two, is_e);
      tr = _mm256_blendv_epi8(tr, v_one, is_match);
      tr = _mm256_blendv_epi8(tr, v_zero, is_zero);
      tr = _mm256_or_si256(tr, _mm256_and_si256(e_ext, v_four));
      tr = _mm256_or_si256(tr, _mm256_and_si256(f_ext, v_eight));
      __m256i packed = _mm256_permute4x64_epi64(_mm256_packus_epi16(tr, tr), 0xD8);
      _mm_storeu_si128((__m128i*)(trace.data() + (i * trace_w + j) * L),
                       _mm256_castsi256_si128(packed));
      const __m256i nb = _mm256_cmpgt_epi16(h, best_v);
      best_v = _mm256_max_epi16(best_v, h);
      const __m256i j_vec = _mm256_set1_epi16((int16_t)j);
      best_i_v = _mm256_blendv_epi8(best_i_v, i_vec, nb);
      best_j_v = _mm256_blendv_epi8(best_j_v, j_vec, nb);
      if (i == q_len) {
        const __m256i nq = _mm256_cmpgt_epi16(h, best_qlen_v);
        best_qlen_v = _mm256_max_epi16(best_qlen_v, h);
        best_qlen_j_v = _mm256_blendv_epi8(best_qlen_j_v, j_vec, nq);
      }
    }
    // Per-row abort check; the batch stops only when every lane is done (mod.rs:2058-2081).
    const int32_t remaining = (int32_t)(q_len - i);
    _mm256_store_si256((__m256i*)best_arr, best_v);
    bool all_done = true;
    for (int k = 0; k < lanes; ++k) {
      if (lane_done[k]) continue;
      if (aborts[k] > kI32Min / 8) {
        const int32_t mp = (int32_t)best_arr[k] + remaining * cfg.match_score;
        if (mp < aborts[k]) lane_done[k] = true;
      }
      if (!lane_done[k]) all_done = false;
    }
    if (all_done) break;
    std::swap(prev_hp, cur_hp);
    std::swap(prev_ep, cur_ep);
  }
  alignas(32) int16_t bs[L], bi[L], bj[L], bq[L], bqj[L];
  _mm256_store_si256((__m256i*)bs, best_v);
  _mm256_store_si256((__m256i*)bi, best_i_v);
  _mm256_store_si256((__m256i*)bj, best_j_v);
  _mm256_store_si256((__m256i*)bq, best_qlen_v);
  _mm256_store_si256((__m256i*)bqj, best_qlen_j_v);
  for (int k = 0; k < lanes; ++k)
    finish_lane(trace.data(), trace.size(), trace_w, L, (size_t)k, q_len, bs[k], bi[k], bj[k], bq[k],
                bqj[k], cfg.clip_penalty, lane_done[k], outs[k]);
}

// int8_path_viable (sw_int8_vnni.rs:47-55).
bool int8_viable(size_t read_len, const orc_cfg& cfg) {
  const int64_t ms = std::max(cfg.match_score, 1);
  const int64_t upper = (int64_t)read_len * ms;
  auto in = [](int32_t v) { return v >= 0 && v <= 32; };
  return upper < 120 && in(cfg.match_score) && in(cfg.mismatch) && in(cfg.gap_open) &&
         in(cfg.gap_extend);
}

__attribute__((target("avx2"))) void sw_int8_inner(int lanes, const uint8_t* const* reads,
                                                   const uint8_t* const* wins, size_t q_len,
                                                   size_t r_len, const int32_t* aborts,
                                                   const orc_cfg& cfg, SwOut* outs,
                                                   bool* saturated) {
  constexpr size_t L = 32;
  const __m256i v_zero = _mm256_setzero_si256();
  const __m256i v_neg = _mm256_set1_epi8(-100);
  const __m256i v_go = _mm256_set1_epi8((int8_t)(-(int8_t)sat_add_i32(cfg.gap_open, cfg.gap_extend)));
  const __m256i v_ge = _mm256_set1_epi8((int8_t)(-(int8_t)cfg.gap_extend));
  const __m256i v_match = _mm256_set1_epi8((int8_t)cfg.match_score);
  const __m256i v_mism = _mm256_set1_epi8((int8_t)(-(int8_t)cfg.mismatch));
  const __m256i v_one = _mm256_set1_epi8(1), v_two = _mm256_set1_epi8(2), v_three = _mm256_set1_epi8(3);
  const __m256i v_four = _mm256_set1_epi8(TRACE_E_EXTEND), v_eight = _mm256_set1_epi8(TRACE_F_EXTEND);
  const __m256i v_sat = _mm256_set1_epi8(120);
  const size_t trace_w = r_len + 1;
  std::vector<int8_t> ph_buf((r_len + 1) * L, 0), pe_buf((r_len + 1) * L, -100),
      ch_buf((r_len + 1) * L, 0), ce_buf((r_len + 1) * L, -100);
  int8_t* prev_hp = ph_buf.data();
  int8_t* prev_ep = pe_buf.data();
  int8_t* cur_hp = ch_buf.data();
  int8_t* cur_ep = ce_buf.data();
  std::vector<uint8_t> trace((q_len + 1) * (r_len + 1) * L, 0);
  std::vector<uint8_t> read_cols((q_len + 1) * L, 0), ref_cols((r_len + 1) * L, 0);
  for (size_t i = 1; i <= q_len; ++i)
    for (int k = 0; k < lanes; ++k) read_cols[i * L + k] = reads[k][i - 1];
  for (size_t j = 1; j <= r_len; ++j)
    for (int k = 0; k < lanes; ++k) ref_cols[j * L + k] = wins[k][j - 1];
  __m256i best_v = v_zero, best_qlen_v = v_zero, sat_v = v_zero;
  int32_t best_i[L] = {}, best_j[L] = {}, best_qlen_j[L] = {};
  bool lane_done[L] = {};
  alignas(32) int8_t best_arr[L];
  for (size_t i = 1; i <= q_len; ++i) {
    ST(cur_hp, v_zero);
    ST(cur_ep, v_neg);
    __m256i cur_f = v_neg;
    const __m256i read_v = _mm256_loadu_si256((const __m256i*)(read_cols.data() + i * L));
    for (size_t j = 1; j <= r_len; ++j) {
      const __m256i ref_v = _mm256_loadu_si256((const __m256i*)(ref_cols.data() + j * L));
      const __m256i eq = _mm256_cmpeq_epi8(read_v, ref_v);
      const __m256i score = _mm256_blendv_epi8(v_mism, v_match, eq);
      const __m256i h_match = _mm256_adds_epi8(LD(prev_hp + (j - 1) * L), score);
      const __m256i e_from_h = _mm256_adds_epi8(LD(prev_hp + j * L), v_go);
      const __m256i e_from_e = _mm256_adds_epi8(LD(prev_ep + j * L), v_ge);
      const __m256i e = _mm256_max_epi8(e_from_h, e_from_e);
      const __m256i e_ext = _mm256_cmpgt_epi8(e_from_e, e_from_h);
      const __m256i f_from_h = _mm256_adds_epi8(LD(cur_hp + (j - 1) * L), v_go);
      const __m256i f_from_f = _mm256_adds_epi8(cur_f, v_ge);
      const __m256i f = _mm256_max_epi8(f_from_h, f_from_f);
      const __m256i f_ext = _mm256_cmpgt_epi8(f_from_f, f_from_h);
      const __m256i h = _mm256_max_epi8(_mm256_max_epi8(_mm256_max_epi8(h_match, e), f), v_zero);
      ST(cur_hp + j * L, h);
      ST(cur_ep + j * L, e);
      cur_f = f;
      const __m256i is_zero = _mm256_cmpeq_epi8(h, v_zero);
      const __m256i eq_m = _mm256_cmpeq_epi8(h, h_match);
      const __m256i eq_e = _mm256_cmpeq_epi8(h, e);
      const __m256i is_match = _mm256_andnot_si256(is_zero, eq_m);
      const __m256i is_e = _mm256_andnot_si256(is_zero, _mm256_andnot_si256(eq_m, eq_e));
      __m256i tr = _mm256_blendv_epi8(v_three, v_two, is_e);
      tr = _mm256_blendv_epi8(tr, v_one, is_match);
      tr = _mm256_blendv_epi8(tr, v_zero, is_zero);
      tr = _mm256_or_si256(tr, _mm256_and_si256(e_ext, v_four));
      tr = _mm256_or_si256(tr, _mm256_and_si256(f_ext, v_eight));
      _mm256_storeu_si256((__m256i*)(trace.data() + (i * trace_w + j) * L), tr);
      const __m256i nb = _mm256_cmpgt_epi8(h, best_v);
      best_v = _mm256_max_epi8(best_v, h);
      uint32_t mask = (uint32_t)_mm256_movemask_epi8(nb);
      while (mask) {
        const int k = __builtin_ctz(mask);
        mask &= mask - 1;
        if (k < lanes) {
          best_i[k] = (int32_t)i;
          best_j[k] = (int32_t)j;
        }
      }
      if (i == q_len) {
        const __m256i nq = _mm256_cmpgt_epi8(h, best_qlen_v);
        best_qlen_v = _mm256_max_epi8(best_qlen_v, h);
        uint32_t m2 = (uint32_t)_mm256_movemask_epi8(nq);
        while (m2) {
          const int k = __builtin_ctz(m2);
          m2 &= m2 - 1;
          if (k < lanes) best_qlen_j[k] = (int32_t)j;
        }
      }
      sat_v = _mm256_or_si256(sat_v, _mm256_cmpgt_epi8(h, v_sat));
    }
    const int32_t remaining = (int32_t)(q_len - i);
    _mm256_store_si256((__m256i*)best_arr, best_v);
    bool all_done = true;
    for (int k = 0; k < lanes; ++k) {
      if (lane_done[k]) continue;
      if (aborts[k] > kI32Min / 8) {
        const int32_t mp = (int32_t)best_arr[k] + remaining * cfg.match_score;
        if (mp < aborts[k]) lane_done[k] = true;
      }
      if (!lane_done[k]) all_done = false;
    }
    if (all_done) break;
    std::swap(prev_hp, cur_hp);
    std::swap(prev_ep, cur_ep);
  }
  alignas(32) int8_t bs[L], bq[L];
  alignas(32) uint8_t sat[L];
  _mm256_store_si256((__m256i*)bs, best_v);
  _mm256_store_si256((__m256i*)bq, best_qlen_v);
  _mm256_store_si256((__m256i*)sat, sat_v);
  for (int k = 0; k < lanes; ++k) {
    saturated[k] = sat[k] != 0;
    if (saturated[k]) continue;
    finish_lane(trace.data(), trace.size(), trace_w, L, (size_t)k, q_len, bs[k], best_i[k],
                best_j[k], bq[k], best_qlen_j[k], cfg.clip_penalty, lane_done[k], outs[k]);
  }
}

// Portable model of the full-window kernels: identical recurrence with explicit
// saturation to `bits`-wide lanes (16 -> i16 AVX2 kernel, 8 -> i8 kernel) and the
// same all-lanes-done row break. The group is the whole argument list.
void sw_full_window_model(int lanes, const uint8_t* const* reads, const uint8_t* const* wins,
                          size_t q_len, size_t r_len, const int32_t* aborts, const orc_cfg& cfg,
                          int bits, SwOut* outs) {
  const int32_t lo = bits == 8 ? -128 : -32768, hi = bits == 8 ? 127 : 32767;
  auto sat = [&](int32_t v) { return std::min(std::max(v, lo), hi); };
  auto adds = [&](int32_t a, int32_t b) { return sat(a + b); };
  auto cast = [&](int32_t v) {  // value of an integer constant set into a narrow lane
    return bits == 8 ? (int32_t)(int8_t)v : (int32_t)(int16_t)v;
  };
  const int32_t neg = bits == 8 ? -100 : -16384;
  const int32_t go = bits == 8 ? cast(-(int32_t)(int8_t)sat_add_i32(cfg.gap_open, cfg.gap_extend))
                               : cast(-sat_add_i32(cfg.gap_open, cfg.gap_extend));
  const int32_t ge = bits == 8 ? cast(-(int32_t)(int8_t)cfg.gap_extend) : cast(-cfg.gap_extend);
  const int32_t vm = cast(cfg.match_score);
  const int32_t vx = bits == 8 ? cast(-(int32_t)(int8_t)cfg.mismatch) : cast(-cfg.mismatch);
  const size_t W = r_len + 1;
  const size_t L = (size_t)lanes;
  std::vector<int32_t> ph(W * L, 0), pe(W * L, neg), ch(W * L, 0), ce(W * L, neg);
  std::vector<uint8_t> trace((q_len + 1) * W * L, 0);
  std::vector<int32_t> best(L, 0), bi(L, 0), bj(L, 0), bq(L, 0), bqj(L, 0);
  std::vector<char> done(L, 0);
  for (size_t i = 1; i <= q_len; ++i) {
    for (size_t k = 0; k < L; ++k) {
      ch[0 * L + k] = 0;
      ce[0 * L + k] = neg;
      int32_t cf = neg;
      for (size_t j = 1; j <= r_len; ++j) {
        const int32_t s = reads[k][i - 1] == wins[k][j - 1] ? vm : vx;
        const int32_t hm = adds(ph[(j - 1) * L + k], s);
        const int32_t efh = adds(ph[j * L + k], go), efe = adds(pe[j * L + k], ge);
        const int32_t e = std::max(efh, efe);
        const int32_t ffh = adds(ch[(j - 1) * L + k], go), fff = adds(cf, ge);
        const int32_t f = std::max(ffh, fff);
        const int32_t h = std::max(std::max(std::max(hm, e), f), 0);
        ch[j * L + k] = h;
        ce[j * L + k] = e;
        cf = f;
        uint8_t tr = h == 0 ? 0 : (h == hm ? 1 : (h == e ? 2 : 3));
        if (efe > efh) tr |= TRACE_E_EXTEND;
        if (fff > ffh) tr |= TRACE_F_EXTEND;
        trace[(i * W + j) * L + k] = tr;
        if (h > best[k]) {
          best[k] = h;
          bi[k] = (int32_t)i;
          bj[k] = (int32_t)j;
        }
        if (i == q_len && h > bq[k]) {
          bq[k] = h;
          bqj[k] = (int32_t)j;
        }
      }
    }
    const int32_t remaining = (int32_t)(q_len - i);
    bool all_done = true;
    for (size_t k = 0; k < L; ++k) {
      if (done[k]) continue;
      if (aborts[k] > kI32Min / 8) {
        const int32_t mp = best[k] + remaining * cfg.match_score;
        if (mp < aborts[k]) done[k] = 1;
      }
      if (!done[k]) all_done = false;
    }
    if (all_done) break;
    std::swap(ph, ch);
    std::swap(pe, ce);
  }
  for (size_t k = 0; k < L; ++k)
    finish_lane(trace.data(), trace.size(), W, L, k, q_len, best[k], bi[k], bj[k], bq[k], bqj[k],
                cfg.clip_penalty, done[k] != 0, outs[k]);
}

// i16 fit check of sw_batch_avx2 (mod.rs:1854-1868).
bool i16_fits(size_t q_len, size_t r_len, const orc_cfg& cfg) {
  const int32_t max_lane = 32767;
  const bool costs_fit = cfg.match_score >= 0 && cfg.match_score <= max_lane && cfg.mismatch >= 0 &&
                         cfg.mismatch <= max_lane && cfg.gap_open >= 0 && cfg.gap_extend >= 0 &&
                         sat_add_i32(cfg.gap_open, cfg.gap_extend) <= max_lane;
  if (!costs_fit || q_len > (size_t)max_lane || r_len > (size_t)max_lane) return false;
  const int64_t mn = (int64_t)std::min(q_len, r_len) * cfg.match_score;
  return mn <= max_lane;
}

bool cpu_avx2() { return __builtin_cpu_supports("avx2"); }
bool cpu_vnni() {
#if defined(__GNUC__) && !defined(__clang__) && (__GNUC__ >= 11)
  return __builtin_cpu_supports("avxvnni");
#else
  return false;
#endif
}

// certificate (mod.rs:688-776).
size_t bounded_hamming(const uint8_t* a, size_t na, const uint8_t* b, size_t nb, size_t limit) {
  if (na != nb) return limit + 1;
  size_t m = 0;
  for (size_t i = 0; i < na; ++i) {
    m += a[i] != b[i] ? 1 : 0;
    if (m > limit) break;
  }
  return m;
}

bool certified(const uint8_t* read, const uint8_t* ref, size_t len, size_t mism, bool has_second,
               size_t second, size_t max_mism, bool strict) {
  if (mism > max_mism) return false;
  if (has_second && second <= mism + 1) return false;  // saturating_add never saturates here
  if (mism == 0) return true;
  if (mism > 2) return false;
  size_t pos[2] = {SIZE_MAX, SIZE_MAX};
  size_t n = 0;
  for (size_t i = 0; i < len; ++i)
    if (read[i] != ref[i]) {
      if (n < 2) pos[n] = i;
      ++n;
    }
  if (n != mism) return false;
  const size_t edge = std::min<size_t>(len, 8);
  for (size_t k = 0; k < n; ++k)
    if (pos[k] < edge || pos[k] + edge >= len) return false;
  if (n == 2 && (pos[1] > pos[0] ? pos[1] - pos[0] : 0) <= 4) return false;
  const size_t p = pos[0];
  const size_t suffix_len = len > p + 1 ? len - (p + 1) : 0;
  const size_t min_suffix = strict ? 4 : 8;
  if (suffix_len >= min_suffix) {
    const bool read_ins = bounded_hamming(read + p + 1, len - p - 1, ref + p, len - 1 - p, 1) <= 1;
    const bool ref_ins = bounded_hamming(read + p, len - 1 - p, ref + p + 1, len - p - 1, 1) <= 1;
    if (read_ins || ref_ins) return false;
    if (strict && suffix_len >= 6) {
      const bool r2 = bounded_hamming(read + p + 2, len - p - 2, ref + p, len - 2 - p, 1) <= 1;
      const bool f2 = bounded_hamming(read + p, len - 2 - p, ref + p + 2, len - p - 2, 1) <= 1;
      if (r2 || f2) return false;
    }
  }
  return true;
}

size_t spectral_max_mismatches(size_t read_len) {  // router.rs:191-195 (defaults 3 %, floor 2)
  return std::max<size_t>((read_len * 3) / 100, 2);
}
size_t myers_reject_bound(size_t read_len) {  // router.rs:199-203 (defaults 15 %, floor 4)
  return (read_len * 15) / 100 + 4;
}

constexpr uint32_t kStatusCertified = 1, kStatusMyersReject = 2, kStatusSw = 3;

void verify_pair(const uint8_t* read, size_t q, const uint8_t* win, size_t w,
                 const orc_verify_params& p, orc_verify_result* out, uint32_t* cigar,
                 uint32_t cap) {
  std::memset(out, 0, sizeof(*out));
  size_t shift = 0, mism = 0, second = 0;
  bool has_second = false;
  const bool hit = packed_scan(read, q, win, w, &shift, &mism, &has_second, &second);
  out->sieve_shift = hit ? (int32_t)shift : -1;
  out->sieve_mism = hit ? (int32_t)mism : INT32_MAX;
  out->sieve_second = hit && has_second ? (int32_t)second : INT32_MAX;
  out->myers_dist = -1;
  out->myers_end = -1;
  const size_t thr = p.sieve_threshold < 0 ? spectral_max_mismatches(q) : (size_t)p.sieve_threshold;
  if (hit && mism <= thr &&
      certified(read, win + shift, q, mism, has_second, second, thr, p.cert_strict != 0)) {
    // build_certified_spectral_alignment (mod.rs:636-686): ungapped qM.
    out->status = kStatusCertified;
    out->sw.score = (int32_t)(q - mism) * p.cfg.match_score - (int32_t)mism * p.cfg.mismatch;
    out->sw.ref_start = (uint32_t)shift;
    out->sw.ref_end = (uint32_t)(shift + q);
    out->sw.read_start = 0;
    out->sw.read_end = (int32_t)q;
    out->sw.n_cigar = 1;
    if (cigar && cap) cigar[0] = cig((uint32_t)q, 0);
    return;
  }
  const size_t k = p.myers_k < 0 ? myers_reject_bound(q) : (size_t)p.myers_k;
  size_t dist = 0, end = 0;
  if (!myers(read, q, win, w, k, 0, &dist, &end)) {
    out->status = kStatusMyersReject;
    return;
  }
  out->myers_dist = (int32_t)dist;
  out->myers_end = (int32_t)end;
  const int32_t offset = hit ? (int32_t)shift : 0;
  SwOut s = banded_sw_with(read, q, win, w, offset, p.cfg, p.abort_score, p.adaptive != 0,
                           p.max_drift, p.dp_xdrop);
  out->status = kStatusSw;
  emit(s, &out->sw, cigar, cap);
}

template <class F>
void parallel_for(uint32_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 2) {
    for (uint32_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        const uint32_t i0 = next.fetch_add(64);
        if (i0 >= n) break;
        const uint32_t i1 = std::min<uint32_t>(n, i0 + 64);
        for (uint32_t i = i0; i < i1; ++i) f(i);
      }
    });
  for (auto& th : pool) th.join();
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int orc_pack(const uint8_t* seq, size_t n, uint8_t* bits) {
  std::vector<uint8_t> b;
  const bool v = pack_into(seq, n, b);
  if (!b.empty()) std::memcpy(bits, b.data(), b.size());
  return v ? 1 : 0;
}

void orc_shift_bits_right(const uint8_t* bits, size_t nbytes, int off, uint8_t* out) {
  shift_bits_right(bits, nbytes, off, out);
}

void orc_pre_shift(const uint8_t* bits, size_t nbytes, uint8_t* out4) {  // bitpacked.rs:95-99
  for (int p = 0; p < 4; ++p) shift_bits_right(bits, nbytes, 2 * p, out4 + p * nbytes);
}

size_t orc_mismatch_count(const uint8_t* read, const uint8_t* ref, size_t n_bytes, size_t n_nucs) {
  return mismatch_count(read, ref, n_bytes, n_nucs);
}

int orc_scan_best_with_second_raw(const uint8_t* read_bits, size_t read_bytes, size_t read_len,
                                  int read_valid, const uint8_t* ref_pre4, size_t ref_bytes,
                                  size_t ref_len, int64_t* shift, int64_t* mism, int64_t* second) {
  const uint8_t* ph[4] = {ref_pre4, ref_pre4 + ref_bytes, ref_pre4 + 2 * ref_bytes,
                          ref_pre4 + 3 * ref_bytes};
  size_t s = 0, m = 0, sec = 0;
  bool hs = false;
  if (!scan_best_with_second_raw(read_bits, read_bytes, read_len, read_valid != 0, ph, ref_bytes,
                                 ref_len, &s, &m, &hs, &sec))
    return 0;
  *shift = (int64_t)s;
  *mism = (int64_t)m;
  *second = hs ? (int64_t)sec : -1;
  return 1;
}

int orc_scan(const uint8_t* read_bits, size_t read_bytes, size_t read_len, int read_valid,
             const uint8_t* ref_pre4, size_t ref_bytes, size_t ref_len, size_t max_mism,
             int64_t* shift, int64_t* mism) {  // bitpacked.rs:122-133
  if (!read_valid) return 0;
  int64_t sec;
  if (!orc_scan_best_with_second_raw(read_bits, read_bytes, read_len, 1, ref_pre4, ref_bytes,
                                     ref_len, shift, mism, &sec))
    return 0;
  return (uint64_t)*mism <= max_mism ? 1 : 0;
}

void orc_gpu_sieve_semantics(const uint8_t* read_bits, uint32_t read_nucs, const uint8_t* ref_bits,
                             uint32_t ref_nucs, uint32_t max_mismatches, int32_t* shift,
                             int32_t* mism, int32_t* second) {
  // spectral.cu:154-163 sentinels; rank order (mism, shift) as spectral.cu:183-203,
  // which is the same order scan_best_with_second_raw keeps. Limit: backend.rs:185-188.
  if (read_nucs == 0 || ref_nucs < read_nucs) {
    *shift = -1;
    *mism = INT32_MAX;
    *second = INT32_MAX;
    return;
  }
  const size_t rb = (read_nucs + 3) / 4, tb = (ref_nucs + 3) / 4;
  std::vector<uint8_t> ph(4 * tb);
  for (int p = 0; p < 4; ++p) shift_bits_right(ref_bits, tb, 2 * p, ph.data() + p * tb);
  const uint8_t* phases[4] = {ph.data(), ph.data() + tb, ph.data() + 2 * tb, ph.data() + 3 * tb};
  size_t s = 0, m = 0, sec = 0;
  bool hs = false;
  scan_best_with_second_raw(read_bits, rb, read_nucs, true, phases, tb, ref_nucs, &s, &m, &hs, &sec);
  const uint32_t limit = std::min(max_mismatches, read_nucs);
  const bool acc = m <= limit;
  *shift = acc ? (int32_t)s : -1;
  *mism = acc ? (int32_t)m : INT32_MAX;
  *second = hs ? (int32_t)sec : INT32_MAX;
}

// spectral.rs:15-76 (scalar; the AVX2 variant :81-146 returns the same hit).
int orc_byte_scan(const uint8_t* read, size_t r, const uint8_t* win, size_t w, size_t max_mism,
                  int64_t* shift, int64_t* mism) {
  if (r == 0 || w < r) return 0;
  const size_t n_shifts = w - r + 1;
  const size_t need = r > max_mism ? r - max_mism : 0;
  size_t best_matches = 0, best_shift = 0;
  for (size_t t = 0; t < n_shifts; ++t) {
    const size_t target = std::max(need, best_matches + 1);
    size_t matches = 0;
    for (size_t i = 0; i < r; ++i) {
      if (read[i] == win[t + i]) {
        ++matches;
      } else {
        const size_t remaining = r - i - 1;
        if (matches + remaining < target) {
          matches = 0;
          break;
        }
      }
    }
    if (matches > best_matches) {
      best_matches = matches;
      best_shift = t;
      if (best_matches == r) break;
    }
  }
  if (best_matches >= need) {
    *shift = (int64_t)best_shift;
    *mism = (int64_t)(r - best_matches);
    return 1;
  }
  return 0;
}

int orc_myers(const uint8_t* pat, size_t m, const uint8_t* text, size_t n, size_t max_k, int path,
              uint64_t* dist, uint64_t* end) {
  size_t d = 0, e = 0;
  if (!myers(pat, m, text, n, max_k, path, &d, &e)) return 0;
  *dist = d;
  *end = e;
  return 1;
}

int orc_banded_sw(const uint8_t* read, size_t q, const uint8_t* ref, size_t r, int32_t offset,
                  const orc_cfg* cfg, int32_t abort_score, int adaptive, int32_t max_drift,
                  int32_t dp_xdrop, orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  SwOut s = banded_sw_with(read, q, ref, r, offset, *cfg, abort_score, adaptive != 0, max_drift,
                           dp_xdrop);
  emit(s, out, cigar, cap);
  return 1;
}

// banded_sw_with plus its DP matrix: h and tr are (q + 1) x row_cap, row i holding
// row_len[i] cells from window column row_start[i] (test infrastructure: checks of
// traceback forms that do not store the STOP direction).
int orc_banded_sw_matrix(const uint8_t* read, size_t q, const uint8_t* ref, size_t r,
                         int32_t offset, const orc_cfg* cfg, int32_t abort_score, int adaptive,
                         int32_t max_drift, int32_t dp_xdrop, orc_sw_result* out, uint32_t* cigar,
                         uint32_t cap, int32_t* row_start, int32_t* row_len, int32_t* h,
                         uint8_t* tr, size_t row_cap) {
  SwOut s = banded_sw_with(read, q, ref, r, offset, *cfg, abort_score, adaptive != 0, max_drift,
                           dp_xdrop, true);
  emit(s, out, cigar, cap);
  for (size_t i = 0; i <= q; ++i) {
    const auto& hr = s.h_rows[i];
    const auto& trr = s.trace_rows[i];
    row_start[i] = s.row_starts[i];
    row_len[i] = (int32_t)std::min(hr.size(), trr.size());
    if ((size_t)row_len[i] > row_cap) return -1;
    for (size_t c = 0; c < (size_t)row_len[i]; ++c) {
      h[i * row_cap + c] = hr[c];
      tr[i * row_cap + c] = trr[c];
    }
  }
  return 1;
}

int orc_cpu_has_avx2(void) { return cpu_avx2() ? 1 : 0; }
int orc_cpu_has_avx_vnni(void) { return cpu_vnni() ? 1 : 0; }

int orc_sw_batch_avx2(int n, const uint8_t* const* reads, const uint8_t* const* wins, size_t q,
                      size_t r, const int32_t* aborts, const int32_t* scalar_offsets,
                      const orc_cfg* cfg, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                      orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  if (n <= 0 || n > 16) return -1;
  std::vector<SwOut> outs((size_t)n);
  if (!i16_fits(q, r, *cfg)) {  // scalar banded fallback per input (BatchInput::scalar_sw)
    for (int k = 0; k < n; ++k) {
      SwOut s = banded_sw_with(reads[k], q, wins[k], r, scalar_offsets[k], *cfg, aborts[k],
                               adaptive != 0, max_drift, dp_xdrop);
      emit(s, out + k, cigar ? cigar + (size_t)k * cap : nullptr, cap);
    }
    return 0;
  }
  sw_avx2_inner(n, reads, wins, q, r, aborts, *cfg, outs.data());
  for (int k = 0; k < n; ++k) {
    outs[k].cells = (uint64_t)q * r;
    emit(outs[k], out + k, cigar ? cigar + (size_t)k * cap : nullptr, cap);
  }
  return 1;
}

int orc_sw_full_window_model(int n, const uint8_t* const* reads, const uint8_t* const* wins,
                             size_t q, size_t r, const int32_t* aborts, const orc_cfg* cfg, int bits,
                             orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  if (n <= 0) return -1;
  std::vector<SwOut> outs((size_t)n);
  sw_full_window_model(n, reads, wins, q, r, aborts, *cfg, bits, outs.data());
  for (int k = 0; k < n; ++k) {
    outs[k].cells = (uint64_t)q * r;
    emit(outs[k], out + k, cigar ? cigar + (size_t)k * cap : nullptr, cap);
  }
  return 1;
}

int orc_int8_path_viable(size_t read_len, const orc_cfg* cfg) { return int8_viable(read_len, *cfg); }

int orc_sw_batch_int8(int n, const uint8_t* const* reads, const uint8_t* const* wins, size_t q,
                      size_t r, const int32_t* aborts, const int32_t* scalar_offsets,
                      const orc_cfg* cfg, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                      orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  if (n <= 0 || n > 32) return -1;
  std::vector<SwOut> outs((size_t)n);
  bool sat[32] = {};
  sw_int8_inner(n, reads, wins, q, r, aborts, *cfg, outs.data(), sat);
  for (int k = 0; k < n; ++k) {
    if (sat[k]) {  // sw_int8_vnni.rs:339-343: saturated lane re-runs the scalar banded SW
      outs[k] = banded_sw_with(reads[k], q, wins[k], r, scalar_offsets[k], *cfg, aborts[k],
                               adaptive != 0, max_drift, dp_xdrop);
    } else {
      outs[k].cells = (uint64_t)q * r;
    }
    emit(outs[k], out + k, cigar ? cigar + (size_t)k * cap : nullptr, cap);
  }
  return 1;
}

int orc_align_batch_simd(int n, const uint8_t* const* reads, const uint32_t* read_lens,
                         const uint8_t* const* wins, const uint32_t* win_lens,
                         const int32_t* aborts, const int32_t* scalar_offsets, const orc_cfg* cfg,
                         int mode, int detected, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                         orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  if (n <= 0) return 0;  // mod.rs:1116-1118
  const uint32_t q = read_lens[0], r = win_lens[0];
  bool mixed = false;
  for (int k = 0; k < n; ++k) mixed = mixed || read_lens[k] != q || win_lens[k] != r;
  auto scalar_all = [&]() {
    for (int k = 0; k < n; ++k) {
      SwOut s = banded_sw_with(reads[k], read_lens[k], wins[k], win_lens[k], scalar_offsets[k],
                               *cfg, aborts[k], adaptive != 0, max_drift, dp_xdrop);
      emit(s, out + k, cigar ? cigar + (size_t)k * cap : nullptr, cap);
    }
  };
  if (mixed) {  // mod.rs:1121-1129
    scalar_all();
    return 0;
  }
  enum { kScalar = 0, kAvx2 = 1, kVnni = 2 };
  auto avx2_chunks = [&]() {
    for (int k0 = 0; k0 < n; k0 += 16) {
      const int m = std::min(16, n - k0);
      orc_sw_batch_avx2(m, reads + k0, wins + k0, q, r, aborts + k0, scalar_offsets + k0, cfg,
                        adaptive, max_drift, dp_xdrop, out + k0,
                        cigar ? cigar + (size_t)k0 * cap : nullptr, cap);
    }
  };
  if (mode == kVnni && detected == kVnni) {  // sw_dispatch_avx_vnni (mod.rs:1824-1841)
    if (int8_viable(q, *cfg) && n <= 32) {
      orc_sw_batch_int8(n, reads, wins, q, r, aborts, scalar_offsets, cfg, adaptive, max_drift,
                        dp_xdrop, out, cigar, cap);
      return 2;
    }
    avx2_chunks();
    return 1;
  }
  if (mode == kAvx2 && (detected == kAvx2 || detected == kVnni)) {
    avx2_chunks();
    return 1;
  }
  scalar_all();
  return 0;
}

int orc_spectral_certified(const uint8_t* read, const uint8_t* ref_aligned, size_t len, size_t mism,
                           int64_t second, size_t max_mism, int strict) {
  return certified(read, ref_aligned, len, mism, second >= 0, second >= 0 ? (size_t)second : 0,
                   max_mism, strict != 0)
             ? 1
             : 0;
}

size_t orc_spectral_max_mismatches(size_t read_len) { return spectral_max_mismatches(read_len); }
size_t orc_myers_reject_bound(size_t read_len) { return myers_reject_bound(read_len); }

int orc_verify_pair(const uint8_t* read, size_t q, const uint8_t* win, size_t w,
                    const orc_verify_params* p, orc_verify_result* out, uint32_t* cigar,
                    uint32_t cap) {
  verify_pair(read, q, win, w, *p, out, cigar, cap);
  return out->status;
}

int orc_verify_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                     const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                     const uint32_t* win_len, const orc_verify_params* p, int nthreads,
                     orc_verify_result* out, uint32_t* cigar, uint32_t cap) {
  parallel_for(n, nthreads, [&](uint32_t i) {
    verify_pair(reads + read_off[i], read_len[i], wins + win_off[i], win_len[i], *p, out + i,
                cigar ? cigar + (size_t)i * cap : nullptr, cap);
  });
  return 0;
}

int orc_banded_sw_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                        const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                        const uint32_t* win_len, const int32_t* offsets, const orc_cfg* cfg,
                        int32_t abort_score, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                        int nthreads, orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  parallel_for(n, nthreads, [&](uint32_t i) {
    SwOut s = banded_sw_with(reads + read_off[i], read_len[i], wins + win_off[i], win_len[i],
                             offsets ? offsets[i] : 0, *cfg, abort_score, adaptive != 0, max_drift,
                             dp_xdrop);
    emit(s, out + i, cigar ? cigar + (size_t)i * cap : nullptr, cap);
  });
  return 0;
}

int orc_sw_avx2_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off, uint32_t q,
                      const uint8_t* wins, const uint64_t* win_off, uint32_t r, const orc_cfg* cfg,
                      int nthreads, orc_sw_result* out, uint32_t* cigar, uint32_t cap) {
  const uint32_t chunks = (n + 15) / 16;
  parallel_for(chunks, nthreads, [&](uint32_t c) {
    const uint32_t k0 = c * 16, m = std::min<uint32_t>(16, n - k0);
    const uint8_t* rp[16];
    const uint8_t* wp[16];
    int32_t ab[16], off[16];
    for (uint32_t k = 0; k < m; ++k) {
      rp[k] = reads + read_off[k0 + k];
      wp[k] = wins + win_off[k0 + k];
      ab[k] = kI32Min / 8;
      off[k] = 0;
    }
    orc_sw_batch_avx2((int)m, rp, wp, q, r, ab, off, cfg, 1, 16, cfg->xdrop, out + k0,
                      cigar ? cigar + (size_t)k0 * cap : nullptr, cap);
  });
  return 0;
}

int orc_myers_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                    const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                    const uint32_t* win_len, uint32_t max_k, int nthreads, int64_t* dist,
                    int64_t* end) {
  parallel_for(n, nthreads, [&](uint32_t i) {
    size_t d = 0, e = 0;
    if (myers(reads + read_off[i], read_len[i], wins + win_off[i], win_len[i], max_k, 0, &d, &e)) {
      dist[i] = (int64_t)d;
      end[i] = (int64_t)e;
    } else {
      dist[i] = -1;
      end[i] = -1;
    }
  });
  return 0;
}

int orc_sieve_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                    const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                    const uint32_t* win_len, int nthreads, int32_t* shift, int32_t* mism,
                    int32_t* second) {
  parallel_for(n, nthreads, [&](uint32_t i) {
    size_t s = 0, m = 0, sec = 0;
    bool hs = false;
    if (packed_scan(reads + read_off[i], read_len[i], wins + win_off[i], win_len[i], &s, &m, &hs,
                    &sec)) {
      shift[i] = (int32_t)s;
      mism[i] = (int32_t)m;
      second[i] = hs ? (int32_t)sec : INT32_MAX;
    } else {
      shift[i] = -1;
      mism[i] = INT32_MAX;
      second[i] = INT32_MAX;
    }
  });
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// NM / MD:Z (src/alignment/md.rs). MdBuilder (md.rs:24-133): a match extends
// the run; a mismatch writes the run count and the reference letter; a deletion
// writes the count, '^' and the deleted reference letters; an insertion only
// adds to NM; a skip is invisible; the string always ends with a count.
// ---------------------------------------------------------------------------
namespace {

struct Md {
  std::string text;
  uint32_t run = 0, nm = 0;
  void flush() {
    text += std::to_string(run);
    run = 0;
  }
  // reference_letter (md.rs:52-58): ASCII letters upper-cased, anything else 'N'.
  static char letter(uint8_t b) {
    const bool alpha = (b >= 'A' && b <= 'Z') || (b >= 'a' && b <= 'z');
    return alpha ? (char)(b & 0xDF) : 'N';
  }
  void matched() { ++run; }
  void mismatch(uint8_t rb) {
    flush();
    text += letter(rb);
    ++nm;
  }
  // identical_base_is_edit (md.rs:135-138)
  static bool ident_edit(uint8_t b) {
    const uint8_t u = (b >= 'a' && b <= 'z') ? (uint8_t)(b - 32) : b;
    return !(u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == '=');
  }
  // column (md.rs:77-86): '=' or case-insensitive equality extends the run.
  void column(uint8_t qb, uint8_t rb) {
    const auto low = [](uint8_t c) { return (c >= 'A' && c <= 'Z') ? (uint8_t)(c + 32) : c; };
    if (qb == '=' || low(qb) == low(rb)) {
      matched();
      nm += ident_edit(qb) ? 1u : 0u;
    } else {
      mismatch(rb);
    }
  }
  void insertion(uint32_t len) { nm += len; }
  void deletion(const uint8_t* bases, size_t len) {
    if (!len) return;
    flush();
    text += '^';
    for (size_t i = 0; i < len; ++i) text += letter(bases[i]);
    nm += (uint32_t)len;
  }
  uint32_t finish(uint32_t* nm_out, char* md, uint32_t cap) {
    flush();
    *nm_out = nm;
    std::memcpy(md, text.data(), std::min<size_t>(cap, text.size()));
    return (uint32_t)text.size();
  }
};

}  // namespace

extern "C" uint32_t orc_nm_md(const uint8_t* read, size_t read_len, const uint8_t* ref,
                              size_t ref_len, size_t read_start, size_t ref_start,
                              const uint32_t* cigar, uint32_t n_cigar, uint32_t* nm, char* md,
                              uint32_t md_cap) {
  Md b;
  size_t q = read_start, r = ref_start;
  for (uint32_t k = 0; k < n_cigar; ++k) {
    const size_t len = cigar[k] >> 4;
    switch (cigar[k] & 15u) {
      case 0:  // M: positions past either end read as 'N' (md.rs:176-181)
        for (size_t t = 0; t < len; ++t, ++q, ++r)
          b.column(q < read_len ? read[q] : 'N', r < ref_len ? ref[r] : 'N');
        break;
      case 1:
        b.insertion((uint32_t)len);
        q += len;
        break;
      case 2: {  // D: bases past the reference end still count toward NM (md.rs:188-194)
        const size_t end = std::min(r + len, ref_len), start = std::min(r, end);
        b.deletion(ref + start, end - start);
        b.nm += (uint32_t)(len - (end - start));
        r += len;
        break;
      }
      case 3:
        r += len;
        break;
      default:  // S
        q += len;
        break;
    }
  }
  return b.finish(nm, md, md_cap);
}

extern "C" uint32_t orc_md_builder(const char* script, const uint8_t* read, const uint8_t* ref,
                                   const uint32_t* lens, uint32_t n, uint32_t* nm, char* md,
                                   uint32_t md_cap) {
  Md b;
  size_t at = 0;
  for (uint32_t i = 0; i < n; ++i) {
    switch (script[i]) {
      case 'M': b.matched(); break;
      case 'X': b.mismatch(ref[at++]); break;
      case 'C': b.column(read[at], ref[at]); ++at; break;
      case 'I': b.insertion(lens[i]); break;
      case 'D': b.deletion(ref + at, lens[i]); at += lens[i]; break;
      default: break;
    }
  }
  return b.finish(nm, md, md_cap);
}

extern "C" int orc_nm_md_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                               const uint32_t* read_len, const uint8_t* wins,
                               const uint64_t* win_off, const uint32_t* win_len,
                               const int32_t* read_start, const uint32_t* ref_start,
                               const uint32_t* cig_off, const uint32_t* n_cig,
                               const uint32_t* ops, int nthreads, uint32_t* nm,
                               uint32_t* md_len, char* md, uint32_t md_stride) {
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(64);
      if (i >= n) return;
      for (uint32_t p = i; p < std::min(n, i + 64); ++p) {
        if (!n_cig[p]) {
          nm[p] = 0xFFFFFFFFu;
          md_len[p] = 0;
          continue;
        }
        md_len[p] = orc_nm_md(reads + read_off[p], read_len[p], wins + win_off[p], win_len[p],
                              (size_t)read_start[p], ref_start[p], ops + cig_off[p], n_cig[p],
                              nm + p, md + (size_t)p * md_stride, md_stride);
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < std::max(nthreads, 1); ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  return 0;
}

// ---------------------------------------------------------------------------
// WFA (src/alignment/wfa.rs): wfa_align_with_costs (:549-648), step (:374-526),
// extend_wavefront (:277-291), prune_wavefront (:293-346), check_done
// (:348-358), build_cigar (:762-952). Same recurrence, same edge order.
// ---------------------------------------------------------------------------
namespace {

constexpr int32_t kWfaNone = INT32_MIN / 4;

struct Wf {
  int32_t lo = 0, hi = -1;
  std::vector<int32_t> off;
  bool empty() const { return hi < lo; }
  int32_t get(int32_t k) const { return (k < lo || k > hi) ? kWfaNone : off[(size_t)(k - lo)]; }
};

struct WfaCostsO {
  int32_t x, o, ei, ed;
};

int32_t wfa_extend_diag(const uint8_t* p, int32_t m, const uint8_t* t, int32_t n, int32_t k,
                        int32_t off) {
  for (;;) {
    const int32_t i = off, j = off + k;
    if (i >= m || j < 0 || j >= n) break;
    if (p[i] != t[j]) break;
    ++off;
  }
  return off;
}

void wfa_extend(const uint8_t* p, int32_t m, const uint8_t* t, int32_t n, Wf& w) {
  for (int32_t k = w.lo; k <= w.hi; ++k) {
    int32_t& o = w.off[(size_t)(k - w.lo)];
    if (o != kWfaNone) o = wfa_extend_diag(p, m, t, n, k, o);
  }
}

void wfa_prune(Wf& w, int32_t drop) {
  if (w.empty()) return;
  int32_t max_ad = INT32_MIN;
  for (int32_t k = w.lo; k <= w.hi; ++k) {
    const int32_t o = w.off[(size_t)(k - w.lo)];
    if (o != kWfaNone) max_ad = std::max(max_ad, 2 * o + k);
  }
  if (max_ad == INT32_MIN) return;
  const int32_t th = max_ad - drop;
  int32_t lo = w.lo;
  while (lo <= w.hi) {
    const int32_t o = w.off[(size_t)(lo - w.lo)];
    if (o != kWfaNone && 2 * o + lo >= th) break;
    ++lo;
  }
  int32_t hi = w.hi;
  while (hi >= lo) {
    const int32_t o = w.off[(size_t)(hi - w.lo)];
    if (o != kWfaNone && 2 * o + hi >= th) break;
    --hi;
  }
  if (lo > hi) {
    w = Wf();
    return;
  }
  std::vector<int32_t> nv((size_t)(hi - lo + 1));
  for (int32_t k = lo; k <= hi; ++k) {
    int32_t o = w.off[(size_t)(k - w.lo)];
    if (o != kWfaNone && 2 * o + k < th) o = kWfaNone;
    nv[(size_t)(k - lo)] = o;
  }
  w.lo = lo;
  w.hi = hi;
  w.off.swap(nv);
}

bool wfa_done(const Wf& w, int32_t m, int32_t* k_end) {
  for (int32_t k = w.lo; k <= w.hi; ++k)
    if (w.off[(size_t)(k - w.lo)] >= m) {
      *k_end = k;
      return true;
    }
  return false;
}

const Wf* wfa_src(const std::vector<Wf>& h, int32_t s) {
  if (s < 0 || (size_t)s >= h.size() || h[(size_t)s].empty()) return nullptr;
  return &h[(size_t)s];
}

void wfa_step(int32_t s, const WfaCostsO& c, const std::vector<Wf>& M, const std::vector<Wf>& I,
              const std::vector<Wf>& D, int32_t m, int32_t n, Wf& nm, Wf& ni, Wf& nd) {
  const Wf* mx = wfa_src(M, s - c.x);
  const Wf* moi = wfa_src(M, s - c.o - c.ei);
  const Wf* mod = wfa_src(M, s - c.o - c.ed);
  const Wf* ie = wfa_src(I, s - c.ei);
  const Wf* de = wfa_src(D, s - c.ed);
  int32_t ilo = INT32_MAX, ihi = INT32_MIN, dlo = INT32_MAX, dhi = INT32_MIN;
  if (moi) ilo = std::min(ilo, moi->lo - 1), ihi = std::max(ihi, moi->hi - 1);
  if (ie) ilo = std::min(ilo, ie->lo - 1), ihi = std::max(ihi, ie->hi - 1);
  if (mod) dlo = std::min(dlo, mod->lo + 1), dhi = std::max(dhi, mod->hi + 1);
  if (de) dlo = std::min(dlo, de->lo + 1), dhi = std::max(dhi, de->hi + 1);
  int32_t mlo = INT32_MAX, mhi = INT32_MIN;
  if (mx) mlo = std::min(mlo, mx->lo), mhi = std::max(mhi, mx->hi);
  if (ilo <= ihi) mlo = std::min(mlo, ilo), mhi = std::max(mhi, ihi);
  if (dlo <= dhi) mlo = std::min(mlo, dlo), mhi = std::max(mhi, dhi);
  ni = Wf();
  if (ilo <= ihi) {
    ni.lo = ilo, ni.hi = ihi, ni.off.assign((size_t)(ihi - ilo + 1), kWfaNone);
    for (int32_t k = ilo; k <= ihi; ++k) {
      int32_t b = kWfaNone;
      if (moi) {
        const int32_t v = moi->get(k + 1);
        if (v != kWfaNone && v < m) b = std::max(b, v + 1);
      }
      if (ie) {
        const int32_t v = ie->get(k + 1);
        if (v != kWfaNone && v < m) b = std::max(b, v + 1);
      }
      ni.off[(size_t)(k - ilo)] = b;
    }
  }
  nd = Wf();
  if (dlo <= dhi) {
    nd.lo = dlo, nd.hi = dhi, nd.off.assign((size_t)(dhi - dlo + 1), kWfaNone);
    for (int32_t k = dlo; k <= dhi; ++k) {
      int32_t b = kWfaNone;
      if (mod) {
        const int32_t v = mod->get(k - 1);
        if (v != kWfaNone && v + k <= n) b = std::max(b, v);
      }
      if (de) {
        const int32_t v = de->get(k - 1);
        if (v != kWfaNone && v + k <= n) b = std::max(b, v);
      }
      nd.off[(size_t)(k - dlo)] = b;
    }
  }
  nm = Wf();
  if (mlo <= mhi) {
    nm.lo = mlo, nm.hi = mhi, nm.off.assign((size_t)(mhi - mlo + 1), kWfaNone);
    for (int32_t k = mlo; k <= mhi; ++k) {
      int32_t b = kWfaNone;
      if (mx) {
        const int32_t v = mx->get(k);
        if (v != kWfaNone && v < m && v + k < n) b = std::max(b, v + 1);
      }
      const int32_t vi = ni.get(k);
      if (vi != kWfaNone) b = std::max(b, vi);
      const int32_t vd = nd.get(k);
      if (vd != kWfaNone) b = std::max(b, vd);
      nm.off[(size_t)(k - mlo)] = b;
    }
  }
}

struct CigarRev {  // push_cigar (wfa.rs:954-962) on the reversed op list
  std::vector<uint32_t> ops;
  void push(uint32_t op, uint32_t len) {
    if (!ops.empty() && (ops.back() & 15u) == op) {
      ops.back() += len << 4;
      return;
    }
    ops.push_back((len << 4) | op);
  }
};

int32_t wfa_traceback(const uint8_t* p, int32_t m, const uint8_t* t, int32_t n,
                      const std::vector<Wf>& M, const std::vector<Wf>& I,
                      const std::vector<Wf>& D, int32_t s, int32_t k, const WfaCostsO& c,
                      CigarRev& cr) {
  int32_t off = m;
  int layer = 0;  // 0 M, 1 I, 2 D
  auto get = [&](int L, int32_t sc, int32_t kk) -> int32_t {
    const std::vector<Wf>& h = L == 0 ? M : (L == 1 ? I : D);
    if (sc < 0 || (size_t)sc >= h.size()) return kWfaNone;
    const Wf& w = h[(size_t)sc];
    return w.empty() ? kWfaNone : w.get(kk);
  };
  while (!(s == 0 && layer == 0 && off == 0)) {
    if (layer == 0) {
      int32_t walk = off;
      while (walk != 0) {
        if (get(1, s, k) == walk) break;
        if (get(2, s, k) == walk) break;
        if (s >= c.x) {
          const int32_t prev = get(0, s - c.x, k);
          if (prev != kWfaNone && prev + 1 == walk) break;
        }
        const int32_t i = walk - 1, j = walk - 1 + k;
        if (i < 0 || j < 0 || i >= m || j >= n) break;
        if (p[i] != t[j]) break;
        --walk;
      }
      if (off - walk > 0) cr.push(0, (uint32_t)(off - walk));
      off = walk;
      if (s == 0 && off == 0) break;
      bool took = false;
      if (s >= c.x) {
        const int32_t prev = get(0, s - c.x, k);
        if (prev != kWfaNone && prev + 1 == off) {
          cr.push(0, 1);
          off -= 1;
          s -= c.x;
          took = true;
        }
      }
      if (!took && get(1, s, k) == off) layer = 1, took = true;
      if (!took && get(2, s, k) == off) layer = 2, took = true;
      if (!took) break;
    } else if (layer == 1) {
      bool took = false;
      if (s >= c.o + c.ei) {
        const int32_t prev = get(0, s - c.o - c.ei, k + 1);
        if (prev != kWfaNone && prev + 1 == off) {
          cr.push(1, 1);
          off -= 1, k += 1, s -= c.o + c.ei, layer = 0, took = true;
        }
      }
      if (!took && s >= c.ei) {
        const int32_t prev = get(1, s - c.ei, k + 1);
        if (prev != kWfaNone && prev + 1 == off) {
          cr.push(1, 1);
          off -= 1, k += 1, s -= c.ei, took = true;
        }
      }
      if (!took) break;
    } else {
      bool took = false;
      if (s >= c.o + c.ed) {
        const int32_t prev = get(0, s - c.o - c.ed, k - 1);
        if (prev != kWfaNone && prev == off) {
          cr.push(2, 1);
          k -= 1, s -= c.o + c.ed, layer = 0, took = true;
        }
      }
      if (!took && s >= c.ed) {
        const int32_t prev = get(2, s - c.ed, k - 1);
        if (prev != kWfaNone && prev == off) {
          cr.push(2, 1);
          k -= 1, s -= c.ed, took = true;
        }
      }
      if (!took) break;
    }
  }
  return k;
}

}  // namespace

extern "C" int orc_wfa(const uint8_t* pattern, size_t m_, const uint8_t* text, size_t n_,
                       const orc_wfa_cfg* cfg, int32_t* score, uint32_t* text_start,
                       uint32_t* text_end, uint32_t* cigar, uint32_t cap, uint32_t* n_cigar) {
  const int32_t m = (int32_t)m_, n = (int32_t)n_;
  *n_cigar = 0;
  WfaCostsO c;
  if (cfg->scored) {  // WfaCosts::scored (wfa.rs:41-52)
    if (cfg->match_score <= 0 || cfg->mismatch <= 0 || cfg->gap_open < 0 || cfg->gap_extend <= 0)
      return -1;
    c = {cfg->match_score + cfg->mismatch, cfg->gap_open, cfg->match_score + cfg->gap_extend,
         cfg->gap_extend};
  } else {
    c = {cfg->mismatch, cfg->gap_open, cfg->gap_extend, cfg->gap_extend};
  }
  if (m == 0) {
    *score = 0, *text_start = 0, *text_end = 0;
    return 1;
  }
  const int32_t tbf = std::min(std::max(cfg->text_begin_free, 0), std::max(n - 1, 0));
  std::vector<Wf> M, I, D;
  Wf m0;
  m0.lo = 0, m0.hi = tbf, m0.off.assign((size_t)(tbf + 1), 0);
  wfa_extend(pattern, m, text, n, m0);
  if (cfg->adaptive_drop >= 0) wfa_prune(m0, cfg->adaptive_drop);
  int32_t k_end = 0, s_end = -1;
  M.push_back(m0), I.push_back(Wf()), D.push_back(Wf());
  if (wfa_done(M[0], m, &k_end)) s_end = 0;
  for (int32_t s = 1; s_end < 0 && s <= cfg->max_score; ++s) {
    Wf nm, ni, nd;
    wfa_step(s, c, M, I, D, m, n, nm, ni, nd);
    wfa_extend(pattern, m, text, n, nm);
    if (cfg->adaptive_drop >= 0) wfa_prune(nm, cfg->adaptive_drop);
    M.push_back(nm), I.push_back(ni), D.push_back(nd);
    if (wfa_done(M[(size_t)s], m, &k_end)) s_end = s;
  }
  if (s_end < 0) return 0;
  *score = s_end;
  *text_end = (uint32_t)(m + k_end);
  *text_start = 0;
  if (cfg->traceback) {
    CigarRev cr;
    const int32_t k0 = wfa_traceback(pattern, m, text, n, M, I, D, s_end, k_end, c, cr);
    *text_start = (uint32_t)std::max(k0, 0);
    const uint32_t nc = (uint32_t)cr.ops.size();
    for (uint32_t t = 0; t < nc && t < cap; ++t) cigar[t] = cr.ops[nc - 1 - t];
    *n_cigar = nc;
  }
  return 1;
}

extern "C" int orc_wfa_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                             const uint32_t* read_len, const uint8_t* wins,
                             const uint64_t* win_off, const uint32_t* win_len,
                             const orc_wfa_cfg* c, int nthreads, int32_t* found, int32_t* score,
                             uint32_t* text_start, uint32_t* text_end, uint32_t* n_cigar,
                             uint32_t* cigar, uint32_t cap_per_pair) {
  std::atomic<uint32_t> next{0};
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(16);
      if (i >= n) return;
      for (uint32_t p = i; p < std::min(n, i + 16); ++p)
        found[p] = orc_wfa(reads + read_off[p], read_len[p], wins + win_off[p], win_len[p], c,
                           score + p, text_start + p, text_end + p,
                           cigar + (size_t)p * cap_per_pair, cap_per_pair, n_cigar + p);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < std::max(nthreads, 1); ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  return 0;
}

// ---------------------------------------------------------------------------
// Ungapped extension prefilter (src/alignment/prefilter.rs) and exact matches
// (src/alignment/mod.rs:779-832). count_mismatches (kira-simd 0.1.0,
// compare::count_mismatches) is the number of unequal bytes of two equal-length
// slices; every call site passes equal lengths.
// ---------------------------------------------------------------------------
namespace {

size_t pf_count_mismatches(const uint8_t* a, const uint8_t* b, size_t n) {
  size_t c = 0;
  for (size_t i = 0; i < n; ++i) c += a[i] != b[i];
  return c;
}

// identity_x10000 (prefilter.rs:84-91)
uint16_t pf_identity_x10000(size_t len, size_t mism) {
  if (len == 0) return 0;
  const uint64_t matches = len > mism ? len - mism : 0;
  uint64_t prod = matches * 10000ull;
  if (prod > UINT32_MAX) prod = UINT32_MAX;  // u32 saturating_mul
  const uint64_t id = prod / (uint32_t)len;
  return (uint16_t)std::min<uint64_t>(id, 65535);
}

// min_len_required (prefilter.rs:297-315)
size_t pf_min_len_required(size_t read_len, uint16_t id, size_t mism, size_t span_slack) {
  size_t slack = 0;
  if (id >= 9933) slack = 15;
  else if (id >= 9900 && mism <= 2) slack = 10;
  else if (id >= 9870 && mism <= 3) slack = 5;
  if (span_slack > 0) slack = std::min(slack, span_slack);
  const size_t min_len = read_len > slack ? read_len - slack : 0;
  const size_t floor = read_len * 85 / 100;
  return std::max(floor, min_len);
}

// ungapped_extend (prefilter.rs:356-453): x-drop over 32-byte blocks on each
// side of the anchor, then the sub-block remainder when the walk did not drop.
void pf_ungapped_extend(const uint8_t* read, size_t read_len, const uint8_t* ref, size_t ref_len,
                        const orc_chain& c, const orc_prefilter_cfg& cfg, size_t* left_out,
                        size_t* right_out) {
  const size_t block = 32;
  size_t left = 0, right = 0;
  const size_t max_left = std::min(c.read_start, c.ref_start);
  const size_t max_right = std::min<size_t>(read_len - c.read_end, ref_len - c.ref_end);
  for (int side = 0; side < 2; ++side) {
    const size_t maxe = side ? max_right : max_left;
    size_t& ext = side ? right : left;
    int32_t score = 0, best = 0;
    size_t i = 0;
    bool broke = false;
    auto offs = [&](size_t at, size_t len, size_t* ro, size_t* fo) {
      if (side == 0) {
        *ro = c.read_start - at - len;
        *fo = c.ref_start - at - len;
      } else {
        *ro = c.read_end + at;
        *fo = c.ref_end + at;
      }
    };
    while (i + block <= maxe) {
      size_t ro, fo;
      offs(i, block, &ro, &fo);
      const int32_t mism = (int32_t)pf_count_mismatches(read + ro, ref + fo, block);
      score += ((int32_t)block - mism) * cfg.match_score - mism * cfg.mismatch;
      if (score > best) {
        best = score;
        ext = i + block;
      } else if (best - score > cfg.xdrop) {
        broke = true;
        break;
      }
      i += block;
    }
    if (cfg.tail && !broke && i < maxe) {
      const size_t rem = maxe - i;
      size_t ro, fo;
      offs(i, rem, &ro, &fo);
      const int32_t mism = (int32_t)pf_count_mismatches(read + ro, ref + fo, rem);
      score += ((int32_t)rem - mism) * cfg.match_score - mism * cfg.mismatch;
      if (score > best) ext = i + rem;
    }
  }
  *left_out = left;
  *right_out = right;
}

}  // namespace

extern "C" uint32_t orc_identical_nm(const uint8_t* bases, size_t len) {
  uint32_t nm = 0;  // md::identical_nm (md.rs:134-145)
  for (size_t i = 0; i < len; ++i) {
    const uint8_t u = (bases[i] >= 'a' && bases[i] <= 'z') ? bases[i] - 32 : bases[i];
    nm += !(u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == '=');
  }
  return nm;
}

extern "C" int orc_exact_match_exists(const uint8_t* read, size_t read_len, const uint8_t* ref,
                                      size_t ref_len, const orc_chain* c) {
  // exact_match_exists (mod.rs:819-832)
  if (c->read_start != 0 || c->read_end != read_len || c->ref_end < c->ref_start ||
      c->ref_end - c->ref_start != read_len)
    return 0;
  const size_t start = c->ref_start;
  if (start + read_len > ref_len) return 0;
  return pf_count_mismatches(read, ref + start, read_len) == 0;
}

extern "C" int orc_prefilter(const uint8_t* read, size_t read_len, const uint8_t* ref,
                             size_t ref_len, const orc_chain* cp, int is_top1,
                             int32_t score_margin, const orc_prefilter_cfg* cfgp,
                             orc_prefilter_out* out, char* md, size_t md_cap) {
  // prefilter_chain (prefilter.rs:93-294)
  const orc_chain& c = *cp;
  const orc_prefilter_cfg& cfg = *cfgp;
  *out = orc_prefilter_out{};
  auto other = [&](int code) {
    out->result = 2;
    out->reason = 9;
    out->other = code;
    return 0;
  };
  if (read_len == 0) return other(1);
  if (c.read_start > c.read_end || c.ref_start > c.ref_end) return other(2);
  const size_t anchor = c.read_end - c.read_start;
  if (anchor == 0) return other(3);
  if (c.read_end > read_len || c.ref_end > ref_len) return -1;
  size_t left = 0, right = 0;
  pf_ungapped_extend(read, read_len, ref, ref_len, c, cfg, &left, &right);
  const size_t total = anchor + left + right;
  if (total == 0) return other(4);
  const int64_t urs = (int64_t)c.read_start - (int64_t)left;
  const int64_t ufs = (int64_t)c.ref_start - (int64_t)left;
  if (urs < 0 || ufs < 0) return other(5);
  if ((size_t)urs + total > read_len || (size_t)ufs + total > ref_len) return other(6);
  const size_t ham = pf_count_mismatches(read + urs, ref + ufs, total);
  const int32_t score = (int32_t)(total > ham ? total - ham : 0) * cfg.match_score -
                        (int32_t)ham * cfg.mismatch;
  const uint16_t len16 = (uint16_t)std::min<size_t>(total, 65535);
  const uint16_t mism16 = (uint16_t)std::min<size_t>(std::min(ham, total), 65535);
  const uint16_t id = pf_identity_x10000(total, ham);
  out->has_metrics = 1;
  out->len = len16;
  out->mism = mism16;
  out->matches = len16 > mism16 ? len16 - mism16 : 0;
  out->identity_x10000 = id;
  out->score = score;
  out->read_start = (uint32_t)urs;
  out->ref_start = (uint32_t)ufs;
  auto fallback = [&](int reason) {
    out->result = 2;
    out->reason = reason;
    return 0;
  };
  if (total < read_len / 2) {
    out->result = 1;
    out->reason = 5;
    return 0;
  }
  if (!cfg.accept_enable) return fallback(1);
  if (cfg.multi_alignments_enabled) return fallback(4);
  if (cfg.accept_only_top1 && !is_top1) return fallback(3);
  if (read_len > cfg.long_read_threshold) return fallback(2);
  if (cfg.accept_require_score_margin > 0 && score_margin < cfg.accept_require_score_margin) {
    out->result = 2;
    out->reason = 9;
    out->other = 7;
    return 0;
  }
  if (c.ref_end - c.ref_start != c.read_end - c.read_start) return fallback(8);
  const size_t hard_max = (read_len * 5 + 149) / 150;
  if (ham > std::min<size_t>(cfg.accept_max_mismatches, hard_max)) return fallback(6);
  const int32_t floor = cfg.min_id_override >= 0 ? cfg.min_id_override : cfg.identity_floor;
  if ((int32_t)id < floor) return fallback(7);
  if (total < pf_min_len_required(read_len, id, ham, cfg.accept_span_slack)) return fallback(5);
  // build_ungapped_alignment (prefilter.rs:455-517): [S] M [S], MdBuilder::columns.
  out->result = 0;
  out->reason = 0;
  const size_t span = len16, rs = (size_t)urs, re = rs + span;
  if (rs > 0) out->cigar[out->n_cigar++] = ((uint32_t)rs << 4) | 4u;
  out->cigar[out->n_cigar++] = ((uint32_t)span << 4) | 0u;
  if (re < read_len) out->cigar[out->n_cigar++] = ((uint32_t)(read_len - re) << 4) | 4u;
  const uint32_t op = ((uint32_t)span << 4) | 0u;
  uint32_t nm = 0;
  const uint32_t mdlen =
      orc_nm_md(read, read_len, ref, ref_len, rs, (size_t)ufs, &op, 1, &nm, nullptr, 0);
  if (md && mdlen <= md_cap)
    orc_nm_md(read, read_len, ref, ref_len, rs, (size_t)ufs, &op, 1, &nm, md, (uint32_t)md_cap);
  out->nm = nm;
  return (int)mdlen;
}

extern "C" int orc_prefilter_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                                   const uint32_t* read_len, const uint8_t* wins,
                                   const uint64_t* win_off, const uint32_t* win_len,
                                   const orc_chain* chains, const uint8_t* is_top1,
                                   const int32_t* score_margin, const orc_prefilter_cfg* cfg,
                                   int exact_first, int nthreads, orc_prefilter_out* out,
                                   char* md, uint32_t md_stride) {
  std::atomic<uint32_t> next{0};
  std::atomic<int> bad{0};
  auto work = [&]() {
    for (;;) {
      const uint32_t i = next.fetch_add(64);
      if (i >= n) return;
      for (uint32_t p = i; p < std::min(n, i + 64); ++p) {
        const uint8_t* rd = reads + read_off[p];
        const uint8_t* wn = wins + win_off[p];
        char* m = md ? md + (size_t)p * md_stride : nullptr;
        if (exact_first && orc_exact_match_exists(rd, read_len[p], wn, win_len[p], chains + p)) {
          out[p] = orc_prefilter_out{};
          out[p].result = 3;
          out[p].nm = orc_identical_nm(rd, read_len[p]);
          out[p].n_cigar = 1;
          out[p].cigar[0] = read_len[p] << 4;
          if (m) snprintf(m, md_stride, "%u", read_len[p]);
          continue;
        }
        if (orc_prefilter(rd, read_len[p], wn, win_len[p], chains + p,
                          is_top1 ? is_top1[p] : 1, score_margin ? score_margin[p] : INT32_MAX,
                          cfg, out + p, m, m ? md_stride : 0) < 0)
          bad = 1;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < std::max(nthreads, 1); ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
  return bad ? -1 : 0;
}
