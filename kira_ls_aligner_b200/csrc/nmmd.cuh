// nmmd.cuh -- NM and MD:Z of each alignment, replayed from its CIGAR
// (nm_md_from_cigar, src/alignment/md.rs:162-205, with the MdBuilder rules of
// md.rs:24-146), one thread per pair.
//
// SAM rules as the reference states them: a matching column extends the
// current run; a mismatching column writes the run count and the reference
// letter; a deletion writes the count, '^' and the deleted reference letters
// and starts a new run; an insertion only adds to NM; a reference skip is
// invisible; the string always ends with a count. A column matches when the
// read byte is '=' or equals the reference byte ignoring ASCII case; a matching
// read byte outside ACGT/acgt/'=' still counts one edit. Reference letters are
// ASCII letters upper-cased, any other byte 'N'. Positions past the end of the
// read or window read as 'N'; deleted bases past the window end count toward NM.
//
// Pass 1 (out == nullptr) returns the MD length; pass 2 writes the MD bytes.
#pragma once

#include "common.cuh"

namespace kira {

__device__ __forceinline__ uint32_t nmmd_lower(uint32_t c) {
  return (c >= 'A' && c <= 'Z') ? c + 32u : c;
}

__device__ __forceinline__ char nmmd_letter(uint32_t b) {
  const bool alpha = (b >= 'A' && b <= 'Z') || (b >= 'a' && b <= 'z');
  return alpha ? (char)(b & 0xDFu) : 'N';
}

__device__ __forceinline__ uint32_t nmmd_digits(uint32_t v) {
  uint32_t d = 1;
  while (v >= 10u) {
    v /= 10u;
    ++d;
  }
  return d;
}

// Appends the decimal digits of v at out[len] (when out is set); returns the new length.
__device__ __forceinline__ uint32_t nmmd_put_count(char* out, uint32_t len, uint32_t v) {
  const uint32_t d = nmmd_digits(v);
  if (out) {
    for (uint32_t i = 0; i < d; ++i) {
      out[len + d - 1 - i] = (char)('0' + v % 10u);
      v /= 10u;
    }
  }
  return len + d;
}

__device__ __forceinline__ uint32_t nmmd_walk(const uint8_t* __restrict__ read, uint32_t read_len,
                                              const uint8_t* __restrict__ ref, uint32_t ref_len,
                                              uint32_t q, uint32_t r,
                                              const uint32_t* __restrict__ cig, uint32_t ncig,
                                              uint32_t& nm_out, char* __restrict__ out) {
  uint32_t len = 0, run = 0, nm = 0;
  for (uint32_t k = 0; k < ncig; ++k) {
    const uint32_t w = __ldg(cig + k), n = w >> 4, op = w & 15u;
    if (op == 0u) {  // M
      for (uint32_t t = 0; t < n; ++t, ++q, ++r) {
        const uint32_t qb = q < read_len ? ldb(read, q) : 'N';
        const uint32_t rb = r < ref_len ? ldb(ref, r) : 'N';
        if (qb == '=' || nmmd_lower(qb) == nmmd_lower(rb)) {
          ++run;
          const uint32_t u = (qb >= 'a' && qb <= 'z') ? qb - 32u : qb;
          nm += (u == 'A' || u == 'C' || u == 'G' || u == 'T' || u == '=') ? 0u : 1u;
        } else {
          len = nmmd_put_count(out, len, run);
          run = 0;
          if (out) out[len] = nmmd_letter(rb);
          ++len;
          ++nm;
        }
      }
    } else if (op == 1u) {  // I
      nm += n;
      q += n;
    } else if (op == 2u) {  // D
      const uint32_t end = min(r + n, ref_len), start = min(r, end);
      if (end > start) {
        len = nmmd_put_count(out, len, run);
        run = 0;
        if (out) out[len] = '^';
        ++len;
        for (uint32_t t = start; t < end; ++t, ++len)
          if (out) out[len] = nmmd_letter(ldb(ref, t));
      }
      nm += n;
      r += n;
    } else if (op == 3u) {  // N
      r += n;
    } else {  // S
      q += n;
    }
  }
  len = nmmd_put_count(out, len, run);
  nm_out = nm;
  return len;
}

}  // namespace kira
