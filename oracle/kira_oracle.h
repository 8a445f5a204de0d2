/*
 * kira_oracle.h -- CPU restatement of kira-ls-aligner's candidate-verification
 * hot path, used ONLY as test infrastructure: the parity checker for the CUDA
 * library and the timed CPU baseline of bench.py. Nothing in the product links
 * or calls this library.
 *
 * Every function restates a reference function (file:line in the
 * kira-ls-aligner v0.8.3 source tree) and reproduces its integer semantics,
 * tie-breaking and sentinel values exactly.
 *
 * CIGAR ops are packed BAM-style: (len << 4) | op, op 0=M 1=I 2=D 3=N 4=S.
 */
#ifndef KIRA_ORACLE_H
#define KIRA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* AlignmentConfig (src/alignment/mod.rs:26-35). */
typedef struct orc_cfg {
  int32_t match_score;
  int32_t mismatch;
  int32_t gap_open;
  int32_t gap_extend;
  int32_t bandwidth;
  int32_t xdrop;
  int32_t clip_penalty;
} orc_cfg;

/* SwResult (src/alignment/mod.rs:1190-1198) plus executed-cell count. */
typedef struct orc_sw_result {
  uint32_t ref_start;
  uint32_t ref_end;
  int32_t read_start;
  int32_t read_end;
  int32_t score;
  uint32_t n_cigar;     /* ops in the CIGAR (written up to the caller's cap) */
  uint32_t early_abort; /* 0/1 */
  uint32_t pad;
  uint64_t cells;       /* sum of executed row lengths (band cells) */
} orc_sw_result;

/* ---- bitpacked.rs ---- */
int orc_pack(const uint8_t* seq, size_t n, uint8_t* bits);
void orc_shift_bits_right(const uint8_t* bits, size_t nbytes, int bit_offset, uint8_t* out);
void orc_pre_shift(const uint8_t* bits, size_t nbytes, uint8_t* out4);
size_t orc_mismatch_count(const uint8_t* read, const uint8_t* ref, size_t n_bytes, size_t n_nucs);
int orc_scan_best_with_second_raw(const uint8_t* read_bits, size_t read_bytes, size_t read_len,
                                  int read_valid, const uint8_t* ref_pre4, size_t ref_bytes,
                                  size_t ref_len, int64_t* shift, int64_t* mism, int64_t* second);
int orc_scan(const uint8_t* read_bits, size_t read_bytes, size_t read_len, int read_valid,
             const uint8_t* ref_pre4, size_t ref_bytes, size_t ref_len, size_t max_mism,
             int64_t* shift, int64_t* mism);
/* spectral_scan_kernel result semantics (src/cuda/spectral.cu:136-213) with the
 * host-side limit of backend.rs:185-188; sentinels -1 / INT32_MAX. */
void orc_gpu_sieve_semantics(const uint8_t* read_bits, uint32_t read_nucs, const uint8_t* ref_bits,
                             uint32_t ref_nucs, uint32_t max_mismatches, int32_t* shift,
                             int32_t* mism, int32_t* second);

/* ---- spectral.rs (byte-resolution sieve) ---- */
int orc_byte_scan(const uint8_t* read, size_t r, const uint8_t* win, size_t w, size_t max_mism,
                  int64_t* shift, int64_t* mism);

/* ---- myers.rs; path 0 = dispatch as bounded_edit_distance, 1 = fixed, 2 = heap ---- */
int orc_myers(const uint8_t* pat, size_t m, const uint8_t* text, size_t n, size_t max_k, int path,
              uint64_t* dist, uint64_t* end);

/* ---- mod.rs banded_sw_with (scalar, banded, adaptive/fixed) ---- */
int orc_banded_sw(const uint8_t* read, size_t q, const uint8_t* ref, size_t r, int32_t offset,
                  const orc_cfg* cfg, int32_t abort_score, int adaptive, int32_t max_drift,
                  int32_t dp_xdrop, orc_sw_result* out, uint32_t* cigar, uint32_t cigar_cap);
/* The same with the DP matrix (H and trace byte per cell, rows of row_len[i] cells
 * from column row_start[i], stride row_cap); -1 when a row exceeds row_cap. Test
 * infrastructure for traceback forms. */
int orc_banded_sw_matrix(const uint8_t* read, size_t q, const uint8_t* ref, size_t r,
                         int32_t offset, const orc_cfg* cfg, int32_t abort_score, int adaptive,
                         int32_t max_drift, int32_t dp_xdrop, orc_sw_result* out, uint32_t* cigar,
                         uint32_t cap, int32_t* row_start, int32_t* row_len, int32_t* h,
                         uint8_t* tr, size_t row_cap);

/* ---- mod.rs sw_batch_avx2 (16-lane i16, full window). n <= 16, equal shapes.
 * Returns 1 when the AVX2 kernel ran, 0 when the i16 fit check sent the chunk to
 * the scalar banded fallback (mod.rs:1854-1868), -1 on bad arguments. ---- */
int orc_sw_batch_avx2(int n, const uint8_t* const* reads, const uint8_t* const* wins, size_t q,
                      size_t r, const int32_t* abort_scores, const int32_t* scalar_offsets,
                      const orc_cfg* cfg, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                      orc_sw_result* out, uint32_t* cigar, uint32_t cap_per_lane);
/* Portable scalar model of the same kernel (saturating i16 lanes), lane group
 * size 16 (AVX2) or 32 (i8). Used to pin the CUDA full-window mode. */
int orc_sw_full_window_model(int n, const uint8_t* const* reads, const uint8_t* const* wins,
                             size_t q, size_t r, const int32_t* abort_scores, const orc_cfg* cfg,
                             int bits, orc_sw_result* out, uint32_t* cigar, uint32_t cap_per_lane);
/* ---- sw_int8_vnni.rs ---- */
int orc_int8_path_viable(size_t read_len, const orc_cfg* cfg);
int orc_sw_batch_int8(int n, const uint8_t* const* reads, const uint8_t* const* wins, size_t q,
                      size_t r, const int32_t* abort_scores, const int32_t* scalar_offsets,
                      const orc_cfg* cfg, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                      orc_sw_result* out, uint32_t* cigar, uint32_t cap_per_lane);
int orc_cpu_has_avx2(void);
int orc_cpu_has_avx_vnni(void);

/* ---- align_batch_simd dispatch (mod.rs:1111-1169). mode/detected: 0 Scalar,
 * 1 Avx2, 2 AvxVnni, 3 Neon. scalar_offsets = BatchInput::scalar_sw offset. ---- */
int orc_align_batch_simd(int n, const uint8_t* const* reads, const uint32_t* read_lens,
                         const uint8_t* const* wins, const uint32_t* win_lens,
                         const int32_t* abort_scores, const int32_t* scalar_offsets,
                         const orc_cfg* cfg, int mode, int detected, int adaptive,
                         int32_t max_drift, int32_t dp_xdrop, orc_sw_result* out, uint32_t* cigar,
                         uint32_t cap_per_lane);

/* ---- certificate + router (mod.rs:688-776, router.rs:191-203) ---- */
int orc_spectral_certified(const uint8_t* read, const uint8_t* ref_aligned, size_t len,
                           size_t mism, int64_t second, size_t max_mism, int strict);
size_t orc_spectral_max_mismatches(size_t read_len);
size_t orc_myers_reject_bound(size_t read_len);

/* ---- composed verification of one (read x window) pair ---- */
typedef struct orc_verify_params {
  orc_cfg cfg;
  int32_t sieve_threshold; /* certificate mismatch bound; <0 -> router default */
  int32_t myers_k;         /* <0 -> router::myers_reject_bound(read_len) */
  int32_t abort_score;     /* i32::MIN/8 disables */
  int32_t adaptive;
  int32_t max_drift;
  int32_t dp_xdrop;
  int32_t cert_strict;
} orc_verify_params;

/* status: 1 certified ungapped, 2 rejected by Myers, 3 banded SW */
typedef struct orc_verify_result {
  int32_t status;
  int32_t sieve_shift; /* -1 when the packed scan returned None */
  int32_t sieve_mism;
  int32_t sieve_second; /* INT32_MAX when None */
  int32_t myers_dist;   /* -1 when rejected / not run */
  int32_t myers_end;
  orc_sw_result sw;
} orc_verify_result;

int orc_verify_pair(const uint8_t* read, size_t q, const uint8_t* win, size_t w,
                    const orc_verify_params* p, orc_verify_result* out, uint32_t* cigar,
                    uint32_t cigar_cap);

/* Threaded batch drivers (the CPU baseline; dynamic scheduling over pairs). */
int orc_verify_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                     const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                     const uint32_t* win_len, const orc_verify_params* p, int nthreads,
                     orc_verify_result* out, uint32_t* cigar, uint32_t cap_per_pair);
int orc_banded_sw_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                        const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                        const uint32_t* win_len, const int32_t* offsets, const orc_cfg* cfg,
                        int32_t abort_score, int adaptive, int32_t max_drift, int32_t dp_xdrop,
                        int nthreads, orc_sw_result* out, uint32_t* cigar, uint32_t cap_per_pair);
/* AVX2 i16 path over pairs of one shape: chunks of 16 consecutive pairs. */
int orc_sw_avx2_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off, uint32_t q,
                      const uint8_t* wins, const uint64_t* win_off, uint32_t r,
                      const orc_cfg* cfg, int nthreads, orc_sw_result* out, uint32_t* cigar,
                      uint32_t cap_per_pair);
int orc_myers_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                    const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                    const uint32_t* win_len, uint32_t max_k, int nthreads, int64_t* dist,
                    int64_t* end);
int orc_sieve_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                    const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                    const uint32_t* win_len, int nthreads, int32_t* shift, int32_t* mism,
                    int32_t* second);

/* NM and MD:Z of one alignment: nm_md_from_cigar (src/alignment/md.rs:162-205)
 * with the MdBuilder rules (md.rs:24-146). cigar words are len << 4 | op with
 * op 0 M, 1 I, 2 D, 3 N, 4 S. Writes at most md_cap bytes of MD (no NUL) and
 * returns the full MD length. */
uint32_t orc_nm_md(const uint8_t* read, size_t read_len, const uint8_t* ref, size_t ref_len,
                   size_t read_start, size_t ref_start, const uint32_t* cigar, uint32_t n_cigar,
                   uint32_t* nm, char* md, uint32_t md_cap);
/* MdBuilder driven directly (the md_format.rs cases): ops 'M' matched, 'X'
 * mismatch(ref[i]), 'C' column(read[i], ref[i]), 'I' insertion(len), 'D'
 * deletion(ref bytes of length len). */
uint32_t orc_md_builder(const char* script, const uint8_t* read, const uint8_t* ref,
                        const uint32_t* lens, uint32_t n, uint32_t* nm, char* md, uint32_t md_cap);
/* Threaded batch: NM/MD of each pair's alignment (window coordinates). */
int orc_nm_md_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                    const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                    const uint32_t* win_len, const int32_t* read_start, const uint32_t* ref_start,
                    const uint32_t* cig_off, const uint32_t* n_cig, const uint32_t* ops,
                    int nthreads, uint32_t* nm, uint32_t* md_len, char* md, uint32_t md_stride);

/* Wavefront alignment (src/alignment/wfa.rs): affine-gap, the whole pattern
 * against a text prefix (ends-free leading text up to text_begin_free, free
 * trailing text). Costs: plain (WfaPenalties: ins = del = gap_extend) or scored
 * (WfaCosts::scored, wfa.rs:41-52: mismatch = a + b, ins_extend = a + e,
 * del_extend = e). adaptive_drop < 0: exact. Returns 1 with the cost (score),
 * text span and CIGAR (len << 4 | op, 5'->3') when an alignment of cost <=
 * max_score exists, else 0. traceback = 0 leaves the CIGAR empty (wfa_score_only). */
typedef struct orc_wfa_cfg {
  int32_t mismatch, gap_open, gap_extend, match_score, scored;
  int32_t max_score, adaptive_drop, text_begin_free, traceback;
} orc_wfa_cfg;
int orc_wfa(const uint8_t* pattern, size_t m, const uint8_t* text, size_t n, const orc_wfa_cfg* c,
            int32_t* score, uint32_t* text_start, uint32_t* text_end, uint32_t* cigar,
            uint32_t cap, uint32_t* n_cigar);
int orc_wfa_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                  const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                  const uint32_t* win_len, const orc_wfa_cfg* c, int nthreads, int32_t* found,
                  int32_t* score, uint32_t* text_start, uint32_t* text_end, uint32_t* n_cigar,
                  uint32_t* cigar, uint32_t cap_per_pair);

/* Ungapped extension prefilter (src/alignment/prefilter.rs:93-453) and the
 * exact-match fast path (src/alignment/mod.rs:779-832) for one chain. */
typedef struct orc_chain {
  uint32_t ref_start, ref_end, read_start, read_end;
} orc_chain;
typedef struct orc_prefilter_cfg {
  int32_t match_score, mismatch, xdrop;
  int32_t accept_enable, accept_only_top1;
  uint32_t accept_span_slack;
  int32_t identity_floor;        /* (accept_min_identity * 100).round() as u16 */
  uint32_t accept_max_mismatches;
  int32_t accept_require_score_margin;
  uint32_t long_read_threshold;
  int32_t multi_alignments_enabled;
  int32_t tail;                  /* KIRA_UNGAP_TAIL (default 1) */
  int32_t min_id_override;       /* KIRA_UNGAP_MINID, < 0: unset */
} orc_prefilter_cfg;
typedef struct orc_prefilter_out {
  int32_t result;  /* 0 Accept, 1 Reject, 2 Fallback */
  int32_t reason;  /* PrefilterReason::idx() */
  int32_t other;   /* Other(..): 1 read_len0 2 non_monotonic 3 anchor0 4 span0 5 neg_start 6 span_oob 7 margin_fail */
  int32_t has_metrics;
  uint32_t len, mism, matches, identity_x10000;
  int32_t score;
  uint32_t read_start, ref_start;
  uint32_t nm, n_cigar, cigar[3];  /* Accept: build_ungapped_alignment */
} orc_prefilter_out;
/* Returns the MD length (Accept), written to md when md_cap allows; -1 when the
 * chain lies outside the read or reference (the reference panics there). */
int orc_prefilter(const uint8_t* read, size_t read_len, const uint8_t* ref, size_t ref_len,
                  const orc_chain* chain, int is_top1, int32_t score_margin,
                  const orc_prefilter_cfg* cfg, orc_prefilter_out* out, char* md, size_t md_cap);
int orc_exact_match_exists(const uint8_t* read, size_t read_len, const uint8_t* ref,
                           size_t ref_len, const orc_chain* chain);
uint32_t orc_identical_nm(const uint8_t* bases, size_t len);
/* Stage-4 order over a batch on host threads: exact_match_exists first when
 * exact_first (result 3), else orc_prefilter; md_stride bytes of MD per chain. */
int orc_prefilter_batch(uint32_t n, const uint8_t* reads, const uint64_t* read_off,
                        const uint32_t* read_len, const uint8_t* wins, const uint64_t* win_off,
                        const uint32_t* win_len, const orc_chain* chains, const uint8_t* is_top1,
                        const int32_t* score_margin, const orc_prefilter_cfg* cfg,
                        int exact_first, int nthreads, orc_prefilter_out* out, char* md,
                        uint32_t md_stride);

#ifdef __cplusplus
}
#endif
#endif
