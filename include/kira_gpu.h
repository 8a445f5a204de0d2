/*
 * kira_gpu.h -- C ABI of the B200 (sm_100a) candidate-verification library.
 *
 * Replaces the GPU backend and the CPU DP kernels of kira-ls-aligner's
 * verification/extension hot path:
 *   - the 2-bit multi-shift Hamming sieve   (src/alignment/bitpacked.rs,
 *                                            src/cuda/spectral.cu, src/cuda/backend.rs)
 *   - Myers bounded edit distance            (src/alignment/myers.rs)
 *   - banded affine Smith-Waterman + CIGAR   (src/alignment/mod.rs:1331-1771)
 *   - full-window batch SW (align_batch_simd) (src/alignment/mod.rs:1111-1169,1846-2135,
 *                                            src/alignment/sw_int8_vnni.rs)
 * and the steps on either side of it:
 *   - wavefront alignment (WFA)              (src/alignment/wfa.rs)
 *   - exact matches + ungapped prefilter     (src/alignment/mod.rs:779-832,
 *                                            src/alignment/prefilter.rs)
 *   - NM / MD:Z from the CIGARs              (src/alignment/md.rs)
 *
 * Conventions
 *   - Every entry point returns an int status (kira_status). 0 is success.
 *   - Host buffers passed to the non-"_dev" entry points are borrowed for the
 *     duration of the call; results are written into caller-owned buffers.
 *   - The library owns all device memory it allocates (grow-only arena per ctx).
 *   - One kira_ctx per host thread; a ctx is not thread-safe (like CudaBackend,
 *     which is pinned to its thread: src/cuda/backend.rs:264-269).
 *   - Sequences are ASCII bytes exactly as the Rust API receives them; byte
 *     equality (SW), case-insensitive ACGT (Myers) and the 2-bit code with the
 *     valid flag (sieve) follow the reference functions bit for bit.
 *   - CIGAR ops are packed BAM-style: (len << 4) | op, op 0=M 1=I 2=D 3=N 4=S.
 */
#ifndef KIRA_GPU_H
#define KIRA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KIRA_GPU_ABI_VERSION 1

/* Status codes; the first five map onto CudaError (src/cuda/mod.rs:18-34). */
enum kira_status {
  KIRA_OK = 0,
  KIRA_ERR_NOT_BUILT = 1,     /* CudaError::NotBuilt */
  KIRA_ERR_DRIVER = 2,        /* CudaError::Driver */
  KIRA_ERR_RUNTIME = 3,       /* CudaError::Runtime */
  KIRA_ERR_NO_DEVICE = 4,     /* CudaError::NoDevice */
  KIRA_ERR_READ_TOO_LONG = 5, /* CudaError::ReadTooLong */
  KIRA_ERR_TIMEOUT = 6,       /* a bounded wait expired */
  KIRA_ERR_INVALID = 7,       /* argument outside the supported domain */
  KIRA_ERR_OOM = 8,           /* device memory exhausted / admission refused */
  KIRA_ERR_CAPACITY = 9,      /* caller's output buffer too small (see *_used) */
  KIRA_ERR_SCRATCH_LIMIT = 10, /* batch needs more than the fixed no-alloc scratch */
  KIRA_PENDING = 11            /* server request still queued or running (not an error) */
};

/* Per-pair status of the composed verification. */
enum kira_pair_status {
  KIRA_PAIR_PENDING = 0,
  KIRA_PAIR_CERTIFIED = 1,    /* ungapped hit accepted by the certificate */
  KIRA_PAIR_MYERS_REJECT = 2, /* bounded edit distance above k */
  KIRA_PAIR_SW = 3,           /* banded SW alignment */
  KIRA_PAIR_OUT_OF_BOUNDS = 4 /* banded SW: the pair exceeds the call's declared maxima
                                 (read_len > max_read_len, or a band wider than the
                                 launch shape); not aligned, n_cigar 0 */
};

/* Maximum packed read length of the sieve drop-in (src/cuda/mod.rs:35-37). */
#define KIRA_READ_BYTES_MAX 64

typedef struct kira_ctx kira_ctx;

/* ---------------------------------------------------------------- context */

/* cuda::is_available (src/cuda/mod.rs:39-49). 1 when a CUDA device is usable. */
int kira_gpu_is_available(void);

/* CudaBackend::new (src/cuda/backend.rs:61-93): bind `device`, create the
 * ctx's stream and arena. */
int kira_gpu_init(int device, kira_ctx** out);

/* CudaBackend drop / release_buffers (src/cuda/backend.rs:251-261). */
void kira_gpu_destroy(kira_ctx* ctx);

/* Text of the last error on this ctx (the String inside CudaError). Returns the
 * full length; writes at most len-1 bytes plus a NUL. */
int kira_gpu_last_error(const kira_ctx* ctx, char* buf, size_t len);

/* Bytes of device memory the ctx arena currently holds. */
uint64_t kira_gpu_arena_bytes(const kira_ctx* ctx);

/* No counterpart in the reference (launch accounting for benchmarks): the number
 * of kernels this library has launched in this process, over all contexts and
 * threads; a CUDA-graph replay adds the kernels of the replayed graph. */
uint64_t kira_gpu_launch_count(void);

/* No counterpart in the reference (the denominator of the integer roofline of
 * the DP kernels): measures this GPU's integer instruction rate. Every thread of
 * a full grid runs `rounds` rounds of 16 independent instructions -- op 0 the
 * DPX add-max on packed int16 pairs, op 1 a three-input add, op 2 a three-input
 * logic op, op 3 an integer multiply-add, op 4 logic op and multiply-add
 * alternating, op 5 DPX add-max and multiply-add alternating -- and
 * *thread_ops_per_s receives the thread-instructions per second (CUDA events
 * around one launch after a warm-up launch). */
int kira_gpu_alu_probe(int device, int op, uint32_t rounds, double* thread_ops_per_s);

/* ------------------------------------------------------- sieve (drop-in) */

/* CudaJob (src/cuda/backend.rs:13-26). Only phase 0 of ref_shifted is read:
 * the kernel derives the other three bit phases in registers, so the 4x
 * pre-shifted host copies (bitpacked.rs:95-119) are not needed. */
typedef struct kira_sieve_job {
  const uint8_t* read_packed; /* 2-bit packed, (read_nucs + 3) / 4 bytes */
  uint32_t read_bytes;        /* length of read_packed */
  uint32_t read_nucs;
  const uint8_t* ref_packed;  /* ref_shifted[0] */
  uint32_t ref_bytes;         /* length of ref_packed, >= (ref_nucs + 3) / 4 */
  uint32_t ref_nucs;
  uint32_t max_mismatches;
} kira_sieve_job;

/* CudaResult (src/cuda/backend.rs:28-35): shift -1 / mismatches INT32_MAX when
 * the best hit is above min(max_mismatches, read_nucs); second_mismatches is
 * INT32_MAX for None. */
typedef struct kira_sieve_result {
  int32_t shift;
  int32_t mismatches;
  int32_t second_mismatches;
} kira_sieve_result;

/* CudaBackend::run_batch (src/cuda/backend.rs:95-249). Returns
 * KIRA_ERR_READ_TOO_LONG when a read exceeds KIRA_READ_BYTES_MAX packed bytes. */
int kira_gpu_sieve_batch(kira_ctx* ctx, const kira_sieve_job* jobs, uint32_t n,
                         kira_sieve_result* out);

/* ------------------------------------------------ pairs and configuration */

/* A batch of (read x window) pairs. Reads and windows are ASCII arenas; pair p
 * uses read_seq[read_off[p] .. +read_len[p]] and win_seq[win_off[p] .. +win_len[p]].
 * Pairs may share a read (candidate windows of one read). win_seq == NULL selects
 * the device-resident reference (kira_gpu_ref_upload); win_off is then a
 * reference coordinate. Optional per-pair arrays may be NULL. */
typedef struct kira_pairs {
  uint32_t n;
  uint32_t max_read_len;      /* upper bound of read_len[]; 0 -> computed (host API only) */
  uint32_t max_win_len;       /* upper bound of win_len[];  0 -> computed (host API only) */
  uint32_t max_bandwidth;     /* upper bound of bandwidth[]; 0 -> computed (host API only) */
  const uint8_t* read_seq;
  uint64_t read_seq_bytes;
  const uint64_t* read_off;
  const uint32_t* read_len;
  const uint8_t* win_seq;
  uint64_t win_seq_bytes;
  const uint64_t* win_off;
  const uint32_t* win_len;
  const int32_t* band_offset; /* banded_sw `offset` (mod.rs:1331-1337); NULL -> 0 */
  const int32_t* abort_score; /* NULL -> disabled (i32::MIN / 8) */
  const int32_t* bandwidth;   /* per-pair half-width; NULL -> cfg.bandwidth */
} kira_pairs;

/* AlignmentConfig (src/alignment/mod.rs:24-35) plus the hot-path knobs that the
 * reference reads from the environment once (mod.rs:1256-1329). */
typedef struct kira_sw_cfg {
  int32_t match_score;
  int32_t mismatch;
  int32_t gap_open;
  int32_t gap_extend;
  int32_t bandwidth;    /* half-width; rows cover centre +- bandwidth */
  int32_t xdrop;
  int32_t clip_penalty;
  int32_t adaptive;     /* KIRA_ADAPTIVE_BAND, default 1 */
  int32_t max_drift;    /* KIRA_ADAPTIVE_MAX_DRIFT, default 16 */
  int32_t dp_xdrop;     /* KIRA_DP_XDROP; < 0 -> use xdrop */
} kira_sw_cfg;

/* SwPublicResult (src/alignment/mod.rs:910-920) in window coordinates; the
 * CIGAR is ops[cigar_off .. cigar_off + n_cigar) of the call's CIGAR buffer. */
typedef struct kira_sw_result {
  int32_t score;
  uint32_t ref_start;
  uint32_t ref_end;
  int32_t read_start;
  int32_t read_end;
  uint32_t cigar_off;
  uint32_t n_cigar;
  uint8_t status;      /* kira_pair_status (verify) or KIRA_PAIR_SW */
  uint8_t early_abort;
  uint16_t reserved;   /* banded SW: 1 when the pair's CIGAR overflowed its device slot
                          (the row is then incomplete; the host entry points return an
                          error for the call) */
} kira_sw_result;

/* Caller-owned CIGAR output: ops[cap]; *used receives the number of ops the
 * call produced. KIRA_ERR_CAPACITY when used > cap (nothing past cap written). */
typedef struct kira_cigar_buf {
  uint32_t* ops;
  uint64_t cap;
  uint64_t used;
} kira_cigar_buf;

/* Opt-in stage timing (CUDA events on the work stream). After a verification
 * call has completed, kira_gpu_stage_times fills ms[] with the durations of:
 * 0 sieve + certificate, 1 Myers, 2 banded-SW DP, 3 traceback, 4 CIGAR
 * compaction, and returns how many were filled. */
int kira_gpu_profile(kira_ctx* ctx, int enable);
int kira_gpu_stage_times(kira_ctx* ctx, float* ms, int max_stages);

/* Launch shapes of the banded-SW stage (lanes per pair x cells per lane; packed =
 * int16 score lanes, two cells per 32-bit register, used only when the batch's
 * scores provably fit). kira_gpu_bsw_shapes lists them (returns the count; any
 * output array may be null); kira_gpu_set_bsw_shape installs a shape for every
 * band in band's class (<=16, 33, 64, 128, 256, 511; -1 restores the default
 * pick). The autotuner (Python runtime) times the shapes that cover a band on a
 * sample and installs the fastest. */
int kira_gpu_bsw_shapes(int* lanes, int* cells, int* packed, int max_shapes);
int kira_gpu_set_bsw_shape(kira_ctx* ctx, uint32_t band, int shape);

/* kira_gpu_bsw_batch buckets pairs by band class (one tuned launch shape and trace
 * geometry per class, longest reads first, dynamic work fetching). plain = 1
 * selects the one-launch form instead: the kernel the bucketed path would pick
 * for the batch's widest band (packed int16 when the batch's scores fit, else
 * int32), one launch over every pair in input order, no graph replay -- the
 * baseline the bucketed form is measured against. Results are identical either
 * way. */
int kira_gpu_set_plain(kira_ctx* ctx, int plain);

/* Device bytes the banded-SW trace arena (trace slots + row metadata) may hold at
 * once; 0 (default) = half of the free device memory plus what the arena holds,
 * clamped to [64 MiB, 64 GiB]. Batches needing more run their DP sweep and
 * traceback in rounds over the same arena; results are identical. */
int kira_gpu_set_trace_budget(kira_ctx* ctx, uint64_t bytes);

/* No counterpart in the reference: the number of trace rounds (DP + traceback
 * passes over the reused trace arena, summed over band classes) that the last
 * kira_gpu_bsw_batch call on this ctx ran. */
uint32_t kira_gpu_bsw_rounds(const kira_ctx* ctx);

/* CUDA-graph replay of the bucketed banded-SW launches (per-class DP sweeps,
 * tracebacks, CIGAR scan and compaction) of kira_gpu_bsw_batch: a call whose
 * launch parameters (device buffers, per-class counts, shapes, rounds) equal the
 * previous graph's replays it, any other call captures a new one. enable: 1 on,
 * 0 off, -1 unchanged; captures / replays (optional) receive the counts so far.
 * Results are identical with and without graphs. */
int kira_gpu_set_graphs(kira_ctx* ctx, int enable, uint64_t* captures, uint64_t* replays);

/* Host batches of at least 2 chunks run chunk by chunk through separate copy-in,
 * compute and copy-out streams, so uploads, kernels and downloads of consecutive
 * chunks overlap (pinned host buffers make the copies asynchronous); this applies
 * to kira_gpu_verify_batch, kira_gpu_wfa_batch and kira_gpu_prefilter_batch.
 * pairs < 0: automatic (the default: a quarter of the batch, at least 2^18
 * pairs; verification batches of at least 2^20 pairs in chunks of 1/8, 1/4, 1/4,
 * 1/4 and 1/8), 0: off, else the chunk size. Results are identical either way. */
int kira_gpu_set_chunk_pairs(kira_ctx* ctx, int64_t pairs);

/* Upload the reference as ASCII bases (Index::ref_bases, src/index/mod.rs:1098);
 * it stays resident until the next upload or kira_gpu_destroy. */
int kira_gpu_ref_upload(kira_ctx* ctx, const uint8_t* seq, uint64_t len);

/* ------------------------------------------------------------ Myers */

/* myers::bounded_edit_distance (src/alignment/myers.rs:47-70) per pair:
 * dist[p] = -1 for None. Patterns up to 2048 bases. */
int kira_gpu_myers_batch(kira_ctx* ctx, const kira_pairs* pairs, uint32_t max_k, int32_t* dist,
                         int32_t* end_pos);

/* ------------------------------------------------------- banded SW */

/* banded_sw_public (src/alignment/mod.rs:890-908) per pair. Requires gap_open,
 * gap_extend, mismatch >= 0, bandwidth <= 1023 and read_len * match_score < 2^21.
 * cells (optional) receives the executed band cells. */
int kira_gpu_bsw_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                       kira_sw_result* out, kira_cigar_buf* cigar, uint64_t* cells);

/* SimdMode (src/simd/mod.rs:5-12). */
enum kira_simd_mode {
  KIRA_SIMD_SCALAR = 0,
  KIRA_SIMD_AVX2 = 1,
  KIRA_SIMD_AVX_VNNI = 2,
  KIRA_SIMD_NEON = 3
};

/* align_batch_simd (src/alignment/mod.rs:1111-1169), SW results per input before
 * build_alignment. `mode` is the requested SimdMode, `detected` the host's
 * simd::detect_cached(); the GPU reproduces the kernel the reference would pick:
 *   - inputs of mixed (read, window) lengths, scalar mode, or a failed i16 fit
 *     check -> banded_sw per input with band_offset = BatchInput::scalar_sw's
 *     offset (mod.rs:60-72);
 *   - AVX2 (or AVX-VNNI without the i8 path) -> full-window i16 semantics in
 *     groups of 16 consecutive inputs (sw_batch_avx2_inner, mod.rs:1914-2135);
 *   - AVX-VNNI with int8_path_viable and <= 32 inputs -> one group of 32
 *     (sw_batch_int8, sw_int8_vnni.rs:141-370, identical values under viability).
 * The group matters only for abort bounds: a group stops after the first row at
 * which every member's bound has fired. Full-window windows up to 544 bases. */
int kira_gpu_align_batch_simd(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                              int mode, int detected, kira_sw_result* out, kira_cigar_buf* cigar);

/* ------------------------------------------- composed verification */

/* Parameters of the composed path (sieve -> certificate -> Myers -> banded SW). */
typedef struct kira_verify_params {
  kira_sw_cfg sw;
  int32_t sieve_threshold; /* certificate mismatch bound; < 0 -> spectral_max_mismatches */
  int32_t myers_k;         /* < 0 -> myers_reject_bound(read_len) */
  int32_t cert_strict;     /* KIRA_CERT_STRICT */
  int32_t flags;           /* KIRA_VERIFY_* bits */
} kira_verify_params;

/* kira_verify_params.flags: turn off the exact 4-gram prefilter in front of the
 * Myers stage. The filter only removes pairs whose edit distance provably
 * exceeds k (q-gram lemma), so results are identical either way. */
#define KIRA_VERIFY_NO_QGRAM 1

/* Optional per-stage detail. */
typedef struct kira_verify_detail {
  int32_t sieve_shift;  /* -1 when the packed scan returned None */
  int32_t sieve_mism;   /* INT32_MAX when None */
  int32_t sieve_second; /* INT32_MAX when None */
  int32_t myers_dist;   /* -1 when rejected or not run */
  int32_t myers_end;
} kira_verify_detail;

/* For every pair: packed_scan_scratch + spectral_hit_is_certified
 * (mod.rs:594-762) -> ungapped qM when certified; else bounded_edit_distance
 * (myers.rs:47) with k -> KIRA_PAIR_MYERS_REJECT on None; else banded_sw
 * (mod.rs:1331) with offset = the sieve's best shift (0 without a hit). */
int kira_gpu_verify_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_verify_params* p,
                          kira_sw_result* out, kira_cigar_buf* cigar, kira_verify_detail* detail,
                          uint64_t* cells);

/* Compact result form of kira_gpu_verify_batch, for callers that use only the
 * pairs with an alignment -- stage 4's consumer of the GPU sieve keeps the
 * accepted hits and drops the rest (src/pipeline/stage4_alignment.rs:1317-1356).
 * Same computation and the same rows; what comes back is
 *   status[i]   the kira_pair_status of pair i (one byte per pair);
 *   rows[0..k)  the full rows of the pairs whose status is KIRA_PAIR_CERTIFIED or
 *               KIRA_PAIR_SW, in pair order (row r belongs to the r-th such pair);
 *               *rows_used = k. Rows past rows_cap are not written and the call
 *               returns KIRA_ERR_CAPACITY (the status bytes are complete);
 *   cigar       as in kira_gpu_verify_batch (cigar_off of each row indexes it).
 * On the 2M-pair short-read batch this moves about 11 MB back instead of 65 MB. */
int kira_gpu_verify_batch_compact(kira_ctx* ctx, const kira_pairs* pairs,
                                  const kira_verify_params* p, uint8_t* status,
                                  kira_sw_result* rows, uint64_t rows_cap, uint64_t* rows_used,
                                  kira_cigar_buf* cigar, uint64_t* cells);

/* Device-pointer form of kira_gpu_verify_batch: every pointer in `pairs` and the
 * outputs are device pointers; work is enqueued on `stream` (a cudaStream_t) and
 * the call returns without synchronising. Arena allocations must be readable up
 * to the next 16-byte boundary past their last byte. cigar_ops receives the
 * packed CIGAR (capacity cigar_cap ops); *cigar_used_dev (device) the op count. */
int kira_gpu_verify_dev(kira_ctx* ctx, const kira_pairs* pairs, const kira_verify_params* p,
                        kira_sw_result* out, uint32_t* cigar_ops, uint64_t cigar_cap,
                        uint64_t* cigar_used_dev, kira_verify_detail* detail,
                        unsigned long long* cells_dev, void* stream);

/* ------------------------------------------- allocation-free banded SW */

/* Size of the fixed scratch array that kira_gpu_bsw_batch_noalloc uses: one
 * file-scope device array inside the library, held on every GPU that loads the
 * library until the process exits. */
#define KIRA_NOALLOC_SCRATCH_BYTES (32u << 20)

/* No counterpart in the reference: an extra entry point for callers that cannot
 * allocate device memory -- code whose device memory is owned by another
 * allocator (a serving framework's pool, a fixed arena handed down by the host
 * application) or that cannot afford the implicit device-wide synchronisation
 * of cudaMalloc / cudaFree on its path.
 *
 * Same results as kira_gpu_bsw_batch (banded_sw_public per pair), but every
 * pointer in `pairs`, `out`, `cigar_ops` and `cigar_used` is a device pointer
 * owned by the caller, no kira_ctx is needed, and the call allocates nothing:
 * no cudaMalloc, cudaFree or allocating library routine. All scratch (trace
 * arena, CIGAR slots, scan buffers, flags) lives in the library's fixed
 * KIRA_NOALLOC_SCRATCH_BYTES device array.
 *   - pairs->max_read_len and max_win_len (and max_bandwidth when a per-pair
 *     bandwidth array is given) are required and must bound every pair; the
 *     scratch a batch needs grows with n, max_read_len, max_win_len and the band.
 *     A batch that does not fit returns KIRA_ERR_SCRATCH_LIMIT before any GPU
 *     work: split it into smaller batches.
 *   - Work is enqueued on `stream` (a cudaStream_t) and the call returns without
 *     synchronising; *cigar_used (device) receives the op count, and ops beyond
 *     cigar_cap are not written (the caller compares the two after syncing; a
 *     pair whose ops would cross cigar_cap gets none).
 *   - Problems found on the device are reported per pair, since the call does
 *     not wait for the GPU: a pair that exceeds the declared maxima (read_len >
 *     max_read_len, or a per-pair band wider than max_bandwidth allows) is not
 *     aligned and its row has status KIRA_PAIR_OUT_OF_BOUNDS and n_cigar 0; a
 *     row with reserved == 1 lost part of its CIGAR (device slot overflow). Every
 *     other row has status KIRA_PAIR_SW.
 *   - The first call on a device looks up the scratch array's device address on
 *     that device (cudaGetSymbolAddress, with the device current) and caches it;
 *     make that first call before any stream capture.
 *   - Every call shares the one array and it keeps the previous call's
 *     contents. Calls that overlap on the GPU (different streams without
 *     ordering, or several host threads) race on it: order them on one stream or
 *     synchronise between them. */
int kira_gpu_bsw_batch_noalloc(const kira_pairs* pairs, const kira_sw_cfg* cfg,
                               kira_sw_result* out, uint32_t* cigar_ops, uint64_t cigar_cap,
                               uint64_t* cigar_used, void* stream);

/* ------------------------------------------------------------- NM and MD:Z
 *
 * compute_nm_md / nm_md_from_cigar (src/alignment/mod.rs:1774-1782,
 * src/alignment/md.rs:162-205) for every pair of a batch, on the device, from the
 * results and CIGAR ops that kira_gpu_verify_batch / kira_gpu_bsw_batch /
 * kira_gpu_align_batch_simd returned for the same `pairs` (window coordinates:
 * read_start / ref_start into the pair's read and window). nm[i] is the SAM NM
 * (0xFFFFFFFF for a pair without an alignment, n_cigar == 0); pair i's MD:Z text
 * is md[md_off[i] .. md_off[i + 1]) (no NUL; md_off has n + 1 entries).
 * KIRA_ERR_CAPACITY when the text exceeds md_cap (*md_used gives the need; nm and
 * md_off are filled). Stage times (kira_gpu_stage_times): [0] inputs uploaded,
 * [1] NM + MD lengths + offsets, [2] host check, [3] MD text. */
int kira_gpu_nm_md(kira_ctx* ctx, const kira_pairs* pairs, const kira_sw_result* results,
                   const uint32_t* cigar_ops, uint64_t n_ops, uint32_t* nm, uint32_t* md_off,
                   char* md, uint64_t md_cap, uint64_t* md_used);

/* ------------------------------------------------------------------- WFA
 *
 * Wavefront alignment (src/alignment/wfa.rs), the cascade step between Myers and
 * banded SW: try_fast_dp_alignment's wfa_align_scored call (src/alignment/
 * mod.rs:344-439) and the score probes ungapped_beaten_by_gap /
 * locus_alignment_score (mod.rs:162-240). The whole read (pattern) is aligned to
 * a prefix of the window (text) with affine gaps; trailing text is free and up to
 * text_begin_free leading text bases are free. */

/* WfaPenalties / AlignmentConfig plus WfaOptions (wfa.rs:9-17, 81-111). */
typedef struct kira_wfa_params {
  int32_t mismatch;        /* WfaPenalties.mismatch, or AlignmentConfig.mismatch when scored */
  int32_t gap_open;
  int32_t gap_extend;
  int32_t match_score;     /* scored only */
  int32_t scored;          /* 1: WfaCosts::scored (wfa.rs:41-52): mismatch + match per
                              mismatch, gap_extend + match per inserted base */
  int32_t max_score;       /* WfaOptions.max_score; < 0: router::wfa_score_budget of each
                              read (router.rs:160-165) */
  int32_t budget_pct;      /* KIRA_WFA_BUDGET_PCT of that budget; < 0: 25 */
  int32_t adaptive_drop;   /* WfaOptions.adaptive_drop: >= 0 Some(drop), < 0 None */
  int32_t text_begin_free; /* WfaOptions.text_begin_free */
  int32_t traceback;       /* 1: wfa_align / wfa_align_scored (CIGAR + text_start);
                              0: wfa_score_only / wfa_score_only_scored */
} kira_wfa_params;

/* WfaAlignment (wfa.rs:113-124) of one pair. found = 0 for None (no alignment of
 * cost <= max_score, or scored costs that WfaCosts::scored refuses). */
typedef struct kira_wfa_result {
  int32_t cost;        /* WfaAlignment.score: the WFA cost (the loss when scored); -1 for None */
  int32_t score;       /* scored: read_len * match_score - cost (wfa_score_only_scored); else cost */
  uint32_t text_start; /* traceback only (0 otherwise) */
  uint32_t text_end;
  uint32_t cigar_off;  /* ops[cigar_off .. + n_cigar) of the call's CIGAR buffer (M, I, D) */
  uint32_t n_cigar;
  uint32_t found;
  uint32_t reserved;
} kira_wfa_result;

/* wfa_align / wfa_score_only (and the scored forms) for every pair of the batch.
 * Per-pair max_score and text_begin_free arrays override the params when given
 * (the per-read budgets of ungapped_beaten_by_gap, the ends-free retry of
 * mod.rs:393-419). Reads and windows up to 30000 bases. Plain penalties need
 * mismatch >= 1, gap_open >= 0 and gap_extend >= 1 (KIRA_ERR_INVALID otherwise);
 * cigar may be NULL when traceback = 0. Stage times: [0] inputs uploaded,
 * [1] wavefronts and traceback, [2] CIGAR scan and compaction, [3] results
 * downloaded. */
int kira_gpu_wfa_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_wfa_params* p,
                       const int32_t* max_score, const int32_t* text_begin_free,
                       kira_wfa_result* out, kira_cigar_buf* cigar);

/* Lanes that align one WFA pair: 8, 16 or 32 (32 / lanes pairs share a warp and
 * step in lockstep); 0 (default) picks 8 for reads up to 512 bases, else 32.
 * Results are identical for every choice. */
int kira_gpu_set_wfa_lanes(kira_ctx* ctx, int lanes);

/* ------------------------------------- ungapped prefilter and exact matches
 *
 * The step before the cascade in stage-4 alignment (src/pipeline/
 * stage4_alignment.rs:728-776): exact_match_alignment (src/alignment/
 * mod.rs:779-832) and prefilter_chain (src/alignment/prefilter.rs:93-517). A
 * pair's window is the chain's reference sequence (index.ref_bases(ref_id), or
 * the slice of it the caller ships; a resident reference with win_off = the
 * contig start); the chain's coordinates are relative to it. */

/* AnchorSpan (src/alignment/mod.rs) without ref_id / strand: the read is already
 * oriented for the strand. */
typedef struct kira_chain {
  uint32_t ref_start;
  uint32_t ref_end;
  uint32_t read_start;
  uint32_t read_end;
} kira_chain;

/* prefilter_chain's arguments (prefilter.rs:93-108) and the knobs it reads from
 * the environment. */
typedef struct kira_prefilter_cfg {
  int32_t match_score;            /* AlignmentConfig.match_score */
  int32_t mismatch;               /* AlignmentConfig.mismatch */
  int32_t xdrop;                  /* AlignmentConfig.xdrop */
  int32_t accept_enable;
  int32_t accept_only_top1;
  uint32_t accept_span_slack;
  float accept_min_identity;      /* percent; floor = (x * 100).round() as u16 */
  uint32_t accept_max_mismatches;
  int32_t accept_require_score_margin;
  uint32_t long_read_threshold;
  int32_t multi_alignments_enabled;
  int32_t tail;                   /* KIRA_UNGAP_TAIL (default 1) */
  int32_t min_identity_x10000;    /* KIRA_UNGAP_MINID; < 0: unset */
  int32_t exact_first;            /* 1: exact_match_alignment first, as stage 4 does */
} kira_prefilter_cfg;

enum kira_prefilter_kind {
  KIRA_PREFILTER_ACCEPT = 0,      /* PrefilterResult::Accept */
  KIRA_PREFILTER_REJECT = 1,      /* PrefilterResult::Reject */
  KIRA_PREFILTER_FALLBACK = 2,    /* PrefilterResult::Fallback */
  KIRA_PREFILTER_EXACT = 3        /* exact_match_alignment returned Some (exact_first) */
};

/* PrefilterOutcome (prefilter.rs:76-82) of one chain. reason = PrefilterReason::idx();
 * reason 9 (Other) carries other = 1 read_len0, 2 non_monotonic, 3 anchor0,
 * 4 span0, 5 neg_start, 6 span_oob, 7 margin_fail. len .. ref_start are the
 * UngappedStats when has_metrics; for ACCEPT and EXACT they also give the
 * alignment's span (read_start, ref_start, len M columns) and score, with nm,
 * the CIGAR ([S] M [S]; EXACT: read_len M) and the MD:Z text md[md_off, +md_len). */
typedef struct kira_prefilter_result {
  uint8_t result;
  uint8_t reason;
  uint8_t other;
  uint8_t has_metrics;
  uint16_t len;
  uint16_t mism;
  uint16_t matches;
  uint16_t identity_x10000;
  int32_t score;
  uint32_t read_start;
  uint32_t ref_start;
  uint32_t nm;
  uint32_t cigar_off;
  uint32_t n_cigar;
  uint32_t md_off;
  uint32_t md_len;
  uint32_t reserved;
} kira_prefilter_result;

/* prefilter_chain per chain (with exact_match_alignment first when cfg.exact_first).
 * is_top1 (NULL: all 1) and score_margin (NULL: INT32_MAX) are per chain. Reads up
 * to 65535 bases; a chain that reaches the extension must end inside its read and
 * window (the reference panics otherwise): KIRA_ERR_INVALID. KIRA_ERR_CAPACITY when
 * the CIGAR or MD output is too small (cigar->used / *md_used give the need).
 * Stage times: [0] inputs uploaded, [1] extension + decisions, [2] offsets,
 * [3] CIGAR + MD text, [4] downloaded. The opt-in WFA gap check
 * (KIRA_UNGAP_GAP_CHECK) is the score-only kira_gpu_wfa_batch with per-pair
 * max_score = mism * (match_score + mismatch) - 1 (ungapped_beaten_by_gap,
 * mod.rs:162-204), run by the caller on the accepted chains. */
int kira_gpu_prefilter_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_chain* chains,
                             const uint8_t* is_top1, const int32_t* score_margin,
                             const kira_prefilter_cfg* cfg, kira_prefilter_result* out,
                             kira_cigar_buf* cigar, char* md, uint64_t md_cap,
                             uint64_t* md_used);

/* exact_match_exists (mod.rs:819-832) per chain: out[i] = 1 when the whole read
 * equals the window bytes at the chain's co-linear span. */
int kira_gpu_exact_match_batch(kira_ctx* ctx, const kira_pairs* pairs, const kira_chain* chains,
                               uint8_t* out);

/* ------------------------------------------------ serving (continuous batching)
 *
 * No counterpart in the reference, whose dispatcher thread runs one blocking
 * CudaBackend::run_batch at a time (src/cuda/dispatcher.rs:21-78); this is the
 * asynchronous serving mode of the same path. A server owns `slots` worker
 * threads, each with its own context (stream + device arena); all share one
 * device-resident reference. A free slot takes the oldest queued request plus
 * every later queued request of the same kind and parameters (up to
 * max_batch_pairs pairs), runs them as one batch and writes each request's
 * results into that request's buffers. A batch starts only when its device-memory
 * estimate fits in mem_fraction of the free device memory (plus what the slot
 * already holds). Results are identical to the direct calls (kira_gpu_verify_batch
 * / kira_gpu_bsw_batch) on the request alone.
 *
 * The caller's input arrays and output buffers are borrowed from submit until the
 * request leaves KIRA_PENDING. out[i].cigar_off indexes the request's own
 * cigar_ops; a request whose CIGAR ops exceed cigar_cap ends with
 * KIRA_ERR_CAPACITY (cigar_used in kira_request_info gives the need). */
typedef struct kira_server kira_server;

typedef struct kira_server_cfg {
  int device;
  int slots;                /* concurrent batches (worker threads / streams), 1..64 */
  uint32_t max_batch_pairs; /* batch cap in pair-equivalents (a banded-SW pair counts its
                               band cells / 10050, a 150 bp read at band 33); 0 -> 2^20 */
  double mem_fraction;      /* admission: share of free device memory; 0 -> 0.5 */
} kira_server_cfg;

typedef struct kira_request_info {
  int32_t status;           /* KIRA_PENDING, KIRA_OK or the batch's error */
  uint32_t n_pairs;
  uint64_t cigar_used;
  int64_t t_submit_ns;      /* steady clock */
  int64_t t_start_ns;       /* batch start (0 while queued) */
  int64_t t_done_ns;
  uint64_t batch_id;        /* batch that ran the request */
  uint32_t batch_requests;  /* requests in that batch */
  uint32_t reserved;
} kira_request_info;

int kira_server_create(const kira_server_cfg* cfg, kira_server** out);
/* Waits for running batches, cancels queued requests (KIRA_ERR_RUNTIME). */
void kira_server_destroy(kira_server* srv);
/* Replaces the resident reference (between batches; bounded wait). */
int kira_server_ref_upload(kira_server* srv, const uint8_t* seq, uint64_t len);
/* Short-read requests: the composed verification (kira_gpu_verify_batch). */
int kira_server_submit_verify(kira_server* srv, const kira_pairs* pairs,
                              const kira_verify_params* params, kira_sw_result* out,
                              uint32_t* cigar_ops, uint64_t cigar_cap, uint64_t* ticket);
/* Long gap-fill requests: banded SW per pair (kira_gpu_bsw_batch). */
int kira_server_submit_bsw(kira_server* srv, const kira_pairs* pairs, const kira_sw_cfg* cfg,
                           kira_sw_result* out, uint32_t* cigar_ops, uint64_t cigar_cap,
                           uint64_t* ticket);
/* KIRA_PENDING while queued or running, else the request's final status. */
int kira_server_poll(kira_server* srv, uint64_t ticket);
/* Bounded wait: the final status, or KIRA_ERR_TIMEOUT after timeout_ms. */
int kira_server_wait(kira_server* srv, uint64_t ticket, int64_t timeout_ms);
int kira_server_info(kira_server* srv, uint64_t ticket, kira_request_info* info);
/* Forgets a finished ticket (KIRA_ERR_INVALID while pending). */
int kira_server_release(kira_server* srv, uint64_t ticket);
int kira_server_stats(kira_server* srv, uint64_t* batches, uint64_t* pairs, uint32_t* queued);
int kira_server_last_error(kira_server* srv, char* buf, size_t len);
/* Host milliseconds summed over batches: [0] staging inputs, [1] the pipeline call
 * (upload, kernels, result copies), [2] scattering results, [3] admission checks. */
int kira_server_profile(kira_server* srv, double* ms4);

#ifdef __cplusplus
}
#endif
#endif /* KIRA_GPU_H */
