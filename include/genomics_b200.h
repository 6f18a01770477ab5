/*
 * genomics_b200.h -- C ABI of libgenomics_b200.so, the B200 (sm_100a)
 * batched pairwise-alignment library.
 *
 * The library computes exactly what the reference's CPU path computes:
 *   - banded Smith-Waterman, genomics/cpu/align_cpu.mojo:229-309
 *     (smith_waterman_banded): score, query_end, ref_end (starts are 0 and
 *     the CIGAR is empty, align_cpu.mojo:302-309);
 *   - gap-affine WFA cost, genomics/cpu/align_cpu.mojo:75-226
 *     (wfa_affine_cpu): minimum cost or -1 past max_error;
 * over sequences stored as the reference's SequenceBatch
 * (genomics/core/sequence.mojo:23-36): 2-bit MSB-first packed uint64 words,
 * one NMask word per packed word, per-sequence word offsets and lengths.
 * N bases are stored as A (sequence.mojo:53-57) and compare equal to A.
 *
 * Conventions: every entry point returns an int status (GB2_OK == 0, the
 * others negative; gb2_strerror names them).  The caller owns every host
 * array; the library never keeps a host pointer after a call returns.
 * Device batches belong to the context that made them.  Calls on one
 * context are serialised by the context; separate contexts may be used
 * from separate threads.
 */
#ifndef GENOMICS_B200_H
#define GENOMICS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define GB2_OK 0
#define GB2_EINVAL (-1)      /* bad argument (NULL, negative size, bad config) */
#define GB2_ENOMEM (-2)      /* device or pinned allocation failed / over budget */
#define GB2_ECUDA (-3)       /* a CUDA runtime call failed */
#define GB2_ENODEV (-4)      /* no CUDA device, or not an sm_100 device */
#define GB2_ERANGE (-5)      /* input outside the exact integer range */
#define GB2_ETIMEOUT (-6)    /* a bounded wait ran out */
#define GB2_ESTATE (-7)      /* wrong state (server not running, ...) */
#define GB2_EKERNEL (-8)     /* a kernel reported an internal error flag */
#define GB2_ESCRATCH (-9)    /* request too large for the fixed no-allocation scratch */
#define GB2_ECANCELED (-10)  /* a served request was cancelled before it ran */

/* ---- configuration and result structs ------------------------------------- */

/* AlignConfig (align_cpu.mojo:18-25).  Penalties are negative. */
typedef struct {
    int32_t match_score;
    int32_t mismatch;
    int32_t gap_open;
    int32_t gap_extend;
    int32_t band_width;
} gb2_sw_cfg;

/* AlignResult (align_cpu.mojo:28-36) minus the fields that are always zero
   (query_start, ref_start) and the always-empty cigar. */
typedef struct {
    int32_t score;
    int32_t query_end;
    int32_t ref_end;
} gb2_sw_result;

/* WFAConfig (align_cpu.mojo:62-68).  Positive costs. */
typedef struct {
    int32_t x;
    int32_t o;
    int32_t e;
    int32_t max_error;
} gb2_wfa_cfg;

typedef struct gb2_ctx gb2_ctx;
typedef struct gb2_batch gb2_batch;

/* ---- flags ------------------------------------------------------------------ */
#define GB2_FLAG_PLAIN 0x0     /* one launch per band class, pairs in input order */
#define GB2_FLAG_BATCHED 0x1   /* length-bucketed device work queue, persistent kernel */
#define GB2_FLAG_INT32 0x2     /* never take the packed int16 Smith-Waterman path */
#define GB2_FLAG_GENERIC 0x4   /* force the literal per-pair kernel (testing) */
#define GB2_FLAG_GRAPH 0x8     /* gb2_sw_banded / gb2_wfa_affine: capture the call's device
                                  work into a CUDA graph on the second call with the same
                                  shape (batches, scoring, n_pairs, flags) and replay it on
                                  later ones; results are those of the eager launches */
#define GB2_FLAG_NAIVE 0x10    /* gb2_sw_banded / gb2_wfa_affine: the baseline the batched
                                  path is measured against -- one launch, one thread block
                                  per pair in input order, no planning, as the reference's
                                  launchers do (genomics/gpu/align_gpu.mojo:482-492, :524-534) */
#define GB2_FLAG_NO_PRUNE 0x20 /* gb2_wfa_affine: skip the bound pass (a banded WFA whose
                                  costs bound the optimum from above) and the exact pass's
                                  pruning by it; results are the same either way */
#define GB2_FLAG_PACKED 0x40  /* gb2_sw_banded*: take the packed int16 kernel with wide keys
                                  for batches of at most 16,384 pairs too (by default they
                                  run the int32 kernels with the most lanes per pair, which
                                  finish a small batch sooner); results are the same */
/* Tuning fields (0 = the library's choice): bits 8-15 select a kernel
 * variant; bits 16-23 set how many chunks the *_host entry points split a
 * batch into for their copy/compute pipeline. */
#define GB2_FLAGS_VARIANT(v) (((v) & 0xff) << 8)
#define GB2_FLAGS_CHUNKS(n) (((n) & 0xff) << 16)
/* gb2_wfa_cigar: cap its history arena at n MiB (1-255; 0 = the library's
   choice), which splits a batch into more groups -- for testing the grouping. */
#define GB2_FLAGS_ARENA_MIB(n) (((n) & 0xff) << 24)

/* ---- library ----------------------------------------------------------------- */

/* Library version as 10000*major + 100*minor + patch. */
int gb2_version(void);

/* Static string naming a status code. */
const char *gb2_strerror(int status);

/* ---- context (replaces GenomicsDevice, genomics/gpu/device.mojo:21-32) ------- */

/* Create a context on CUDA device `device`: one stream set, pinned staging,
   device scratch.  Fails with GB2_ENODEV when the device is not sm_100. */
int gb2_create(int device, gb2_ctx **out);
int gb2_destroy(gb2_ctx *ctx);

/* Wait for all work queued on the context. */
int gb2_sync(gb2_ctx *ctx);

/* Last error text recorded on the context (for messages beyond the code). */
const char *gb2_last_error(gb2_ctx *ctx);

/* ---- device-resident SequenceBatch -------------------------------------------
 * Replaces GenomicsDevice.upload_batch_packed / upload_lengths /
 * upload_offsets (genomics/gpu/device.mojo:60-108): one pinned staging pass
 * and asynchronous copies of the packed words, the NMask words (may be NULL:
 * alignment never reads them), the word offsets and the lengths.  The
 * batch stays on the device until gb2_batch_free. */
int gb2_batch_upload(gb2_ctx *ctx, const uint64_t *packed, int64_t n_words,
                     const uint64_t *nmask, const int64_t *offsets,
                     const int64_t *lengths, int64_t count, gb2_batch **out);
int gb2_batch_free(gb2_ctx *ctx, gb2_batch *batch);
/* Number of sequences / packed words held by a batch. */
int gb2_batch_info(const gb2_batch *batch, int64_t *count, int64_t *n_words);

/* Device-side SequenceBatch.add_sequence (genomics/core/sequence.mojo:38-66)
   for a whole batch: sequence i is ascii[starts[i] .. starts[i]+lengths[i]);
   it is copied to the device once and packed there (2-bit MSB-first words,
   non-ACGT stored as A and flagged in the NMask words), sequences appended
   in order.  The batch keeps its NMask words. */
int gb2_batch_from_ascii(gb2_ctx *ctx, const uint8_t *ascii, int64_t ascii_bytes,
                         const int64_t *starts, const int64_t *lengths, int64_t count,
                         gb2_batch **out);
/* Copies a device batch back (any pointer may be NULL; sizes from
   gb2_batch_info). */
int gb2_batch_download(gb2_ctx *ctx, const gb2_batch *batch, uint64_t *packed,
                       uint64_t *nmask, int64_t *offsets, int64_t *lengths);

/* ---- batched banded Smith-Waterman --------------------------------------------
 * Pair i = (query i of q, reference i of r), as launch_banded_sw
 * (genomics/gpu/align_gpu.mojo:460-492).  `bands` (host, may be NULL) gives
 * a per-pair band width that overrides cfg->band_width; `out` is a host
 * array of n_pairs results.  Blocking. */
int gb2_sw_banded(gb2_ctx *ctx, const gb2_batch *q, const gb2_batch *r,
                  const gb2_sw_cfg *cfg, const int32_t *bands, int64_t n_pairs,
                  gb2_sw_result *out, int flags);

/* Same, end to end from host SequenceBatch arrays: pinned staging, chunked
   host-to-device copies overlapped with the kernels, results copied back.
   Blocking. */
int gb2_sw_banded_host(gb2_ctx *ctx,
                       const uint64_t *q_packed, const int64_t *q_offsets,
                       const int64_t *q_lengths,
                       const uint64_t *r_packed, const int64_t *r_offsets,
                       const int64_t *r_lengths,
                       const gb2_sw_cfg *cfg, const int32_t *bands,
                       int64_t n_pairs, gb2_sw_result *out, int flags);

/* Per-pair drop-in for smith_waterman_banded(query, reference, cfg)
   (align_cpu.mojo:229-233): raw word pointers of one SequenceView each
   (sequence.mojo:78-94).  Upload, launch and synchronise on every call. */
int gb2_sw_pair(gb2_ctx *ctx, const uint64_t *q_words, int64_t qlen,
                const uint64_t *r_words, int64_t rlen, const gb2_sw_cfg *cfg,
                gb2_sw_result *out);

/* ---- batched gap-affine WFA ----------------------------------------------------
 * Pair i as above, as launch_wfa_affine (genomics/gpu/align_gpu.mojo:496-535)
 * but with runtime penalties; out_cost is a host array (-1 = over
 * max_error).  Requires x >= 1, e >= 1, o >= 0, max_error >= 0. */
int gb2_wfa_affine(gb2_ctx *ctx, const gb2_batch *q, const gb2_batch *r,
                   const gb2_wfa_cfg *cfg, int64_t n_pairs, int32_t *out_cost,
                   int flags);

int gb2_wfa_affine_host(gb2_ctx *ctx,
                        const uint64_t *q_packed, const int64_t *q_offsets,
                        const int64_t *q_lengths,
                        const uint64_t *r_packed, const int64_t *r_offsets,
                        const int64_t *r_lengths,
                        const gb2_wfa_cfg *cfg, int64_t n_pairs,
                        int32_t *out_cost, int flags);

/* Per-pair drop-in for wfa_affine_cpu(query, ref_seq, cfg)
   (align_cpu.mojo:75-79). */
int gb2_wfa_pair(gb2_ctx *ctx, const uint64_t *q_words, int64_t qlen,
                 const uint64_t *r_words, int64_t rlen, const gb2_wfa_cfg *cfg,
                 int32_t *out_cost);

/* ---- banded Needleman-Wunsch ------------------------------------------------------
 * needleman_wunsch_banded (genomics/cpu/align_cpu.mojo:312-377) over pairs
 * (q[i], r[i]) of two resident batches, with the intended semantics of the
 * reference (its band rows are created with capacity only and indexed,
 * :327-341; here they have 2*band+1 elements): out[i] = {score, qlen-1,
 * rlen-1}, score -1000000 when the final cell lies outside the band.  bands:
 * optional per-pair band widths (NULL: cfg->band_width).  GB2_ERANGE when a
 * value could leave int32.  GB2_FLAG_GENERIC forces the int64 literal kernel. */
int gb2_nw_banded(gb2_ctx *ctx, const gb2_batch *q, const gb2_batch *r, const gb2_sw_cfg *cfg,
                  const int32_t *bands, int64_t n_pairs, gb2_sw_result *out, int flags);

/* Per-pair drop-in for needleman_wunsch_banded(query, reference, cfg)
   (align_cpu.mojo:312-316). */
int gb2_nw_pair(gb2_ctx *ctx, const uint64_t *q_words, int64_t qlen,
                const uint64_t *r_words, int64_t rlen, const gb2_sw_cfg *cfg,
                gb2_sw_result *out);

/* ---- gap-affine WFA with CIGAR traceback -----------------------------------------
 * wfa_affine_cigar_cpu (genomics/cpu/align_cpu.mojo:380-623) over pairs
 * (q[i], r[i]) of two resident batches.  cost[i] is the gb2_wfa_affine cost
 * (-1 past max_error, then no CIGAR).  The CIGAR of pair i is
 * runs[run_offsets[i] .. run_offsets[i+1]), each run len << 2 | op with op
 * 0 '=', 1 'X', 2 'I', 3 'D' in the reference's order and run-length
 * encoding (:603-621); run_offsets has n_pairs + 1 entries.  runs_cap is the
 * capacity of `runs`: sum(qlen + rlen) over the pairs always suffices; when
 * the runs do not fit, returns GB2_ERANGE with run_offsets[n_pairs] set to the
 * number needed.  Device history: 5 B per visited wavefront cell + 12 B per
 * score, in groups that fit half the free device memory (at most 64 GiB, or
 * GB2_FLAGS_ARENA_MIB); GB2_ENOMEM when one pair alone does not fit. */
int gb2_wfa_cigar(gb2_ctx *ctx, const gb2_batch *q, const gb2_batch *r,
                  const gb2_wfa_cfg *cfg, int64_t n_pairs, int32_t *cost,
                  uint32_t *runs, int64_t runs_cap, int64_t *run_offsets, int flags);

/* Per-pair drop-in for wfa_affine_cigar_cpu(query, ref_seq, cfg)
   (align_cpu.mojo:380-384): cost out, and the CIGAR as the reference's string
   ("2=1X1=", empty when the cost is -1) into cigar[cap]; GB2_ERANGE when cap
   is too small. */
int gb2_wfa_cigar_pair(gb2_ctx *ctx, const uint64_t *q_words, int64_t qlen,
                       const uint64_t *r_words, int64_t rlen, const gb2_wfa_cfg *cfg,
                       int32_t *cost, char *cigar, int64_t cap);

/* ---- gap-affine WFA with no device allocation ------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code whose device memory belongs to a host runtime's own allocator,
 * plug-ins held to a fixed memory budget, request loops that must not
 * allocate.  Inputs and outputs are the caller's device pointers: per side a
 * SequenceBatch (packed words, int64 offsets, int64 lengths) and n_pairs
 * int32 costs out.  The wavefront scratch is a fixed device array of
 * GB2_NOALLOC_SCRATCH_BYTES inside the library, held by every GPU that loads
 * it until the process exits.  max_qlen / max_rlen bound the lengths: a
 * request whose rings ((max(x,o+e)/g + 1 + 2(e/g + 1)) slots x
 * (max_qlen + max_rlen + 5) int32 per warp, g = gcd(x, o, e)) leave room for
 * fewer than four warps returns GB2_ESCRATCH; a pair longer than stated, or
 * with a negative length or one of 2^31 or more, gets cost -2 and the call
 * returns GB2_EINVAL.  Blocking on `stream` (a
 * cudaStream_t; NULL = the legacy default stream).  The first call on a
 * device looks up the array's device address, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
#define GB2_NOALLOC_SCRATCH_BYTES (32ll << 20)
int gb2_wfa_affine_noalloc(const uint64_t *q_packed, int64_t q_words,
                           const int64_t *q_offsets, const int64_t *q_lengths,
                           const uint64_t *r_packed, int64_t r_words,
                           const int64_t *r_offsets, const int64_t *r_lengths,
                           int64_t max_qlen, int64_t max_rlen,
                           const gb2_wfa_cfg *cfg, int64_t n_pairs,
                           int32_t *out_cost, void *stream);

/* ---- one pair list over several devices --------------------------------------------
 * Pairs are independent (the reference gives each its own thread block,
 * genomics/gpu/align_gpu.mojo:80), so a list splits into contiguous slices with
 * no exchange step.  gb2_partition_pairs (host only, no device needed) writes
 * n_parts + 1 bounds: part k is pairs [bounds[k], bounds[k+1]), cut where the
 * cumulative work reaches k/n_parts of the total -- kind 0 Smith-Waterman
 * cells qlen * (2 * band + 1) (bands per pair, or `band`), kind 1 WFA
 * max(qlen, rlen)^2 (the visited cells grow with the square of the cost) --
 * plus a fixed share per pair.  The *_multi entry points run slice k on
 * ctxs[k] (each context on its own device, or several on one) from the
 * caller's host arrays, on one host thread per context, and write each
 * slice's results into `out` at its offset, so `out` is in input order.  The
 * first failing slice's status is returned. */
int gb2_partition_pairs(const int64_t *q_lengths, const int64_t *r_lengths, const int32_t *bands,
                        int32_t band, int kind, int64_t n_pairs, int n_parts, int64_t *bounds);
int gb2_sw_banded_multi(gb2_ctx *const *ctxs, int n_ctx,
                        const uint64_t *q_packed, const int64_t *q_offsets,
                        const int64_t *q_lengths,
                        const uint64_t *r_packed, const int64_t *r_offsets,
                        const int64_t *r_lengths,
                        const gb2_sw_cfg *cfg, const int32_t *bands, int64_t n_pairs,
                        gb2_sw_result *out, int flags);
int gb2_wfa_affine_multi(gb2_ctx *const *ctxs, int n_ctx,
                         const uint64_t *q_packed, const int64_t *q_offsets,
                         const int64_t *q_lengths,
                         const uint64_t *r_packed, const int64_t *r_offsets,
                         const int64_t *r_lengths,
                         const gb2_wfa_cfg *cfg, int64_t n_pairs, int32_t *out_cost, int flags);

/* ---- serving: continuous batching of alignment requests ----------------------------
 * A request is a batch of pairs; each pair is Smith-Waterman or WFA.  Requests
 * are admitted in arrival order while the device memory they need fits the
 * server's HBM budget; admitted requests are grouped and launched as soon as
 * one of the server's executors is free, so requests that arrive while others
 * run on the GPU start before those finish and their work overlaps on the
 * device.  Results are exactly those of gb2_sw_banded / gb2_wfa_affine on the
 * same pairs, whatever else is in flight. */
typedef struct {
    int64_t n_pairs;
    /* host SequenceBatch arrays of the queries and references (pair i = q i, r i);
       they and the output arrays must stay valid until the request is done */
    const uint64_t *q_packed;
    const int64_t *q_offsets;
    const int64_t *q_lengths;
    const uint64_t *r_packed;
    const int64_t *r_offsets;
    const int64_t *r_lengths;
    const int32_t *kinds;    /* per pair 0 = Smith-Waterman, 1 = WFA; NULL: all SW */
    const int32_t *bands;    /* per pair SW band; NULL: sw_cfg.band_width */
    gb2_sw_cfg sw_cfg;
    gb2_wfa_cfg wfa_cfg;
    gb2_sw_result *sw_out;   /* n_pairs entries; written for SW pairs */
    int32_t *wfa_out;        /* n_pairs entries; written for WFA pairs */
} gb2_request;

typedef struct {
    int64_t hbm_budget_bytes;     /* device bytes admitted requests may hold */
    int32_t max_inflight_groups;  /* concurrent groups (executors), 1..8 */
    int32_t max_group_pairs;      /* pairs per group (0: 65536) */
    int32_t flags;                /* GB2_FLAG_* for the launches */
} gb2_server_cfg;

typedef struct {
    int64_t submitted, completed, failed, pairs_completed, groups_launched;
    int64_t inflight_bytes, peak_inflight_bytes;
    int64_t cancelled;
} gb2_server_stats;

typedef struct gb2_server gb2_server;

/* Start a server thread on ctx (which must outlive it). */
int gb2_server_start(gb2_ctx *ctx, const gb2_server_cfg *cfg, gb2_server **out);
/* Queue a request; returns at once with a ticket.  GB2_ENOMEM if the request
   alone can never fit the budget. */
int gb2_server_submit(gb2_server *srv, const gb2_request *req, uint64_t *ticket);
/* Non-blocking: *done = 1 once the request's results are in its output arrays. */
int gb2_server_poll(gb2_server *srv, uint64_t ticket, int *done);
/* Block until the request is done (GB2_ETIMEOUT after timeout_ms; < 0 waits
   forever); returns the request's status and its latency from submit to
   results written.  The ticket is released once reported done. */
int gb2_server_wait(gb2_server *srv, uint64_t ticket, int timeout_ms, double *latency_ms);
int gb2_server_stats_get(gb2_server *srv, gb2_server_stats *st);
/* Hold admission (hold = 1): queued requests stay queued, groups already on
   the GPU finish; hold = 0 resumes.  gb2_server_stop lifts a hold. */
int gb2_server_hold(gb2_server *srv, int hold);
/* Cancel a queued request: it leaves the queue without running, and its wait
   returns GB2_ECANCELED.  A request already on the GPU, or done, cannot be
   cancelled (GB2_ESTATE); an unknown ticket is GB2_EINVAL. */
int gb2_server_cancel(gb2_server *srv, uint64_t ticket);
/* Finish every queued and running request, then stop the thread. */
int gb2_server_stop(gb2_server *srv);

/* ---- autotuner --------------------------------------------------------------------
 * The batched kernels come in variants that compute the same results with
 * different shapes: the int32 Smith-Waterman register kernels split a band row
 * over G lanes of K columns each (bands 16: G 1/2; 32: G 1/2/4; 64: G 2/4;
 * 128: G 4/8), and the WFA kernel takes 4, 2 or 1 diagonals per thread per
 * round with 3-5 resident blocks per SM.  No counterpart in the reference (its
 * kernels have one fixed shape, genomics/gpu/align_gpu.mojo:60-137).
 * gb2_autotune runs every candidate of one kernel on a caller's batch (GB2_TUNE_SW:
 * the register kernel of cfg->band_width's class, forced with GB2_FLAG_INT32;
 * GB2_TUNE_WFA: the batched WFA kernel), `reps` timed runs each after one
 * warm-up, checks that every candidate gives the first candidate's results
 * (GB2_EKERNEL otherwise), and installs the fastest in the context: later calls
 * whose flags leave the variant field (bits 8-15) at 0 use it.  Tune on the
 * batch size that will run: a small batch that leaves SMs idle favours more
 * lanes per pair than a full one.  bands (GB2_TUNE_SW, optional, host): the
 * per-pair bands of a mixed batch; each candidate of the class then runs inside
 * the whole mixed call while the other classes keep their installed variants,
 * so tuning the classes one after another fits the mix.  gb2_tune_set /
 * gb2_tune_get save and restore the table (variant 0 = the built-in choice). */
#define GB2_TUNE_SW 1
#define GB2_TUNE_WFA 2
#define GB2_TUNE_MAX 16
typedef struct gb2_tune_result {
    int32_t kind, band_class;     /* band_class: 16/32/64/128 for GB2_TUNE_SW, 0 for WFA */
    int32_t n_candidates, chosen; /* chosen: the variant now installed */
    int32_t variant[GB2_TUNE_MAX];
    float ms[GB2_TUNE_MAX];       /* median device time of one run per candidate */
} gb2_tune_result;
int gb2_autotune(gb2_ctx *ctx, int kind, const gb2_batch *q, const gb2_batch *r,
                 const void *cfg /* gb2_sw_cfg or gb2_wfa_cfg */, const int32_t *bands,
                 int64_t n_pairs, int reps, gb2_tune_result *out);
int gb2_tune_set(gb2_ctx *ctx, int kind, int band_class, int variant);
int gb2_tune_get(gb2_ctx *ctx, int kind, int band_class, int *variant);

/* ---- failure injection (testing) ---------------------------------------------------
 * No counterpart in the reference (its only failure report is WFA's -1,
 * genomics/cpu/align_cpu.mojo:226).  Arms a countdown: the nth device
 * (GB2_ALLOC_DEVICE) or pinned host (GB2_ALLOC_PINNED) allocation the library
 * makes from now on (0 = the next one) fails as if out of memory; the entry
 * point that made it returns GB2_ENOMEM after waiting for its streams, and the
 * context stays usable.  nth < 0 disarms.  Process-wide. */
#define GB2_ALLOC_DEVICE 1
#define GB2_ALLOC_PINNED 2
int gb2_debug_fail_alloc(int kind, int64_t nth);

/* ---- pinned host memory -----------------------------------------------------------
 * Page-locked host allocations: SequenceBatch arrays built here reach the
 * device by DMA without the library's staging copy. */
int gb2_host_alloc(int64_t bytes, void **out);
int gb2_host_free(void *p);

/* ---- measurement ------------------------------------------------------------------
 * CUDA events recorded on the stream the alignment kernels run on. */
int gb2_timer_start(gb2_ctx *ctx);
int gb2_timer_stop(gb2_ctx *ctx, float *ms);
/* Accumulated device time (ms) and launch count of the library's own
   kernels since the last reset; kernel_ms covers the dominant kernels. */
int gb2_stats(gb2_ctx *ctx, double *kernel_ms, int64_t *launches,
              int64_t *work_units);
int gb2_stats_reset(gb2_ctx *ctx);
/* Enable per-launch event timing (adds two events per launch). */
int gb2_set_profiling(gb2_ctx *ctx, int enable);
/* Write `bytes` into a device buffer larger than L2 on the context stream
   (L2 flush between timed iterations). */
int gb2_flush_l2(gb2_ctx *ctx);
/* Integer ALU throughput probe: runs dependent-chain microkernels of the
   named instruction class over all SMs and reports giga-ops/s.  kind: 0 IADD,
   1 IMNMX, 2 DPX viaddmax_s32, 3 DPX viaddmax_s16x2, 4 DPX vimax3_s32,
   5 LOP3, 6 IMAD, 7 SHFL, 8 vimax3_s16x2, 9 vimax3_u16x2, 10 byte_perm,
   11 viaddmax_s16x2_relu, 12 vimax_s16x2_relu. */
int gb2_int_peak(gb2_ctx *ctx, int kind, double *gops);

#ifdef __cplusplus
}
#endif
#endif /* GENOMICS_B200_H */
