/*
 * ferrous_b200.h -- C ABI of the B200 seed-extension / mate-rescue library.
 *
 * Every entry point takes plain pointers and sizes.  Sequences are byte codes
 * A=0 C=1 G=2 T=3 N=4 (classic_base_to_code, src/core/compute/encoding.rs:208),
 * left-extension jobs already reversed by the caller, exactly as the reference
 * hands them to its kernels (src/pipelines/linear/batch_extension/collect_soa.rs:150-209).
 * Host buffers are owned by the caller; device buffers by the context.
 * A context is used by one host thread at a time; create one per thread.
 * All functions return FA_OK (0) or an FA_ERR_* code; fa_last_error() gives the
 * message of the last failure on the calling thread.
 */
#ifndef FERROUS_B200_H
#define FERROUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FA_OK            0
#define FA_ERR_ARG       1   /* malformed job or parameter (reference: panic)   */
#define FA_ERR_CAPACITY  2   /* job exceeds a kernel limit or device memory     */
#define FA_ERR_CUDA      3   /* CUDA runtime failure                            */
#define FA_ERR_TIMEOUT   4   /* a bounded device wait ran out                   */
#define FA_ERR_STATE     5   /* e.g. no band model loaded                       */

/* Largest query / target lengths a job may have. */
#define FA_MAX_QLEN  4096
#define FA_MAX_TLEN  65535

/* Scoring parameters: mirrors BandedPairWiseSW (src/core/alignment/banded_swa/types.rs:106-120).
 * mat is row-major [target_base * 5 + query_base], as ksw_extend2 indexes it
 * (ksw_affine_gap.rs:990-997, 1042). */
typedef struct {
    int8_t  mat[25];
    uint8_t flags;      /* FA_PARAM_* (0 = ksw_extend2's own argument rules) */
    int8_t  _pad[2];
    int32_t m;          /* alphabet size; must be 5 */
    int32_t o_del, e_del, o_ins, e_ins;
    int32_t zdrop;
    int32_t end_bonus;
    int32_t pen_clip5, pen_clip3;   /* carried for the region merge; unused by the DP */
} fa_params;

/* fa_params.flags.
 * FA_PARAM_H0_ZERO: accept jobs with h0 == 0 and run the ksw_extend2 recurrence on them as
 *   written, without its `assert!(h0 > 0)` (ksw_affine_gap.rs:968).  The reference's job
 *   collection gives every right job h0 = 0 (collect_soa.rs:206), so a caller that hands
 *   those batches over unchanged sets this flag.  With h0 = 0 the first row is all zero, so
 *   every cell is 0 and the first row ends the run: score 0, qle = tle = 0, max_off 0, and
 *   gscore = 0, gtle = 1 when the first row's band reaches the query end (qlen <= w + 1 after
 *   the max_ins/max_del clamp), else gscore = -1, gtle = 0.  Without the flag h0 <= 0 is
 *   FA_ERR_ARG, where ksw_extend2 panics.  Negative h0 is FA_ERR_ARG either way. */
#define FA_PARAM_H0_ZERO 1u

#define FA_DIR_LEFT  0
#define FA_DIR_RIGHT 1

/* One extension job: mirrors BatchedExtensionJob (batch_extension/types.rs:20-41)
 * without the read/chain/seed ids, which the caller keeps (results come back in
 * job order). */
typedef struct {
    uint64_t q_off;     /* offset of the query in the query buffer   */
    uint64_t t_off;     /* offset of the target in the target buffer */
    int32_t  qlen;      /* query_len                                  */
    int32_t  tlen;      /* ref_len                                    */
    int32_t  h0;        /* initial score; > 0 (ksw_affine_gap.rs:968), or 0 with FA_PARAM_H0_ZERO */
    int32_t  w;         /* band_width                                 */
    int32_t  dir;       /* FA_DIR_LEFT / FA_DIR_RIGHT                 */
    int32_t  _pad;
} fa_job;

/* KswExtendResult (ksw_affine_gap.rs:902-916), same field order. */
typedef struct {
    int32_t score, qle, tle, gtle, gscore, max_off;
} fa_ext_result;

/* Band-retry policies.
 * FA_POLICY_SINGLE : one ksw_extend2 run at job.w (what execute_batch_simd_scoring returns).
 * FA_POLICY_BWA    : bwa-mem2 mem_chain2aln: try w << k for k < max_tries; stop when the
 *                    score equals the previous try's (first "previous" = 0 for left jobs,
 *                    h0 for right jobs) or max_off < (w>>1)+(w>>2).
 * FA_POLICY_LEARNED: start at w_first[i] (from the band model or the caller), double up to
 *                    job.w; accept a narrow run per `judge`; at job.w continue as FA_POLICY_BWA. */
#define FA_POLICY_SINGLE  0
#define FA_POLICY_BWA     1
#define FA_POLICY_LEARNED 2

#define FA_JUDGE_CERT    1  /* accept a narrow run only when its band clamp never bound (sound) */
#define FA_JUDGE_MAXOFF  2  /* also accept when max_off < (w>>1)+(w>>2) (the bwa-mem2 test)    */
#define FA_JUDGE_GLOBAL  4  /* with MAXOFF: additionally require gscore == score              */
#define FA_JUDGE_BOUND   8  /* accept when the exit-bound certificate holds (sound): no path
                               leaving the narrow run's region can reach any output statistic */
#define FA_JUDGE_ONCE   16  /* retry rule: a rejected narrow run goes straight to the configured
                               band instead of doubling (one narrow try per job)            */
#define FA_JUDGE_HINT   32  /* with ONCE and BOUND: a rejected first narrow run retries once
                               at the band its certificate's shortfall suggests (rounded up
                               to the band ladder) when that is at most half the configured
                               band; then the configured band                                */

typedef struct {
    int32_t mode;
    int32_t max_tries;   /* bwa-mem2 MAX_BAND_TRY = 2 */
    int32_t judge;       /* FA_JUDGE_* for FA_POLICY_LEARNED */
    int32_t w_min;       /* smallest band the learned path may start at */
} fa_policy;

typedef struct {
    uint64_t cells;          /* sum of (end-beg) of the final accepted runs      */
    uint64_t cells_executed; /* every row range actually computed, retries incl. */
    uint32_t jobs;
    uint32_t retries;        /* extra runs beyond the first, summed over jobs    */
    uint32_t misses;         /* learned path: jobs whose first narrow run failed */
    uint32_t kernel_launches;
    float    kernel_ms;      /* device time of the DP kernels                    */
    float    total_ms;       /* wall time of the call                            */
} fa_ext_stats;

/* Mate-rescue local SW: ksw_align2 flags (ksw_affine_gap.rs:17-21). */
#define FA_KSW_XBYTE  0x10000u
#define FA_KSW_XSTOP  0x20000u
#define FA_KSW_XSUBO  0x40000u
#define FA_KSW_XSTART 0x80000u

typedef struct {
    int8_t  mat[25];
    int8_t  _pad[3];
    int32_t m;                  /* must be 5 */
    int32_t o_del, e_del, o_ins, e_ins;
} fa_mate_params;

typedef struct {
    uint64_t q_off, t_off;
    int32_t  qlen, tlen;
    uint32_t xtra;              /* ksw_align2 xtra word */
    int32_t  _pad;
} fa_mate_job;

/* Kswr (ksw_affine_gap.rs:51-61), same field order. */
typedef struct {
    int32_t score, te, qe, score2, te2, tb, qb;
} fa_kswr;

typedef struct fa_ctx fa_ctx;

/* ---- context ---------------------------------------------------------- */
int         fa_ctx_create(int device, fa_ctx **out);
void        fa_ctx_destroy(fa_ctx *ctx);
const char *fa_last_error(void);
const char *fa_version(void);

/* Diagnostics (no reference counterpart): SM count / opt-in shared memory of the
 * context's device, and the measured throughput of one integer instruction kind
 * (0: __viaddmax_s16x2_relu, 1: __vimax3_s16x2_relu, 2: __viaddmax_s32_relu,
 *  3: __vimax3_s32, 4: add + max as two instructions, 5: half2 max, 6: half2 add,
 *  7: integer multiply-add, 8 / 9: kind 0 and kind 5 / 7 on alternate chains), used as the
 * roofline peak (kind 0) and to tell which instruction kinds share an issue pipe. */
int fa_device_info(fa_ctx *ctx, int *sm_count, int *smem_optin_bytes);
int fa_probe_int_peak(fa_ctx *ctx, int kind, double *ops_per_s, float *ms);

/* xtra word the reference builds for a mate-rescue job
 * (src/pipelines/linear/paired/mate_rescue.rs:314-321, 653-659). */
uint32_t fa_mate_xtra(int32_t mate_len, int32_t match_score, int32_t min_seed_len);

/* ---- seed extension ----------------------------------------------------
 * Replaces execute_batch_simd_scoring (src/pipelines/linear/batch_extension/dispatch.rs:31-86):
 * one result per job, in job order.  Host buffers; copies in and out inside the call.
 * qseq/tseq hold qseq_len/tseq_len bytes; every job's range must lie inside them. */
int fa_ext_batch(fa_ctx *ctx, const fa_params *p, const fa_job *jobs, uint32_t n,
                 const uint8_t *qseq, uint64_t qseq_len,
                 const uint8_t *tseq, uint64_t tseq_len,
                 fa_ext_result *out, fa_ext_stats *stats);

/* Same, with a band-retry policy.  w_first may be NULL (then the loaded band model
 * predicts it for FA_POLICY_LEARNED).  w_final (may be NULL) receives the band of
 * the accepted run per job. */
int fa_ext_batch_policy(fa_ctx *ctx, const fa_params *p, const fa_policy *pol,
                        const fa_job *jobs, uint32_t n,
                        const uint8_t *qseq, uint64_t qseq_len,
                        const uint8_t *tseq, uint64_t tseq_len,
                        const int32_t *w_first, fa_ext_result *out,
                        int32_t *w_final, fa_ext_stats *stats);

/* Device-resident variant (no reference counterpart): every pointer is device memory
 * and the kernels run asynchronously on `stream` (a cudaStream_t, NULL = the
 * context's stream) after one small synchronous read of the query-length histogram.
 * d_order (may be NULL) is a permutation of [0,n) giving the processing order; when
 * NULL the jobs are ordered longest-first on the device.  Results are written at the
 * job's own index.  Job ranges must lie inside the sequence buffers (not checked);
 * argument and capacity violations found by the kernels are reported by the next
 * fa_ctx_sync(). */
int fa_ext_batch_device(fa_ctx *ctx, const fa_params *p, const fa_job *d_jobs, uint32_t n,
                        const uint8_t *d_qseq, const uint8_t *d_tseq,
                        const uint32_t *d_order, fa_ext_result *d_out, void *stream);

/* Waits for the stream of the last device-resident call and reports the errors its
 * kernels detected. */
int fa_ctx_sync(fa_ctx *ctx);

/* ---- 2-bit packed sequences (no reference counterpart) ------------------
 * The same extension on sequences held 2 bits per base, a quarter of the bytes to move and
 * read: base k is bits 2*(k % 4) .. 2*(k % 4) + 1 of byte k / 4 (A=0 C=1 G=2 T=3), and the N
 * bases (code 4, which 2 bits cannot hold) are listed as sorted, non-overlapping runs -- the
 * way the reference's index keeps a 2-bit .pac beside its ambiguous stretches
 * (src/pipelines/linear/index/bntseq.rs:451-535).  The packed value stored at an N position
 * is ignored.  Job offsets q_off / t_off and lengths count bases; left jobs are reversed by
 * the caller as with byte codes.  Results are identical to the byte-code entry points on the
 * same bases. */
typedef struct {
    uint64_t pos;               /* first base of the run */
    uint64_t len;               /* bases; pos + len <= n_bases */
} fa_nrun;

typedef struct {
    const uint8_t *bases;       /* (n_bases + 3) / 4 bytes; device pointers must be 4-byte aligned */
    uint64_t n_bases;
    const fa_nrun *n_runs;      /* sorted by pos, non-overlapping; NULL when n_nruns == 0 */
    uint64_t n_nruns;           /* at most 2^32 - 1 */
} fa_packed_seq;

/* fa_ext_batch_policy on packed host buffers: same policies, results, statistics and
 * errors.  Batches of 32,768 jobs or more upload the packed bases in slices under the kernels
 * (job records first); with every job's sequences at increasing offsets in job order and a
 * pinned `out`, results return slice by slice behind the uploads.  FA_POLICY_BWA and
 * FA_POLICY_LEARNED batches (w_first given) run their rounds slice by slice as each slice
 * arrives. */
int fa_ext_batch_packed(fa_ctx *ctx, const fa_params *p, const fa_policy *pol, const fa_job *jobs, uint32_t n,
                        const fa_packed_seq *qseq, const fa_packed_seq *tseq, const int32_t *w_first,
                        fa_ext_result *out, int32_t *w_final, fa_ext_stats *stats);

/* fa_ext_batch_device on packed device buffers (the fa_packed_seq structs themselves are host
 * memory holding device pointers). */
int fa_ext_batch_packed_device(fa_ctx *ctx, const fa_params *p, const fa_job *d_jobs, uint32_t n,
                               const fa_packed_seq *d_qseq, const fa_packed_seq *d_tseq, const uint32_t *d_order,
                               fa_ext_result *d_out, void *stream);

/* Extension kernel choice for this context (no reference counterpart):
 * FA_KERNEL_AUTO     autotuned: the fastest exact candidate measured on the call's data;
 * FA_KERNEL_INT32    int32 cells, one job per thread;
 * FA_KERNEL_INT16X2  int16x2 cells, two jobs per thread, for bwa-form scoring matrices
 *                    (a on the diagonal with 1 <= a <= 3, -b off it, N = -1 or 0; else int32);
 * FA_KERNEL_ROWS2    int16x2 cells, two target rows per thread with 8-bit column state,
 *                    for bwa-form matrices and queries up to 254 bases; a job whose
 *                    h0 + a * qlen exceeds 255 runs in the int32 kernel within the same call.
 * Every choice gives identical results. */
#define FA_KERNEL_AUTO    0
#define FA_KERNEL_INT32   1
#define FA_KERNEL_INT16X2 2
#define FA_KERNEL_ROWS2   3
int fa_ctx_set_kernel(fa_ctx *ctx, int kernel);
/* The kernel the last call ran (FA_KERNEL_INT32 / _INT16X2 / _ROWS2) and its threads per
 * block, and the last autotuning table (up to cap candidates: kernel, threads per block,
 * ms per sample run); *n_cand = 0 when no tuning has run.  With FA_KERNEL_AUTO (the
 * default) the first call of each (query capacity class, configured band) times every
 * exact candidate on its longest jobs and keeps the fastest. */
int fa_ctx_kernel_choice(fa_ctx *ctx, int *kernel, int *threads_per_block, int cap, int *cand_kernel,
                         int *cand_threads, float *cand_ms, int *n_cand);
/* Threads per block (64, 128 or 256) of the int32 kernel when FA_KERNEL_INT32 is set;
 * with FA_KERNEL_ROWS2, 128 selects 128 threads per block and any other value 64. */
int fa_ctx_set_threads(fa_ctx *ctx, int threads_per_block);

/* Graph mode (no reference counterpart): with it on, fa_ext_batch_policy and
 * fa_ext_batch_learned run their device work -- band features and prediction, every
 * extension round, band check and retry -- as one CUDA graph: recorded at the first call
 * of a shape (job count, longest query, widest band, policy, scoring, model constants,
 * buffer addresses) and replayed by later calls of the same shape, with no host round
 * trip between rounds.  Results are identical either way.  The host-side copies stay
 * outside the graph.  Turning it off releases the recorded graph. */
int fa_ctx_set_graph(fa_ctx *ctx, int enable);

/* Upload slices of host batches of 32,768 jobs or more (no reference counterpart): the job
 * records and sequences of a single-band batch, and of a retry-policy or learned batch that
 * runs its rounds slice by slice, go up in this many graded slices (2..8; 1: the whole batch
 * goes up before one run of the kernels over all of it; 0 keeps a value, -1 restores the
 * defaults: 8 for byte codes, whose uploads are the bottleneck; 3 for the rounds of a packed
 * batch; 6 for a packed single-band batch).  Results are identical for every setting; only
 * the overlap of copies and kernels changes. */
int fa_ctx_set_slices(fa_ctx *ctx, int single_band, int policy_rounds);

/* Kernel timing of device-resident calls (no reference counterpart): with timing on,
 * fa_ext_batch_device brackets its extension kernels with CUDA events on the call's
 * stream; fa_ctx_last_timing waits for them and returns their device time and the
 * number of kernels the last call launched. */
int fa_ctx_set_timing(fa_ctx *ctx, int enable);
int fa_ctx_last_timing(fa_ctx *ctx, float *kernel_ms, int *launches);

/* No reference counterpart.  Device-resident extension for callers that cannot
 * allocate device memory (a pool allocator owns the device memory, a fixed memory
 * budget, or an allocation-free latency path): same arguments and results as
 * fa_ext_batch_device without the context, and no cudaMalloc/cudaFree or other
 * allocation.  Its scratch (query-length histogram, job order, status word) lives in
 * one file-scope device array of about 1 MiB that every GPU loading the library keeps
 * until exit, so a call takes at most FA_NOALLOC_MAX_JOBS jobs (more -> FA_ERR_CAPACITY).
 * It runs on the current device and on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and returns once the results are in d_out, reporting kernel-detected
 * argument errors.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it for the life of the process, which assumes the
 * device's primary context (the runtime API's default) and no cudaDeviceReset between
 * calls; make that first call before any stream capture.  All calls share the one array: calls that overlap on the GPU (from several
 * host threads or streams at once) race and must be serialised by the caller. */
#define FA_NOALLOC_MAX_JOBS (1u << 18)
int fa_ext_batch_device_noalloc(const fa_params *p, const fa_job *d_jobs, uint32_t n,
                                const uint8_t *d_qseq, const uint8_t *d_tseq,
                                fa_ext_result *d_out, void *stream);

/* ---- alignment regions from extension results --------------------------
 * Replaces merge_scores_to_regions (src/pipelines/linear/region.rs:737-890), the consumer
 * of the left/right extension batches: for each seed of a chain, the region its
 * extensions reach -- per side the local bounds (qle/tle) unless gscore > 0 and
 * gscore > score - pen_clip, then the query end and gtle (bwa-mem2's clip decision,
 * region.rs:792-835) -- its total score, true score and seed coverage, and per chain
 * the region of the first seed with the strictly highest total score.  Reference
 * coordinates stay in FM-index space: the conversion to chromosome coordinates
 * (coordinates.rs, needs the index) and the chain's frac_rep stay with the caller. */
typedef struct {
    int32_t a;           /* match score: a seed alone scores len * a (MemOpt.a) */
    int32_t pen_clip5;   /* clipping penalty of left extensions (MemOpt.pen_clip5) */
    int32_t pen_clip3;   /* clipping penalty of right extensions (MemOpt.pen_clip3) */
    int32_t w;           /* band width recorded in every region (MemOpt.w) */
} fa_region_opts;

/* One seed of a chain with its extension jobs: Seed + SeedExtensionMapping (region.rs:230-235). */
typedef struct {
    uint64_t ref_pos;     /* seed.ref_pos (FM-index space) */
    int32_t  query_pos;   /* seed.query_pos */
    int32_t  len;         /* seed.len */
    int32_t  left_job;    /* index into the left results, -1 = none (an index past them is ignored) */
    int32_t  right_job;   /* index into the right results, -1 = none */
} fa_seed_ext;

/* The AlignmentRegion fields (region.rs:47-100) this step sets. */
typedef struct {
    uint64_t rb, re;      /* reference bounds [rb, re), FM-index space */
    int32_t  qb, qe;      /* query bounds [qb, qe) */
    int32_t  score;       /* total score: left result's score (or len * a) + right result's score */
    int32_t  truesc;
    int32_t  seedcov;     /* summed length of the chain's seeds inside the region */
    int32_t  seedlen0;    /* length of the chosen seed */
    int32_t  w;
    int32_t  seed;        /* index into seeds of the chosen seed; -1 = the chain gives no region */
} fa_region;

/* Chain c owns seeds[chain_first[c] .. chain_first[c+1]) in the reference's mapping order
 * (the chain's seeds last to first, region.rs:397) and its read has query_len[c] bases;
 * chain_first has n_chains + 1 entries.  left/right are the results of the left and right
 * extension batches the jobs index.  out[c] for every chain (seed = -1 for an empty chain). */
int fa_merge_regions(fa_ctx *ctx, const fa_region_opts *opt, const uint32_t *chain_first, uint32_t n_chains,
                     const int32_t *query_len, const fa_seed_ext *seeds, uint32_t n_seeds,
                     const fa_ext_result *left, uint32_t n_left, const fa_ext_result *right, uint32_t n_right,
                     fa_region *out);
/* Device-resident variant (no reference counterpart): device pointers, asynchronous on
 * `stream` (NULL = the context's stream); a malformed chain range is reported by the next
 * fa_ctx_sync().  With fa_ctx_set_timing on, fa_ctx_last_timing covers its kernel. */
int fa_merge_regions_device(fa_ctx *ctx, const fa_region_opts *opt, const uint32_t *d_chain_first,
                            uint32_t n_chains, const int32_t *d_query_len, const fa_seed_ext *d_seeds,
                            uint32_t n_seeds, const fa_ext_result *d_left, uint32_t n_left,
                            const fa_ext_result *d_right, uint32_t n_right, fa_region *d_out, void *stream);

/* ---- extension jobs from chains ----------------------------------------
 * Replaces collect_extension_jobs_batch_soa (src/pipelines/linear/batch_extension/
 * collect_soa.rs:28-230): per kept chain with seeds, the reference window
 * [rmax0, rmax1) its seeds can reach (cal_max_gap margins, chaining.rs:1108-1116, kept on
 * one strand), fetched from the 2-bit packed reference (bntseq.rs:451-535: the reverse
 * strand is the reverse complement of the forward one), and for each seed, last to first,
 * a left job (reversed read prefix against the reversed window before the seed, h0 =
 * len * a) and a right job (read suffix against the window after the seed, h0 = 0), with
 * the seed table the region merge reads.  Sequences are written once per read (forward |
 * reversed) and once per chain window (forward | reversed); jobs address slices of them. */
typedef struct {
    int32_t a;                  /* match score */
    int32_t o_del, e_del, o_ins, e_ins;
    int32_t w;                  /* band width given to every job (MemOpt.w) */
} fa_collect_opts;

typedef struct {                /* one chain of a read (SoA chain batch entry) */
    uint32_t read;              /* index of its read */
    uint32_t seed_first;        /* its seeds: seeds[seed_first .. seed_first + n_seeds), chain order */
    uint32_t n_seeds;
    int32_t  kept;              /* 0: filtered out, no jobs (collect_soa.rs:74-80) */
} fa_chain;

typedef struct {                /* one seed (SoA seed batch entry) */
    uint64_t ref_pos;           /* FM-index space: [0, l_pac) forward, [l_pac, 2 l_pac) reverse */
    int32_t  query_pos;
    int32_t  len;
} fa_seed;

typedef struct {
    uint32_t n_left, n_right;   /* jobs written */
    uint32_t n_seed_ext;        /* seed-table entries written */
    uint32_t _pad;
    uint64_t qbuf_len, tbuf_len;   /* bytes of query / target sequence the jobs address */
} fa_collect_counts;

/* The 2-bit packed reference (l_pac bases, the .pac layout below) kept on the device for
 * the collection calls of this context (no reference counterpart): a fa_collect_ext_jobs,
 * fa_collect_ext_jobs_packed or fa_collect_mate_jobs call given pac == NULL and the same
 * l_pac reads this copy instead of uploading the reference again.  pac == NULL drops it. */
int fa_ctx_set_reference(fa_ctx *ctx, const uint8_t *pac, uint64_t l_pac);

/* reads: read r is reads[read_off[r] .. read_off[r+1]) (codes 0-4); pac: the .pac layout,
 * base k in bits 7-6 of byte k/4 for k % 4 == 0, down to bits 1-0 for k % 4 == 3.
 * Outputs (caller-allocated): left_jobs/right_jobs hold up to n_seeds jobs each, in the
 * reference's order; their q_off/t_off address qbuf (2 x the reads' bytes: read r forward
 * at 2 read_off[r], reversed right after it) and tbuf (tbuf_cap bytes: per chain its
 * window forward, then reversed); seed_ext + chain_first (n_chains + 1) are the region-merge seed table,
 * seed_ext's left_job/right_job being indices into left_jobs/right_jobs (the reference
 * numbers them per read; here across the batch); chain_win gets each chain's [rmax0,
 * rmax1) (two u64 per chain; 0,0 for a chain without jobs).  When tbuf_cap is too small
 * nothing is written except counts (with the bytes needed) and FA_ERR_CAPACITY returns.
 * With fa_ctx_set_timing on, fa_ctx_last_timing covers the call's kernels (and the one read
 * of the totals between its planning and filling launches). */
int fa_collect_ext_jobs(fa_ctx *ctx, const fa_collect_opts *opt, const uint8_t *pac, uint64_t l_pac,
                        const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads,
                        const fa_chain *chains, uint32_t n_chains, const fa_seed *seeds, uint32_t n_seeds,
                        fa_job *left_jobs, fa_job *right_jobs, uint8_t *qbuf, uint8_t *tbuf, uint64_t tbuf_cap,
                        fa_seed_ext *seed_ext, uint32_t *chain_first, uint64_t *chain_win,
                        fa_collect_counts *counts);

/* fa_collect_ext_jobs with the query and target buffers 2-bit packed (no reference
 * counterpart; the fa_packed_seq layout, so the jobs go straight to fa_ext_batch_packed):
 * qbases gets (counts->qbuf_len + 3) / 4 bytes and tbases (counts->tbuf_len + 3) / 4 bytes
 * (at most tbases_cap), qruns / truns the sorted N runs of each buffer (at most qruns_cap /
 * truns_cap; n_runs[0] / n_runs[1] their counts).  The jobs, seed table and chain bounds are
 * those of fa_collect_ext_jobs.  The packing runs on the device, so a quarter of the bases'
 * bytes come back.  FA_ERR_CAPACITY with counts (and, for the runs, n_runs) filled when a
 * buffer is too small; nothing else is written then. */
int fa_collect_ext_jobs_packed(fa_ctx *ctx, const fa_collect_opts *opt, const uint8_t *pac, uint64_t l_pac,
                               const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads,
                               const fa_chain *chains, uint32_t n_chains, const fa_seed *seeds, uint32_t n_seeds,
                               fa_job *left_jobs, fa_job *right_jobs, uint8_t *qbases, fa_nrun *qruns,
                               uint64_t qruns_cap, uint8_t *tbases, uint64_t tbases_cap, fa_nrun *truns,
                               uint64_t truns_cap, fa_seed_ext *seed_ext, uint32_t *chain_first,
                               uint64_t *chain_win, fa_collect_counts *counts, uint64_t *n_runs);

/* ---- CIGAR regeneration ------------------------------------------------
 * Replaces scalar_banded_swa (src/core/alignment/banded_swa/scalar/implementation.rs:5-440),
 * the banded alignment with traceback that turns a region's bounds back into a CIGAR
 * (src/pipelines/linear/region.rs:1029-1070, there with h0 = 0 and end_bonus 0): the
 * banded recurrence with the match term clamped at zero, a traceback from the best cell
 * (ties M, then deletion, then insertion), a 5' soft clip for the query left over, and at
 * the 3' end a soft clip or an M run to the query end (clip when gscore <= 0 or
 * gscore <= score - pen_clip3).  Codes above 4 count as N, as the reference clamps them. */
typedef struct {
    uint64_t q_off, t_off;   /* query / target offsets in the sequence buffers */
    int32_t  qlen, tlen;
    int32_t  w;              /* band, as given (>= 0; the reference's infer_band_width at region.rs:1277) */
    int32_t  h0;             /* initial score (0 for CIGAR regeneration) */
} fa_cigar_job;

/* OutScore (banded_swa/types.rs:77-85) and the lengths of the three outputs. */
typedef struct {
    int32_t score, qle, tle, gtle, gscore, max_off;   /* qle = query_end_pos, tle = target_end_pos, gtle = gtarget_end_pos */
    int32_t n_cigar;   /* CIGAR operations: len << 4 | op, op 0 = M, 1 = I, 2 = D, 4 = S */
    int32_t n_ref;     /* aligned reference bases (ref_aligned) */
    int32_t n_query;   /* aligned query bases (query_aligned) */
    int32_t cells;     /* cells the recurrence evaluated */
} fa_cigar_result;

/* Job k's outputs start at cigar[sum over earlier jobs of (qlen + tlen + 2)],
 * ref_aligned[sum of earlier tlen] and query_aligned[sum of earlier qlen] (each job's
 * capacity).  p supplies the scoring matrix, gaps, zdrop and pen_clip3 (end_bonus unused).
 * With fa_ctx_set_timing on, fa_ctx_last_timing covers the kernel. */
int fa_cigar_batch(fa_ctx *ctx, const fa_params *p, const fa_cigar_job *jobs, uint32_t n,
                   const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len,
                   fa_cigar_result *out, uint32_t *cigar, uint8_t *ref_aligned, uint8_t *query_aligned);

/* fa_cigar_batch with the CIGAR words packed: job k's n_cigar words start at
 * cigar[cigar_first[k]], cigar_first[k] being the sum of the earlier jobs' n_cigar (the
 * reference returns one operation vector per alignment; a batch of 151-bp regions has a few
 * words per job against the qlen + tlen + 2 capacity slots above).  ref_aligned and
 * query_aligned keep their slots.  A batch with more than cigar_cap words returns
 * FA_ERR_CAPACITY with out and cigar_first filled, so the caller can size the buffer. */
int fa_cigar_batch_packed(fa_ctx *ctx, const fa_params *p, const fa_cigar_job *jobs, uint32_t n,
                          const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len,
                          fa_cigar_result *out, uint32_t *cigar, uint64_t cigar_cap, uint64_t *cigar_first,
                          uint8_t *ref_aligned, uint8_t *query_aligned);

/* ---- mate rescue -------------------------------------------------------
 * Replaces the ksw_align2 calls of execute_mate_rescue_batch_with_engine
 * (src/pipelines/linear/paired/mate_rescue.rs:595-685). */
int fa_mate_sw_batch(fa_ctx *ctx, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                     const uint8_t *qseq, uint64_t qseq_len,
                     const uint8_t *tseq, uint64_t tseq_len,
                     fa_kswr *out, fa_ext_stats *stats);

/* fa_mate_sw_batch on 2-bit packed host buffers (fa_packed_seq; no reference counterpart):
 * jobs address bases by position.  A quarter of the sequence bytes go up; the device
 * unpacks them (N runs applied) before the SW kernels, so the results and statistics are
 * fa_mate_sw_batch's on the same bases.  Bad N run lists fail the call with FA_ERR_ARG. */
int fa_mate_sw_batch_packed(fa_ctx *ctx, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                            const fa_packed_seq *qseq, const fa_packed_seq *tseq, fa_kswr *out,
                            fa_ext_stats *stats);

/* Mate-rescue jobs (collect_rescue_jobs_for_read_soa, mate_rescue.rs:1804-2045): per rescue
 * candidate -- a read whose mate (the anchor) aligned -- nothing unless its primary
 * alignment scores at least best - pen_unpaired; then the orientations not yet failed
 * (insert-size statistics) nor covered by one of the read's own alignments at a consistent
 * distance (mem_infer_dir, mate_rescue.rs:537-551), and for each a reference window
 * [anchor +/- insert-size bounds, plus the read length] cut to the anchor's chromosome
 * (bns_fetch_seq, bntseq.rs:700-739); a window on that chromosome of at least min_seed_len
 * bases gives a job: the read (reverse complemented for the reverse orientations) against
 * the window, read from the 2-bit packed reference. */
typedef struct { int32_t low, high, failed, _pad; } fa_insert_bounds;   /* InsertSizeStats per orientation */

/* InsertSizeStats (insert_size.rs:23-29). */
typedef struct {
    double  avg, std;
    int32_t low, high;   /* proper-pair bounds */
    int32_t failed;
    int32_t _pad;
} fa_insert_stats;

/* Replaces calculate_insert_size_stats (insert_size.rs:73-243): the four orientations'
 * statistics (FF, FR, RF, RR) of n pairs given as FM-index positions (pairs[2k] = read 1,
 * pairs[2k+1] = read 2, as the reference's (pos1, pos2)), bit-identical to the reference's
 * double arithmetic.  out4[r].low / high / failed are the fa_insert_bounds of the job
 * collection below. */
int fa_insert_size_stats(fa_ctx *ctx, uint64_t l_pac, const int64_t *pairs, uint32_t n, fa_insert_stats *out4);

typedef struct {                /* one alignment of a read (SoAAlignmentResult entry) */
    int64_t pos;                /* 0-based position on its chromosome */
    int32_t ref_id;
    int32_t is_rev;             /* flag & REVERSE */
    int32_t ref_len;            /* reference bases its CIGAR covers */
    int32_t score;
} fa_rescue_aln;

typedef struct {                /* one rescue attempt */
    uint32_t read;              /* the read to rescue: reads[read_off[read] .. read_off[read+1]) */
    uint32_t aln_first;         /* its alignments: alns[aln_first .. aln_first + aln_count) */
    uint32_t aln_count;
    uint32_t primary;           /* index into alns of its primary alignment */
    fa_rescue_aln anchor;       /* the mate's primary alignment */
} fa_rescue_cand;

typedef struct {
    int32_t pen_unpaired, max_matesw, min_seed_len, match_score;
} fa_rescue_opts;

typedef struct {                /* per job: which attempt, orientation and window it came from */
    uint32_t cand;
    int32_t  orientation;       /* 0 FF, 1 FR, 2 RF, 3 RR */
    int32_t  is_rev;
    int32_t  rid;
    int64_t  adj_rb, adj_re;
} fa_rescue_job_info;

/* chr_off/chr_len: the reference sequences (annotations: offset and length, n_chr of them)
 * of the packed reference (pac, l_pac as for fa_collect_ext_jobs).  Outputs: up to
 * 4 n_cand jobs and infos, in the reference's order (attempts in order, orientations 0-3);
 * jobs' q_off/t_off address qbuf (qbuf_cap bytes) and tbuf (tbuf_cap bytes); their xtra is
 * fa_mate_xtra(read length, match_score, min_seed_len).  With too small a buffer nothing is
 * written except counts (n_left = jobs, qbuf_len, tbuf_len) and FA_ERR_CAPACITY returns. */
int fa_collect_mate_jobs(fa_ctx *ctx, const fa_rescue_opts *opt, const fa_insert_bounds *bounds4,
                         const uint8_t *pac, uint64_t l_pac, const uint64_t *chr_off, const uint64_t *chr_len,
                         uint32_t n_chr, const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads,
                         const fa_rescue_aln *alns, uint32_t n_alns, const fa_rescue_cand *cands, uint32_t n_cand,
                         fa_mate_job *jobs, fa_rescue_job_info *info, uint8_t *qbuf, uint64_t qbuf_cap,
                         uint8_t *tbuf, uint64_t tbuf_cap, fa_collect_counts *counts);

/* ---- learned band (no reference counterpart) ----------------------------
 * A 16-64-32-1 MLP (BF16 weights, FP32 accumulation) predicts log2 of the band each
 * extension needs from 16 features of the job (seed length, lengths, h0, the chain's
 * seed-diagonal spread, mismatch counts on the seed diagonal and its neighbours).
 * Trained on the GPU by this library's own forward/backward/Adam kernels. */
#define FA_BAND_NPARAMS 3201
typedef struct {
    int32_t diag_spread;   /* |diagonal difference| between the seed and its chain partner */
    int32_t has_partner;   /* 1 if the chain has a second seed                             */
} fa_band_hint;
typedef struct fa_band_model fa_band_model;

int  fa_band_model_create(uint64_t seed, fa_band_model **out);
void fa_band_model_destroy(fa_band_model *m);
int  fa_band_model_get(const fa_band_model *m, float *weights, float *mean16, float *std16);
int  fa_band_model_set(fa_band_model *m, const float *weights, const float *mean16, const float *std16);
int  fa_band_model_save(const fa_band_model *m, const char *path);   /* versioned, checksummed */
int  fa_band_model_load(const char *path, fa_band_model **out);
/* feature normalisation constants from a training feature matrix (n x 16) */
int  fa_band_model_fit_norm(fa_band_model *m, const float *x, uint32_t n);
/* x[n*16] raw features of host jobs (hints may be NULL) */
int  fa_band_features(fa_ctx *ctx, const fa_params *p, const fa_job *jobs, uint32_t n,
                      const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len,
                      const fa_band_hint *hints, float *x);
/* y[n] = MLP(x) (log2 band); w_out[n] = ceil(2^(y+margin)) raised to w_min and rounded up
 * to the ladder 2, 3, 4, 6, 8, 12, 16, ... (2^k and 3*2^k), or job.w when twice that
 * exceeds job.w (such jobs are better started at the configured band) */
int  fa_band_predict(fa_ctx *ctx, const fa_band_model *m, const float *x, const fa_job *jobs, uint32_t n,
                     float margin, int w_min, float *y_out, int32_t *w_out);
/* mean gradient and loss of the pinball(tau) loss on (x, target = log2 band) */
int  fa_band_grad(fa_ctx *ctx, const fa_band_model *m, const float *x, const float *target, uint32_t n,
                  float tau, float *grad, float *loss);
/* Adam training on the GPU; epoch_loss[epochs] may be NULL */
int  fa_band_train(fa_ctx *ctx, fa_band_model *m, const float *x, const float *target, uint32_t n, int epochs,
                   uint32_t batch, float lr, float tau, uint64_t seed, float *epoch_loss);
/* Learned-band extension: features and prediction on the GPU give each job its first
 * band (w_first_out, may be NULL), then FA_POLICY_LEARNED runs as in fa_ext_batch_policy. */
int  fa_ext_batch_learned(fa_ctx *ctx, const fa_params *p, const fa_policy *pol, const fa_band_model *model,
                          float margin, const fa_job *jobs, uint32_t n,
                          const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len,
                          const fa_band_hint *hints, fa_ext_result *out, int32_t *w_first_out,
                          int32_t *w_final, fa_ext_stats *stats);
/* Learned-band extension on 2-bit packed host buffers (fa_packed_seq above): same results,
 * bands and statistics as fa_ext_batch_learned on the same bases.  Batches of 32,768 jobs or
 * more whose jobs address their sequences at increasing offsets in job order run slice by
 * slice: each slice's job records, hints and bases go up on a copy stream while the slices
 * before it run features, prediction and every extension round on the device, and each
 * slice's results come back as soon as its rounds are done (into a pinned `out`). */
int  fa_ext_batch_learned_packed(fa_ctx *ctx, const fa_params *p, const fa_policy *pol,
                                 const fa_band_model *model, float margin, const fa_job *jobs, uint32_t n,
                                 const fa_packed_seq *qseq, const fa_packed_seq *tseq,
                                 const fa_band_hint *hints, fa_ext_result *out, int32_t *w_first_out,
                                 int32_t *w_final, fa_ext_stats *stats);

/* ---- paired-end batch (no reference counterpart) -------------------------
 * One submission of a paired-end batch's two kinds of work on one context: the seed
 * extensions of execute_batch_simd_scoring (src/pipelines/linear/batch_extension/
 * dispatch.rs:31-86) and the mate-rescue ksw_align2 jobs of
 * execute_mate_rescue_batch_with_engine (src/pipelines/linear/paired/mate_rescue.rs:595-685).
 * Both job sets go up at once; the mate SW kernels run on the context's mate stream while
 * the extension rounds -- fa_ext_batch_policy's, or fa_ext_batch_learned's when `model` is
 * given (pol must then be FA_POLICY_LEARNED) -- run on its main stream, so the GPU's block
 * scheduler works on both kinds of blocks at once; the call returns when both result sets are
 * back.  Results are those of the separate calls.  stats / mate_stats (may be NULL) get
 * each half's statistics and the call's wall time. */
int fa_pair_batch(fa_ctx *ctx, const fa_params *p, const fa_policy *pol, const fa_band_model *model, float margin,
                  const fa_job *jobs, uint32_t n, const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq,
                  uint64_t tseq_len, const fa_band_hint *hints, fa_ext_result *out, const fa_mate_params *mp,
                  const fa_mate_job *mjobs, uint32_t mn, const uint8_t *mqseq, uint64_t mqseq_len,
                  const uint8_t *mtseq, uint64_t mtseq_len, fa_kswr *mout, fa_ext_stats *stats,
                  fa_ext_stats *mate_stats);

/* Device-resident variant (no reference counterpart): device pointers, kernels
 * asynchronous on `stream` after one small synchronous read of the batch's job
 * counts and longest query/target; results at each job's own index.  Job ranges must
 * lie inside the sequence buffers (not checked); kernel-detected errors come back from
 * the next fa_ctx_sync(), the cell count of the last device call from
 * fa_ctx_last_cells().  With fa_ctx_set_timing on, fa_ctx_last_timing covers the SW
 * kernels. */
int fa_mate_sw_batch_device(fa_ctx *ctx, const fa_mate_params *p, const fa_mate_job *d_jobs, uint32_t n,
                            const uint8_t *d_qseq, const uint8_t *d_tseq, fa_kswr *d_out, void *stream);
int fa_ctx_last_cells(fa_ctx *ctx, unsigned long long *cells);

#ifdef __cplusplus
}
#endif
#endif /* FERROUS_B200_H */
