// fa_kernels.h -- internal launcher declarations (C++ linkage, not part of the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <vector>

#include "fa_device.cuh"
#include "fa_packed.cuh"

namespace fa {

constexpr int kExtThreads = 128;     // threads (= jobs) per extension block
constexpr int kPackedHMax = 8191;    // largest H/E the packed column word holds
constexpr int kBandHintNone = 63;    // flags bits 2-7: no band suggested by the certificate
constexpr int kBandBuckets = 13;   // configured band + 12 narrow band classes
constexpr int kPairThreads = 32;     // threads per int16x2 extension block (2 jobs each)

size_t ext_packed_smem_bytes(int qcap, int ring, int tpb);
cudaError_t launch_ext_packed(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n,
                              const uint32_t *d_first, const uint32_t *d_n, const SeqBuf &d_qseq,
                              const SeqBuf &d_tseq, const ExtParams &p, int qcap, int ring,
                              const int32_t *d_w_try, fa_ext_result *d_out, uint8_t *d_clamped, bool cert,
                              uint32_t *d_cells_job, unsigned long long *d_cells, uint32_t *d_status,
                              cudaStream_t stream, int tpb = kExtThreads);

// int16x2 variant: two jobs per thread (extend_pair_kernel.cu).  Eligible for
// bwa-form scoring matrices; same arguments and results as launch_ext_packed.
bool ext_pair_eligible(const ExtParams &p);
size_t ext_pair_smem_bytes(int qcap);
// Byte-code sequences only (cudaErrorNotSupported for packed ones).
cudaError_t launch_ext_pair(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n, const uint32_t *d_n,
                            const SeqBuf &d_qseq, const SeqBuf &d_tseq, const ExtParams &p, int qcap,
                            const int32_t *d_w_try,
                            fa_ext_result *d_out, uint8_t *d_clamped, uint32_t *d_cells_job,
                            unsigned long long *d_cells, uint32_t *d_status, cudaStream_t stream);

// Two target rows per thread in int16x2 cells with 8-bit column state (extend_rows2_kernel.cu).
// Eligible for bwa-form matrices (any capacity whose shared memory fits); jobs whose scores
// can pass 255 -- every job past 254 query columns among them -- are appended to d_ovf (count
// in *d_ovf_n) and run by the int32 kernel in the same call with the same settings.  ring
// 32/64 keeps only that many column words (bands with 2w + 3 <= ring); cert evaluates the
// exit-bound certificate and hint into d_clamped.
// d_first (optional): device-side first index into d_order, as for launch_ext_packed.
// d_work (optional): a device counter that makes the launch persistent, warps claiming 32
// jobs at a time until the order (from d_first on) is used up.
// ovf_stream / ovf_ev (optional): the int32 pass runs on ovf_stream (forked by ovf_ev) and the
// caller joins ovf_stream back before anything reads the results.  ovf_early: its jobs are
// listed first (a short kernel on `stream`) and the pass starts at once while the two-row
// launch skips them -- for launches joined right after, where the longest jobs then overlap
// the two-row work; otherwise the pass follows the two-row launch as usual and only the work
// after it on `stream` overlaps (a persistent two-row launch that shares the GPU with an
// early pass cannot finish before that pass frees its slots).
bool ext_rows2_eligible(const ExtParams &p, int qcap);
size_t ext_rows2_smem_bytes(int qcap, int tpb, int ring);
cudaError_t launch_ext_rows2(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n, const uint32_t *d_first,
                             const uint32_t *d_n, const SeqBuf &d_qseq, const SeqBuf &d_tseq, const ExtParams &p,
                             int qcap, int ring, bool cert, const int32_t *d_w_try, fa_ext_result *d_out,
                             uint8_t *d_clamped, uint32_t *d_cells_job, unsigned long long *d_cells,
                             uint32_t *d_status, uint32_t *d_ovf, uint32_t *d_ovf_n, cudaStream_t stream, int tpb,
                             uint32_t *d_work = nullptr, cudaStream_t ovf_stream = nullptr,
                             cudaEvent_t ovf_ev = nullptr, bool ovf_early = true);
// Queries past this many columns always take the two-row kernel's overflow path (8-bit
// column words: h0 >= 1 and a >= 1 leave qlen <= 254).
constexpr int kRows2MaxQ = 254;

// Band-retry policy step over the jobs of the last extension round (see policy_kernel.cu).
struct PolicyState {
    int32_t *w_cur;      // band of the run just finished / next run
    int32_t *prev;       // previous try's score (bwa-mem2 break rule)
    int32_t *k;          // bwa try index; -1 while on the learned narrow ladder
    int32_t *w_final;    // band of the accepted run
    int32_t *tries;      // runs per job
    uint8_t *missed;     // learned path: first narrow run not accepted
};
cudaError_t launch_policy_step(const fa_job *d_jobs, const uint32_t *d_list, const uint32_t *d_first,
                               const uint32_t *d_count, uint32_t n_max, const fa_ext_result *d_out,
                               const uint8_t *d_clamped, PolicyState st, int max_tries, int judge,
                               uint32_t *d_next, uint32_t *d_next_count, cudaStream_t stream);
// The list reordered into band buckets (the input order kept inside a bucket): d_base gets
// the kBandBuckets bucket starts, d_bounds (may be null) the band-group bounds; d_blk is
// scratch of band_partition_scratch_words(n_max) words.
cudaError_t launch_band_partition(const fa_job *d_jobs, const uint32_t *d_list, const uint32_t *d_count,
                                  uint32_t n_max, const int32_t *d_w_cur, uint32_t *d_out, uint32_t *d_base,
                                  uint32_t *d_blk, uint32_t *d_bounds, cudaStream_t stream);
size_t band_partition_scratch_words(uint32_t n_max);
// dst[atomic positions] = src[0 .. *d_end), *d_end <= n_max (a device-side count)
cudaError_t launch_list_append(const uint32_t *d_src, const uint32_t *d_end, uint32_t n_max, uint32_t *d_dst,
                               uint32_t *d_dst_count, cudaStream_t stream);
// ST_RUNS into *d_status when a packed buffer's N runs are not sorted, disjoint, non-empty
// runs inside its n_bases bases
cudaError_t launch_runs_check(const fa_nrun *d_runs, uint32_t n, uint64_t n_bases, uint32_t *d_status,
                              cudaStream_t stream);
// sums[0..2] = {sum of cells_job, sum of tries (d_tries may be NULL), sum of missed (may be NULL)}
cudaError_t launch_stats_sum(const uint32_t *d_cells_job, const int32_t *d_tries, const uint8_t *d_missed, uint32_t n,
                             unsigned long long *d_sums, int sm_count, cudaStream_t stream);
cudaError_t launch_policy_init(const fa_job *d_jobs, uint32_t n, const int32_t *d_w_first, int w_min,
                               int learned, PolicyState st, cudaStream_t stream);

// Byte codes to 2-bit packed bases (pack_kernel.cu): d_dst gets (n + 3) / 4 bytes, written as
// whole 32-bit words (room for ceil(n / 16) words); d_src 16-byte aligned and readable up to
// a multiple of 16 bytes past n.
cudaError_t launch_pack2(const uint8_t *d_src, uint64_t n, uint8_t *d_dst, cudaStream_t s);
// The N (code 4) runs of n byte codes, sorted: at most cap written to d_runs; the count at
// d_scratch[pack_runs_scratch_words(n) - 1] after the launches (d_scratch: that many words).
cudaError_t launch_nruns(const uint8_t *d_src, uint64_t n, fa_nrun *d_runs, uint64_t cap, uint32_t *d_scratch,
                         cudaStream_t s);
size_t pack_runs_scratch_words(uint64_t n);
// 2-bit packed bases (16-byte readable past (n + 3) / 4, word aligned) to n byte codes with
// the N runs applied; d_dst 16-byte aligned with room for a multiple of 16 bytes past n.
cudaError_t launch_unpack2(const uint8_t *d_src, uint64_t n, const fa_nrun *d_runs, uint32_t n_runs, uint8_t *d_dst,
                           cudaStream_t s);
// positions [p0, p1) only (p0 a multiple of 16; whole 16-base words are written, so p1 is a
// multiple of 16 or the buffer's end), the N runs' bases inside the range back to code 4
cudaError_t launch_unpack2_range(const uint8_t *d_src, uint64_t p0, uint64_t p1, const fa_nrun *d_runs,
                                 uint32_t n_runs, uint8_t *d_dst, cudaStream_t s);

// Mate-rescue local SW.  `byte_lanes` selects the u8 (16-lane) or i16 (8-lane)
// emulation of the reference's striped kernels; d_order lists the jobs of that kind.
// d_rev (2 + n words; needed for u8 jobs, unused for i16 jobs): the list of KSW_XSTART
// reverse passes that a second kernel runs after the forward passes.
// min_qlen: the shortest query of the launch's jobs (u8 jobs whose segment counts all equal
// the register depth run a form without per-segment range checks).
cudaError_t launch_mate_sw(bool byte_lanes, const fa_mate_job *d_jobs, const uint32_t *d_order,
                           uint32_t n, const uint8_t *d_qseq, const uint8_t *d_tseq,
                           const MateParams &p, int min_qlen, int max_qlen, int max_tlen, fa_kswr *d_out,
                           unsigned long long *d_cells, uint32_t *d_status, uint32_t *d_rev,
                           cudaStream_t stream);

// Device-side longest-first ordering by query length (order_kernel.cu).
// Pipelined host batches: validation + (chunk, length) histogram + prefix, then scatter.
// Scratch layout: hist | base | cursor (nchunks * (FA_MAX_QLEN+1) each) | info[4] =
// {status bits, first bad job, longest query, widest configured band} | bounds[nchunks+1] |
// each chunk's lowest and highest job index.  A job belongs to the chunk that holds the
// last byte of its query or of its target, whichever comes later; chunk k of a buffer ends
// at byte end[k] (exclusive; the last end is the buffer's length).  shift: log2 of the
// positions per byte (0 for byte codes, 2 for packed bases); qbytes / tbytes of the prep
// are then the buffers' lengths in positions.
constexpr int kMaxChunks = 8;
struct ChunkEnds {
    uint64_t q[kMaxChunks], t[kMaxChunks];
    int shift;
};
size_t chunk_scratch_bytes(int nchunks);
// h0_min: the smallest valid h0 (1, or 0 with FA_PARAM_H0_ZERO)
cudaError_t launch_chunk_prep(const fa_job *d_jobs, uint32_t n, uint64_t qbytes, uint64_t tbytes, const ChunkEnds &ends,
                              int nchunks, int max_score, int h0_min, int qcap_limit, uint32_t *d_scratch,
                              cudaStream_t s);
cudaError_t launch_chunk_scatter(const fa_job *d_jobs, uint32_t n, const ChunkEnds &ends, int nchunks,
                                 uint32_t *d_scratch, uint32_t *d_order, cudaStream_t s);
// Streamed host batches (order_kernel.cu): one slice of jobs validated against the whole
// buffers (qpos / tpos positions) and the slice's resident ends (q_res / t_res), the valid
// resident jobs ordered longest query first into d_order (local indices).  Scratch of
// slice_scratch_words(1) words; its last 8 words: {status, first bad job, longest query,
// widest band, 0, listed jobs, jobs not resident, 0}.
size_t slice_scratch_words(int nslices);
constexpr int kSliceInfoWords = 8;
cudaError_t launch_slice_prep(const fa_job *d_jobs, uint32_t n, uint64_t qpos, uint64_t tpos, uint64_t q_res,
                              uint64_t t_res, int max_score, int h0_min, int qcap_limit, uint32_t *d_scratch,
                              uint32_t *d_order, cudaStream_t s);
cudaError_t launch_qlen_hist(const fa_job *d_jobs, uint32_t n, uint32_t *d_hist, int sm_count, cudaStream_t s);
cudaError_t launch_qlen_scatter(const fa_job *d_jobs, uint32_t n, uint32_t *d_cursor, uint32_t *d_order,
                                cudaStream_t s);

// Learned band predictor (band_model.cu).
// Device copies of the query / target byte arrays are allocated kSeqPad bytes longer than
// their contents, so readers of aligned 32-bit words never leave the allocation.
constexpr uint64_t kSeqPad = 16;
// d_order (optional): a permutation of the n jobs (the batch's length order), taken in turn by
// the threads; the features stay indexed by job.
cudaError_t launch_band_features(const fa_job *d_jobs, uint32_t n, const SeqBuf &d_q, const SeqBuf &d_t,
                                 const fa_band_hint *d_hints, int max_score, float *d_x, cudaStream_t s,
                                 const uint32_t *d_order = nullptr);
cudaError_t launch_band_predict(const __nv_bfloat16 *d_wbf, const float *mean, const float *std_, const float *d_x,
                                const fa_job *d_jobs, uint32_t n, float margin, int w_min, float *d_y,
                                int32_t *d_w, cudaStream_t s);
cudaError_t launch_band_backward(const __nv_bfloat16 *d_wbf, const float *mean, const float *std_, const float *d_x,
                                 const float *d_target, uint32_t n, float tau, float inv_total, float *d_grad,
                                 float *d_loss, cudaStream_t s);
cudaError_t launch_band_adam(float *d_w, __nv_bfloat16 *d_wbf, float *d_m, float *d_v, const float *d_grad, float lr,
                             int step, cudaStream_t s);
// BF16 weights and normalisation of a model, for device-side prediction (band_api.cu).
void band_model_export(const fa_band_model *m, std::vector<__nv_bfloat16> &wbf, float *mean, float *std_);
// Device of a context (fa_api.cu).
int fa_ctx_device(const fa_ctx *ctx);

// Records the calling thread's fa_last_error() message and returns `code` (fa_api.cu).
int set_last_error(int code, const char *msg);

// Mate-rescue jobs split by lane width into two order lists; info (8 words) =
// {n_byte, n_word, max_q_byte, max_q_word, max_t, bad_lengths, 0xFFFFFFFF - min_q_byte, -}.
cudaError_t launch_mate_split(const fa_mate_job *d_jobs, uint32_t n, uint32_t *d_order_b, uint32_t *d_order_w,
                              uint32_t *d_info, cudaStream_t s);

// Alignment regions from left/right extension results, one thread per chain (region_kernel.cu).
cudaError_t launch_merge_regions(const fa_region_opts &opt, const uint32_t *d_chain_first, uint32_t n_chains,
                                 const int32_t *d_query_len, const fa_seed_ext *d_seeds, uint32_t n_seeds,
                                 const fa_ext_result *d_left, uint32_t n_left, const fa_ext_result *d_right,
                                 uint32_t n_right, fa_region *d_out, uint32_t *d_status, cudaStream_t s);

// Extension jobs from chains and a packed reference (collect_kernel.cu).  Per chain: its
// window [r0, r1), counters v = {window bytes (forward + reversed), left jobs, right jobs,
// seed-table entries} and their exclusive prefix sums off over the chains.
struct CollectPlan {
    uint64_t r0, r1;
    unsigned long long v[4];
    unsigned long long off[4];
};
int collect_max_gap(const fa_collect_opts &o, int qlen);
size_t collect_scan_blocks(uint32_t n_chains);   // entries of the scan's block-sum array, less one
// argument check + plan + scan; d_sums holds collect_scan_blocks(n) + 1 entries, the last one
// the totals; d_bad[2]: the first failing read and chain as index << 8 | code (all ones: none;
// codes in collect_kernel.cu), known before any plan is used
cudaError_t launch_collect_plan(const fa_collect_opts &opt, uint64_t l_pac, const uint64_t *d_read_off,
                                uint32_t n_reads, const fa_chain *d_chains, uint32_t n_chains, const fa_seed *d_seeds,
                                uint32_t n_seeds, CollectPlan *d_plan, ulonglong4 *d_sums, unsigned long long *d_bad,
                                cudaStream_t s);
// the scan alone: plan[i].off = exclusive prefix sums of plan[].v; d_sums[collect_scan_blocks(n)]
// gets the totals
cudaError_t launch_plan_scan(CollectPlan *d_plan, uint32_t n, ulonglong4 *d_sums, cudaStream_t s);
cudaError_t launch_collect_fill(const fa_collect_opts &opt, const uint8_t *d_pac, uint64_t l_pac,
                                const uint8_t *d_reads, const uint64_t *d_read_off, uint32_t n_reads,
                                const fa_chain *d_chains, uint32_t n_chains, const fa_seed *d_seeds,
                                const CollectPlan *d_plan, fa_job *d_left, fa_job *d_right, uint8_t *d_qbuf,
                                uint8_t *d_tbuf, fa_seed_ext *d_seed_ext, uint32_t *d_chain_first,
                                uint64_t *d_chain_win, cudaStream_t s);

// Mate-rescue jobs (mate_collect_kernel.cu): per attempt a plan (v = {target bytes, jobs,
// query bytes, 0}), scanned with launch_plan_scan, then the fill.
struct RescueRef {
    uint64_t l_pac;
    const uint8_t *pac;
    const uint64_t *chr_off, *chr_len;
    uint32_t n_chr;
};
cudaError_t launch_mate_collect_plan(const fa_rescue_opts &opt, const fa_insert_bounds *bounds4, RescueRef ref,
                                     const uint64_t *d_read_off, const fa_rescue_aln *d_alns,
                                     const fa_rescue_cand *d_cands, uint32_t n_cand, CollectPlan *d_plan,
                                     cudaStream_t s);
cudaError_t launch_mate_collect_fill(const fa_rescue_opts &opt, const fa_insert_bounds *bounds4, RescueRef ref,
                                     const uint8_t *d_reads, const uint64_t *d_read_off, const fa_rescue_aln *d_alns,
                                     const fa_rescue_cand *d_cands, uint32_t n_cand, const CollectPlan *d_plan,
                                     fa_mate_job *d_jobs, fa_rescue_job_info *d_info, uint8_t *d_qbuf,
                                     uint8_t *d_tbuf, cudaStream_t s);

// Insert-size statistics (insert_size_kernel.cu): d_hist holds insert_hist_bytes().
size_t insert_hist_bytes();
cudaError_t launch_insert_stats(int64_t l_pac, const int64_t *d_pairs, uint32_t n, uint32_t *d_hist,
                                fa_insert_stats *d_out, cudaStream_t s);

// CIGAR regeneration (cigar_kernel.cu): per job the offsets of its outputs (cigar words,
// aligned reference / query bases) and of its scratch (row state in int2 units, traceback
// in words), and its traceback words per row.
struct CigarPlan {
    uint64_t cig, ref, qry, eh, tb;
    int32_t wpr, _pad;
};
int cigar_band_words(int qlen, int w);
cudaError_t launch_cigar(const fa_cigar_job *d_jobs, const CigarPlan *d_plan, uint32_t n, const uint8_t *d_qseq,
                         const uint8_t *d_tseq, const ExtParams &p, int pen_clip3, int2 *d_eh, uint32_t *d_tb,
                         fa_cigar_result *d_out, uint32_t *d_cigar, uint8_t *d_ref_al, uint8_t *d_qry_al,
                         cudaStream_t s);
// The same with the row state in shared memory as 16-bit pairs: every job's qlen <= qcap <=
// cigar_smem_qcap() and h0 + qlen * max(mat) <= 32767; jobs run in d_order.  qwords: the
// words also carry the query codes (13-bit H and E: h0 + qlen * max(mat) <= 8191).
cudaError_t launch_cigar_smem(const fa_cigar_job *d_jobs, const CigarPlan *d_plan, const uint32_t *d_order,
                              uint32_t n, int qcap, bool qwords, const uint8_t *d_qseq, const uint8_t *d_tseq,
                              const ExtParams &p, int pen_clip3, uint32_t *d_tb, fa_cigar_result *d_out,
                              uint32_t *d_cigar, uint8_t *d_ref_al, uint8_t *d_qry_al, cudaStream_t s);
int cigar_smem_qcap();
// job k's n_cigar words from its slot at plan[k].cig to d_packed[d_first[k]]
cudaError_t launch_cigar_pack(const CigarPlan *d_plan, const fa_cigar_result *d_res, const uint64_t *d_first,
                              uint32_t n, const uint32_t *d_cigar, uint32_t *d_packed, cudaStream_t s);

// Integer / DPX instruction throughput (ops per second) for the roofline denominator.
double probe_int_peak(int kind, int sm_count, cudaStream_t s, float *ms_out);

}  // namespace fa
