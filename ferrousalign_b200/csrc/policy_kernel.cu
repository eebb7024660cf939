// policy_kernel.cu -- device-side band-retry decisions between extension rounds.
//
// Plain policy (bwa-mem2 mem_chain2aln): try band w << k for k < max_tries; stop when
// the score equals the previous try's (initially 0 for a left extension, h0 for a
// right one) or max_off < (w>>1) + (w>>2).  The reference itself runs a single
// ksw_extend2 per job (src/pipelines/linear/batch_extension/dispatch.rs:31-86), which
// is the max_tries = 1 case.
//
// Learned policy: start at a predicted narrow band and double it while it is below
// the configured band.  A narrow run is accepted when its band clamp never bound
// (then every wider band reproduces it exactly), with FA_JUDGE_BOUND when its
// exit-bound certificate holds (it then equals the configured-band run, proven; see
// extend_kernel.cu) and that run would also end the plain ladder, or, with
// FA_JUDGE_MAXOFF (empirical, not exact), when it
// passes the bwa-mem2 max_off test (with FA_JUDGE_GLOBAL also requiring that its best
// score is its end-to-end score); otherwise the band doubles -- or goes straight to
// the configured band with FA_JUDGE_ONCE, or when only the end-to-end test failed --
// and at the configured band the plain policy takes over.
//
// The decisions compact the jobs that need another run into a list whose length
// stays on the device, so a retry round needs no host round trip.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

__global__ void policy_init_kernel(const fa_job *__restrict__ jobs, uint32_t n,
                                   const int32_t *__restrict__ w_first, int w_min, int learned,
                                   PolicyState st)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fa_job jb = jobs[i];
    int w = jb.w, k = 0;
    if (learned) {
        w = w_first ? w_first[i] : jb.w;
        if (w < w_min) w = w_min;
        if (w < jb.w) k = -1; else w = jb.w;
    }
    st.w_cur[i] = w;
    st.k[i] = k;
    st.prev[i] = jb.dir == FA_DIR_RIGHT ? jb.h0 : 0;
    st.w_final[i] = w;
    st.tries[i] = 0;
    if (st.missed) st.missed[i] = 0;
}

__global__ void policy_step_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ list,
                                   const uint32_t *__restrict__ first, const uint32_t *__restrict__ count,
                                   uint32_t n_max, const fa_ext_result *__restrict__ out,
                                   const uint8_t *__restrict__ clamped, PolicyState st, int max_tries,
                                   int judge, uint32_t *__restrict__ next, uint32_t *__restrict__ next_count)
{
    // list entries [*first, *count) (device-side bounds; 0 and n_max when null)
    const uint32_t t = (first ? *first : 0u) + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = count ? min(*count, n_max) : n_max;
    bool again = false;
    uint32_t jid = 0;
    if (t < n) {
        jid = list[t];
        const fa_job jb = jobs[jid];
        const fa_ext_result r = out[jid];
        int w = st.w_cur[jid], k = st.k[jid];
        st.tries[jid] += 1;
        st.w_final[jid] = w;
        if (k < 0) {   // learned narrow ladder
            const uint8_t fl = clamped[jid];   // bit 0: band clamp bound, bit 1: exit-bound certificate
            bool ok = !(fl & 1);
            if (!ok && (judge & FA_JUDGE_BOUND))
                // certified equal to the configured-band run, which the plain policy keeps
                ok = (fl & 2) && (r.score == st.prev[jid] || r.max_off < (jb.w >> 1) + (jb.w >> 2));
            bool jump = false;
            if (!ok && (judge & FA_JUDGE_MAXOFF)) {
                const bool off_ok = r.max_off < (w >> 1) + (w >> 2);
                const bool global = r.gscore == r.score;
                ok = off_ok && (!(judge & FA_JUDGE_GLOBAL) || global);
                // rejected only because the best score is not end-to-end: a wider
                // narrow band would not change that, so go to the configured band
                jump = off_ok && !ok;
            }
            if (!ok) {
                if (st.missed && st.tries[jid] == 1) st.missed[jid] = 1;
                const int hint = fl >> 2;
                int nw = 0;
                if (!jump && (judge & FA_JUDGE_BOUND) && (judge & FA_JUDGE_ONCE) && (judge & FA_JUDGE_HINT) &&
                    st.tries[jid] == 1 && hint < kBandHintNone) {
                    nw = w + hint;                      // up to the band ladder 2^k, 3*2^(k-1)
                    if (nw > 2) {
                        const int p2 = 1 << (32 - __clz(nw - 1));
                        nw = 3 * p2 / 4 >= nw ? 3 * p2 / 4 : p2;
                    }
                    if (2 * nw > jb.w) nw = 0;
                }
                if (nw > 0) {
                    w = nw;                             // one retry at the suggested band
                } else {
                    jump |= (judge & FA_JUDGE_ONCE) != 0;
                    w <<= 1;
                    if (jump || w >= jb.w) { w = jb.w; k = 0; }
                }
                st.w_cur[jid] = w;
                st.k[jid] = k;
                again = true;
            }
        } else {       // bwa-mem2 ladder at w << k
            const bool stop = r.score == st.prev[jid] || r.max_off < (w >> 1) + (w >> 2);
            if (!stop && k + 1 < max_tries) {
                st.prev[jid] = r.score;
                st.k[jid] = k + 1;
                st.w_cur[jid] = jb.w << (k + 1);
                again = true;
            }
        }
    }
    // warp-aggregated append to the next list
    const unsigned mask = __ballot_sync(0xffffffffu, again);
    if (mask) {
        const int lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == __ffs(mask) - 1) base = atomicAdd(next_count, (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
        if (again) next[base + __popc(mask & ((1u << lane) - 1u))] = jid;
    }
}

// Reorders a round's job list into band buckets so that every warp holds jobs of one
// band (a warp runs as long as its widest job): jobs at their configured band first,
// then narrow jobs by decreasing band, so the longest jobs start first and balance the
// end of the launch.  Order inside a bucket is the input list's (the longest-first order
// of the first round), so a warp's jobs also have similar lengths.  Three passes: per-block
// bucket counts, one block scanning them per bucket, then each job written at its bucket's
// base + its block's offset + its rank among the block's jobs of that bucket.
__device__ __forceinline__ int band_bucket(int w, int wj) {
    if (w >= wj) return 0;
    // descending narrow classes: >64, 49-64, 33-48, 25-32, 17-24, 13-16, 9-12, 7-8, 5-6, 4, 3, <=2
    constexpr int lo[kBandBuckets - 1] = {65, 49, 33, 25, 17, 13, 9, 7, 5, 4, 3, 0};
    int b = kBandBuckets - 1;
#pragma unroll
    for (int k = kBandBuckets - 2; k >= 0; --k)
        if (w >= lo[k]) b = k + 1;
    return b;
}

constexpr int kPartThreads = 256;

__device__ __forceinline__ int job_bucket(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ list,
                                          uint32_t t, uint32_t n, const int32_t *__restrict__ w_cur, uint32_t *jid) {
    if (t >= n) return -1;
    *jid = list[t];
    return band_bucket(w_cur[*jid], jobs[*jid].w);
}

__global__ void __launch_bounds__(kPartThreads)
band_count_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ list,
                  const uint32_t *__restrict__ count, uint32_t n_max, const int32_t *__restrict__ w_cur,
                  uint32_t *__restrict__ blk)
{
    __shared__ uint32_t cnt[kBandBuckets];
    if (threadIdx.x < kBandBuckets) cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t n = count ? min(*count, n_max) : n_max;
    uint32_t jid = 0;
    const int b = job_bucket(jobs, list, blockIdx.x * kPartThreads + threadIdx.x, n, w_cur, &jid);
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    if (b >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&cnt[b], (uint32_t)__popc(peers));
    __syncthreads();
    if (threadIdx.x < kBandBuckets) blk[blockIdx.x * kBandBuckets + threadIdx.x] = cnt[threadIdx.x];
}

// one warp per bucket: the per-block counts become exclusive offsets inside the bucket;
// base[b] = the bucket's first slot, and the band-group bounds
__global__ void __launch_bounds__(32 * kBandBuckets)
band_scan_kernel(uint32_t *__restrict__ blk, uint32_t nblk, uint32_t *__restrict__ base,
                 uint32_t *__restrict__ bounds)
{
    __shared__ uint32_t tot[kBandBuckets];
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t run = 0;
    for (uint32_t i0 = 0; i0 < nblk; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t v = i < nblk ? blk[i * kBandBuckets + k] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (i < nblk) blk[i * kBandBuckets + k] = run + x - v;
        run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) tot[k] = run;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0, bs[kBandBuckets];
        for (int q = 0; q < kBandBuckets; ++q) { bs[q] = acc; base[q] = acc; acc += tot[q]; }
        if (bounds) {
            // band groups: buckets 0-4 (configured band, bands > 24), 5-6 (13-24), 7-12 (<= 12);
            // bounds[3]: the end of bucket 0 (the jobs at their configured band)
            bounds[0] = bs[5];
            bounds[1] = bs[7];
            bounds[2] = acc;
            bounds[3] = bs[1];
        }
    }
}

__global__ void __launch_bounds__(kPartThreads)
band_place_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ list,
                  const uint32_t *__restrict__ count, uint32_t n_max, const int32_t *__restrict__ w_cur,
                  const uint32_t *__restrict__ blk, const uint32_t *__restrict__ base, uint32_t *__restrict__ out)
{
    constexpr int W = kPartThreads / 32;
    __shared__ uint32_t wcnt[W][kBandBuckets];
    for (int i = threadIdx.x; i < W * kBandBuckets; i += kPartThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t n = count ? min(*count, n_max) : n_max;
    uint32_t jid = 0;
    const int b = job_bucket(jobs, list, blockIdx.x * kPartThreads + threadIdx.x, n, w_cur, &jid);
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (b >= 0 && lane == __ffs(peers) - 1) wcnt[w][b] = (uint32_t)__popc(peers);
    __syncthreads();
    if (b < 0) return;
    uint32_t pos = base[b] + blk[blockIdx.x * kBandBuckets + b] + __popc(peers & ((1u << lane) - 1u));
    for (int v = 0; v < w; ++v) pos += wcnt[v][b];
    out[pos] = jid;
}

size_t band_partition_scratch_words(uint32_t n_max) {
    return (size_t)((n_max + kPartThreads - 1) / kPartThreads) * kBandBuckets;
}

cudaError_t launch_band_partition(const fa_job *d_jobs, const uint32_t *d_list, const uint32_t *d_count,
                                  uint32_t n_max, const int32_t *d_w_cur, uint32_t *d_out, uint32_t *d_base,
                                  uint32_t *d_blk, uint32_t *d_bounds, cudaStream_t stream)
{
    if (n_max == 0) return cudaSuccess;
    const uint32_t blocks = (n_max + kPartThreads - 1) / kPartThreads;
    band_count_kernel<<<blocks, kPartThreads, 0, stream>>>(d_jobs, d_list, d_count, n_max, d_w_cur, d_blk);
    band_scan_kernel<<<1, 32 * kBandBuckets, 0, stream>>>(d_blk, blocks, d_base, d_bounds);
    band_place_kernel<<<blocks, kPartThreads, 0, stream>>>(d_jobs, d_list, d_count, n_max, d_w_cur, d_blk, d_base,
                                                           d_out);
    return cudaGetLastError();
}

// A batch's statistics summed on the device: sums = {cells of the accepted runs, runs per
// job (tries, when given), missed narrow tries (when given)}, so a call reads back three words
// instead of its per-job arrays.
__global__ void __launch_bounds__(256) stats_sum_kernel(const uint32_t *__restrict__ cells_job,
                                                        const int32_t *__restrict__ tries,
                                                        const uint8_t *__restrict__ missed, uint32_t n,
                                                        unsigned long long *__restrict__ sums)
{
    unsigned long long v[3] = {0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        v[0] += cells_job[i];
        if (tries) v[1] += (uint32_t)tries[i];
        if (missed) v[2] += missed[i];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if ((threadIdx.x & 31) == 0 && v[k]) atomicAdd(&sums[k], v[k]);
    }
}

cudaError_t launch_stats_sum(const uint32_t *d_cells_job, const int32_t *d_tries, const uint8_t *d_missed, uint32_t n,
                             unsigned long long *d_sums, int sm_count, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(d_sums, 0, 3 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess || n == 0) return e;
    uint32_t blocks = (n + 255) / 256;
    if (blocks > (uint32_t)sm_count * 8) blocks = sm_count * 8;
    stats_sum_kernel<<<blocks, 256, 0, stream>>>(d_cells_job, d_tries, d_missed, n, d_sums);
    return cudaGetLastError();
}

// Appends src[0 .. *d_end) (a device-side count, at most n_max) to dst at the positions an
// atomic counter hands out, one claim per warp; the order inside dst is not kept.
__global__ void __launch_bounds__(256) list_append_kernel(const uint32_t *__restrict__ src,
                                                          const uint32_t *__restrict__ d_end, uint32_t n_max,
                                                          uint32_t *__restrict__ dst, uint32_t *__restrict__ dst_count)
{
    const uint32_t n = min(*d_end, n_max);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(dst_count, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (live) dst[base + __popc(mask & ((1u << lane) - 1u))] = src[i];
}

cudaError_t launch_list_append(const uint32_t *d_src, const uint32_t *d_end, uint32_t n_max, uint32_t *d_dst,
                               uint32_t *d_dst_count, cudaStream_t stream)
{
    if (n_max == 0) return cudaSuccess;
    list_append_kernel<<<(n_max + 255) / 256, 256, 0, stream>>>(d_src, d_end, n_max, d_dst, d_dst_count);
    return cudaGetLastError();
}

// One thread per N run of a packed buffer: ST_RUNS when the run is empty, reaches past the
// buffer's bases or starts before the previous run's end.
__global__ void __launch_bounds__(256) runs_check_kernel(const fa_nrun *__restrict__ runs, uint32_t n,
                                                         uint64_t n_bases, uint32_t *__restrict__ status)
{
    const uint32_t k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const fa_nrun r = runs[k];
    bool bad = r.len == 0 || r.pos > n_bases || r.len > n_bases - r.pos;
    if (k > 0) {
        const fa_nrun q = runs[k - 1];
        bad = bad || r.pos < q.pos + q.len;
    }
    if (bad) atomicOr(status, ST_RUNS);
}

cudaError_t launch_runs_check(const fa_nrun *d_runs, uint32_t n, uint64_t n_bases, uint32_t *d_status,
                              cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    runs_check_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_runs, n, n_bases, d_status);
    return cudaGetLastError();
}

cudaError_t launch_policy_init(const fa_job *d_jobs, uint32_t n, const int32_t *d_w_first, int w_min,
                               int learned, PolicyState st, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    policy_init_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_jobs, n, d_w_first, w_min, learned, st);
    return cudaGetLastError();
}

cudaError_t launch_policy_step(const fa_job *d_jobs, const uint32_t *d_list, const uint32_t *d_first,
                               const uint32_t *d_count, uint32_t n_max, const fa_ext_result *d_out,
                               const uint8_t *d_clamped, PolicyState st, int max_tries, int judge,
                               uint32_t *d_next, uint32_t *d_next_count, cudaStream_t stream)
{
    if (n_max == 0) return cudaSuccess;
    policy_step_kernel<<<(n_max + 255) / 256, 256, 0, stream>>>(d_jobs, d_list, d_first, d_count, n_max, d_out,
                                                               d_clamped, st, max_tries, judge, d_next,
                                                               d_next_count);
    return cudaGetLastError();
}

}  // namespace fa
