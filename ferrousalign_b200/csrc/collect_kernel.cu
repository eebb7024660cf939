// collect_kernel.cu -- extension jobs from chains and a 2-bit packed reference (sm_100a).
//
// collect_extension_jobs_batch_soa (src/pipelines/linear/batch_extension/collect_soa.rs:28-230):
// per kept chain with seeds, the reference window its seeds can reach (cal_max_gap margins,
// chaining.rs:1108-1116, kept on the strand of the chain's first seed), read out of the
// packed reference (bntseq.rs:451-535, 564-575: two bits per base, first base in the high
// bits; the reverse strand [l_pac, 2 l_pac) is the reverse complement of the forward one),
// and per seed, last to first, a left job (the reversed read prefix against the reversed
// window before the seed, h0 = len * a) and a right job (the read suffix against the window
// after the seed, h0 = 0).  Instead of copying sequences per job, every read is written
// once forward and once reversed, every window once forward and once reversed, and each job
// addresses a slice of them.
//
// Launches: a plan per chain (window, job counts), a three-pass exclusive scan of the plans
// (block sums, one block over the sums, block-local scans plus the sums), then the windows
// (one warp per chain, lanes on consecutive bases), the reads (one warp per read) and the
// jobs with the seed table (one thread per chain).

#include <climits>

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

// cal_max_gap (chaining.rs:1108-1116) in integers: (int)((double)x / e + 1.0) is
// trunc((x + e) / e) for e != 0; x / 0.0 + 1 is +inf, -inf or NaN, which Rust's `as i32`
// turns into INT_MAX, INT_MIN or 0.
__host__ __device__ __forceinline__ int collect_gap_part(int x, int e) {
    if (e == 0) return x > 0 ? INT_MAX : (x < 0 ? INT_MIN : 0);
    return (int)(((long long)x + e) / e);
}

__host__ __device__ __forceinline__ int max_gap(const fa_collect_opts &o, int qlen) {
    const int l_del = collect_gap_part(qlen * o.a - o.o_del, o.e_del);
    const int l_ins = collect_gap_part(qlen * o.a - o.o_ins, o.e_ins);
    int l = l_del > l_ins ? l_del : l_ins;
    l = l > 1 ? l : 1;
    return l < (o.w << 1) ? l : (o.w << 1);
}

namespace {

constexpr int kCollectThreads = 128;
constexpr int kScanThreads = 1024;

// The argument rules the reference's slices and windows would panic on
// (collect_soa.rs:150-209), one thread per read and per chain.  bad[0] gets the smallest
// r << 8 | code over failing reads, bad[1] the smallest k << 8 | code over failing chains --
// a chain's code is its first failure in the order the rules are listed: the first failing
// read, else the first failing chain, is the one a serial check reports.  Codes: 1 read
// offsets not ascending, 2 read too long, 3 read index out of range, 4 seeds past the seed
// array, 5 a seed outside its read, 6 a seed outside the reference.
__global__ void __launch_bounds__(kCollectThreads)
collect_check_kernel(uint64_t l_pac, const uint64_t *__restrict__ read_off, uint32_t n_reads,
                     const fa_chain *__restrict__ chains, uint32_t n_chains, const fa_seed *__restrict__ seeds,
                     uint32_t n_seeds, unsigned long long *__restrict__ bad)
{
    const uint32_t i = blockIdx.x * kCollectThreads + threadIdx.x;
    if (i < n_reads) {
        const uint64_t a = read_off[i], b = read_off[i + 1];
        const int code = b < a ? 1 : (b - a > (uint64_t)INT32_MAX ? 2 : 0);
        if (code) atomicMin(&bad[0], (unsigned long long)i << 8 | code);
    }
    if (i < n_chains) {
        const fa_chain ch = chains[i];
        int code = 0;
        if (ch.read >= n_reads) {
            code = 3;
        } else if ((uint64_t)ch.seed_first + ch.n_seeds > n_seeds) {
            code = 4;
        } else if (ch.kept) {
            const int64_t qlen = (int64_t)(read_off[ch.read + 1] - read_off[ch.read]);
            for (uint32_t k = 0; k < ch.n_seeds && !code; ++k) {
                const fa_seed sd = seeds[ch.seed_first + k];
                if (sd.query_pos < 0 || sd.len < 0 || (int64_t)sd.query_pos + sd.len > qlen) code = 5;
                else if (sd.ref_pos >= (l_pac << 1) || sd.ref_pos + (uint64_t)sd.len > (l_pac << 1)) code = 6;
            }
        }
        if (code) atomicMin(&bad[1], (unsigned long long)i << 8 | code);
    }
}

// A chain whose read or seed range is out of bounds plans nothing (the check above fails
// the call before anything reads its plan).
__global__ void __launch_bounds__(kCollectThreads)
collect_plan_kernel(fa_collect_opts opt, uint64_t l_pac, const uint64_t *__restrict__ read_off, uint32_t n_reads,
                    const fa_chain *__restrict__ chains, uint32_t n_chains, const fa_seed *__restrict__ seeds,
                    uint32_t n_seeds, CollectPlan *__restrict__ plan)
{
    const uint32_t c = blockIdx.x * kCollectThreads + threadIdx.x;
    if (c >= n_chains) return;
    const fa_chain ch = chains[c];
    CollectPlan pl{};
    if (ch.kept != 0 && ch.n_seeds > 0 && ch.read < n_reads && (uint64_t)ch.seed_first + ch.n_seeds <= n_seeds) {
        const int qlen = (int)(read_off[ch.read + 1] - read_off[ch.read]);
        // collect_soa.rs:97-122: the window every seed's extensions can reach
        uint64_t r0 = l_pac << 1, r1 = 0;
        for (uint32_t k = 0; k < ch.n_seeds; ++k) {
            const fa_seed s = seeds[ch.seed_first + k];
            const int lm = s.query_pos + max_gap(opt, s.query_pos);
            const uint64_t b = s.ref_pos >= (uint64_t)(int64_t)lm ? s.ref_pos - (uint64_t)(int64_t)lm : 0u;
            const int rem = qlen - s.query_pos - s.len;
            const int rm = rem + max_gap(opt, rem);
            const uint64_t e = s.ref_pos + (uint64_t)(int64_t)s.len + (uint64_t)(int64_t)rm;
            r0 = b < r0 ? b : r0;
            r1 = e > r1 ? e : r1;
        }
        r1 = r1 < (l_pac << 1) ? r1 : (l_pac << 1);
        if (r0 < l_pac && l_pac < r1) {   // keep the window on the first seed's strand
            if (seeds[ch.seed_first].ref_pos < l_pac) r1 = l_pac;
            else r0 = l_pac;
        }
        const uint64_t L = r1 > r0 ? r1 - r0 : 0u;
        pl.r0 = r0;
        pl.r1 = r1;
        pl.v[0] = 2 * L;
        pl.v[3] = ch.n_seeds;
        for (uint32_t k = 0; k < ch.n_seeds; ++k) {   // collect_soa.rs:144-209 job conditions
            const fa_seed s = seeds[ch.seed_first + k];
            if (s.query_pos > 0) {
                const uint64_t tmp = s.ref_pos - r0;
                if (tmp > 0 && tmp <= L) ++pl.v[1];
            }
            if (s.query_pos + s.len < qlen && s.ref_pos + (uint64_t)(int64_t)s.len - r0 < L) ++pl.v[2];
        }
    }
    plan[c] = pl;
}

// exclusive scan of the plans' four counters: block sums
__global__ void __launch_bounds__(kScanThreads)
collect_scan_sums_kernel(const CollectPlan *__restrict__ plan, uint32_t n, ulonglong4 *__restrict__ sums)
{
    __shared__ unsigned long long red[4][kScanThreads / 32];
    const uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
    unsigned long long v[4] = {0, 0, 0, 0};
    if (i < n)
        for (int f = 0; f < 4; ++f) v[f] = plan[i].v[f];
    for (int f = 0; f < 4; ++f) {
        for (int o = 16; o > 0; o >>= 1) v[f] += __shfl_down_sync(0xffffffffu, v[f], o);
        if ((threadIdx.x & 31) == 0) red[f][threadIdx.x >> 5] = v[f];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        for (int f = 0; f < 4; ++f) {
            unsigned long long x = red[f][threadIdx.x];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[f] = x;
        }
        if (threadIdx.x == 0) sums[blockIdx.x] = make_ulonglong4(v[0], v[1], v[2], v[3]);
    }
}

// exclusive scan of the block sums in place (one block, chunks of kScanThreads); the grand
// totals go to sums[nb]
__global__ void __launch_bounds__(kScanThreads)
collect_scan_top_kernel(ulonglong4 *__restrict__ sums, uint32_t nb)
{
    __shared__ unsigned long long wsum[4][kScanThreads / 32];
    unsigned long long carry[4] = {0, 0, 0, 0};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nb; base += kScanThreads) {
        const uint32_t i = base + threadIdx.x;
        const ulonglong4 s = i < nb ? sums[i] : make_ulonglong4(0, 0, 0, 0);
        unsigned long long x[4] = {s.x, s.y, s.z, s.w}, incl[4];
        for (int f = 0; f < 4; ++f) {
            incl[f] = x[f];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, incl[f], o);
                if (lane >= o) incl[f] += y;
            }
            if (lane == 31) wsum[f][wid] = incl[f];
        }
        __syncthreads();
        if (wid == 0) {
            for (int f = 0; f < 4; ++f) {
                unsigned long long t = wsum[f][lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
                    if (lane >= o) t += y;
                }
                wsum[f][lane] = t;   // inclusive over warps
            }
        }
        __syncthreads();
        unsigned long long ex[4];
        for (int f = 0; f < 4; ++f) ex[f] = carry[f] + (wid ? wsum[f][wid - 1] : 0) + incl[f] - x[f];
        if (i < nb) sums[i] = make_ulonglong4(ex[0], ex[1], ex[2], ex[3]);
        for (int f = 0; f < 4; ++f) carry[f] += wsum[f][kScanThreads / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = make_ulonglong4(carry[0], carry[1], carry[2], carry[3]);
}

// block-local exclusive scan plus the block's offset: plan[i].off[f]
__global__ void __launch_bounds__(kScanThreads)
collect_scan_apply_kernel(CollectPlan *__restrict__ plan, uint32_t n, const ulonglong4 *__restrict__ sums)
{
    __shared__ unsigned long long wsum[4][kScanThreads / 32];
    const uint32_t i = blockIdx.x * kScanThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long x[4] = {0, 0, 0, 0}, incl[4];
    if (i < n)
        for (int f = 0; f < 4; ++f) x[f] = plan[i].v[f];
    for (int f = 0; f < 4; ++f) {
        incl[f] = x[f];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl[f], o);
            if (lane >= o) incl[f] += y;
        }
        if (lane == 31) wsum[f][wid] = incl[f];
    }
    __syncthreads();
    if (wid == 0) {
        for (int f = 0; f < 4; ++f) {
            unsigned long long t = wsum[f][lane];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[f][lane] = t;
        }
    }
    __syncthreads();
    if (i < n) {
        const ulonglong4 b = sums[blockIdx.x];
        const unsigned long long bo[4] = {b.x, b.y, b.z, b.w};
        for (int f = 0; f < 4; ++f) plan[i].off[f] = bo[f] + (wid ? wsum[f][wid - 1] : 0) + incl[f] - x[f];
    }
}

// windows: one warp per chain, forward then reversed
__global__ void __launch_bounds__(kCollectThreads)
collect_window_kernel(const uint8_t *__restrict__ pac, uint64_t l_pac, const CollectPlan *__restrict__ plan,
                      uint32_t n_chains, uint8_t *__restrict__ tbuf)
{
    const uint32_t c = (blockIdx.x * kCollectThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= n_chains) return;
    const CollectPlan pl = plan[c];
    const uint64_t L = pl.v[0] >> 1;
    uint8_t *fw = tbuf + pl.off[0], *rv = fw + L;
    for (uint64_t p = lane; p < L; p += 32) {
        const uint8_t b = pac_base(pac, l_pac, pl.r0 + p);
        fw[p] = b;
        rv[L - 1 - p] = b;
    }
}

// reads: one warp per read, forward then reversed, at twice the read's offset
__global__ void __launch_bounds__(kCollectThreads)
collect_read_kernel(const uint8_t *__restrict__ reads, const uint64_t *__restrict__ read_off, uint32_t n_reads,
                    uint8_t *__restrict__ qbuf)
{
    const uint32_t r = (blockIdx.x * kCollectThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n_reads) return;
    const uint64_t o = read_off[r], len = read_off[r + 1] - o;
    uint8_t *fw = qbuf + 2 * o, *rv = fw + len;
    for (uint64_t p = lane; p < len; p += 32) {
        const uint8_t b = reads[o + p];
        fw[p] = b;
        rv[len - 1 - p] = b;
    }
}

// jobs and the seed table: one thread per chain, its seeds last to first
__global__ void __launch_bounds__(kCollectThreads)
collect_jobs_kernel(fa_collect_opts opt, const uint64_t *__restrict__ read_off, const fa_chain *__restrict__ chains,
                    uint32_t n_chains, const fa_seed *__restrict__ seeds, const CollectPlan *__restrict__ plan,
                    fa_job *__restrict__ left, fa_job *__restrict__ right, fa_seed_ext *__restrict__ seed_ext,
                    uint32_t *__restrict__ chain_first, uint64_t *__restrict__ chain_win)
{
    const uint32_t c = blockIdx.x * kCollectThreads + threadIdx.x;
    if (c >= n_chains) return;
    const CollectPlan pl = plan[c];
    const fa_chain ch = chains[c];
    chain_first[c] = (uint32_t)pl.off[3];
    chain_win[2 * c] = pl.v[3] ? pl.r0 : 0u;
    chain_win[2 * c + 1] = pl.v[3] ? pl.r1 : 0u;
    if (pl.v[3] == 0) return;
    const uint64_t ro = read_off[ch.read];
    const int qlen = (int)(read_off[ch.read + 1] - ro);
    const uint64_t L = pl.v[0] >> 1, tw = pl.off[0];
    uint64_t li = pl.off[1], ri = pl.off[2], mi = pl.off[3];
    for (uint32_t kk = ch.n_seeds; kk-- > 0;) {
        const fa_seed s = seeds[ch.seed_first + kk];
        int32_t lj = -1, rj = -1;
        if (s.query_pos > 0) {   // collect_soa.rs:150-185
            const uint64_t tmp = s.ref_pos - pl.r0;
            if (tmp > 0 && tmp <= L) {
                fa_job j;
                j.q_off = 2 * ro + (uint64_t)qlen + (uint64_t)(qlen - s.query_pos);   // reversed read prefix
                j.t_off = tw + L + (L - tmp);                                         // reversed window prefix
                j.qlen = s.query_pos;
                j.tlen = (int32_t)tmp;
                j.h0 = s.len * opt.a;
                j.w = opt.w;
                j.dir = FA_DIR_LEFT;
                j._pad = 0;
                lj = (int32_t)li;
                left[li++] = j;
            }
        }
        const int qend = s.query_pos + s.len;   // collect_soa.rs:187-209
        if (qend < qlen) {
            const uint64_t tmp = s.ref_pos + (uint64_t)(int64_t)s.len - pl.r0;
            if (tmp < L) {
                fa_job j;
                j.q_off = 2 * ro + (uint64_t)qend;
                j.t_off = tw + tmp;
                j.qlen = qlen - qend;
                j.tlen = (int32_t)(L - tmp);
                j.h0 = 0;
                j.w = opt.w;
                j.dir = FA_DIR_RIGHT;
                j._pad = 0;
                rj = (int32_t)ri;
                right[ri++] = j;
            }
        }
        fa_seed_ext e;
        e.ref_pos = s.ref_pos;
        e.query_pos = s.query_pos;
        e.len = s.len;
        e.left_job = lj;
        e.right_job = rj;
        seed_ext[mi++] = e;
    }
}

}  // namespace

int collect_max_gap(const fa_collect_opts &o, int qlen) { return max_gap(o, qlen); }

size_t collect_scan_blocks(uint32_t n_chains) { return (n_chains + kScanThreads - 1) / kScanThreads; }

cudaError_t launch_collect_plan(const fa_collect_opts &opt, uint64_t l_pac, const uint64_t *d_read_off,
                                uint32_t n_reads, const fa_chain *d_chains, uint32_t n_chains, const fa_seed *d_seeds,
                                uint32_t n_seeds, CollectPlan *d_plan, ulonglong4 *d_sums, unsigned long long *d_bad,
                                cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(d_bad, 0xFF, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const uint32_t nc = n_reads > n_chains ? n_reads : n_chains;
    if (nc)
        collect_check_kernel<<<(nc + kCollectThreads - 1) / kCollectThreads, kCollectThreads, 0, s>>>(
            l_pac, d_read_off, n_reads, d_chains, n_chains, d_seeds, n_seeds, d_bad);
    if (n_chains == 0) return cudaGetLastError();
    collect_plan_kernel<<<(n_chains + kCollectThreads - 1) / kCollectThreads, kCollectThreads, 0, s>>>(
        opt, l_pac, d_read_off, n_reads, d_chains, n_chains, d_seeds, n_seeds, d_plan);
    return launch_plan_scan(d_plan, n_chains, d_sums, s);
}

cudaError_t launch_plan_scan(CollectPlan *d_plan, uint32_t n, ulonglong4 *d_sums, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const uint32_t nb = (uint32_t)collect_scan_blocks(n);
    collect_scan_sums_kernel<<<nb, kScanThreads, 0, s>>>(d_plan, n, d_sums);
    collect_scan_top_kernel<<<1, kScanThreads, 0, s>>>(d_sums, nb);
    collect_scan_apply_kernel<<<nb, kScanThreads, 0, s>>>(d_plan, n, d_sums);
    return cudaGetLastError();
}

cudaError_t launch_collect_fill(const fa_collect_opts &opt, const uint8_t *d_pac, uint64_t l_pac,
                                const uint8_t *d_reads, const uint64_t *d_read_off, uint32_t n_reads,
                                const fa_chain *d_chains, uint32_t n_chains, const fa_seed *d_seeds,
                                const CollectPlan *d_plan, fa_job *d_left, fa_job *d_right, uint8_t *d_qbuf,
                                uint8_t *d_tbuf, fa_seed_ext *d_seed_ext, uint32_t *d_chain_first,
                                uint64_t *d_chain_win, cudaStream_t s)
{
    if (n_reads) {
        const uint64_t threads = 32ull * n_reads;
        collect_read_kernel<<<(unsigned)((threads + kCollectThreads - 1) / kCollectThreads), kCollectThreads, 0, s>>>(
            d_reads, d_read_off, n_reads, d_qbuf);
    }
    if (n_chains) {
        const uint64_t threads = 32ull * n_chains;
        collect_window_kernel<<<(unsigned)((threads + kCollectThreads - 1) / kCollectThreads), kCollectThreads, 0,
                                s>>>(d_pac, l_pac, d_plan, n_chains, d_tbuf);
        collect_jobs_kernel<<<(n_chains + kCollectThreads - 1) / kCollectThreads, kCollectThreads, 0, s>>>(
            opt, d_read_off, d_chains, n_chains, d_seeds, d_plan, d_left, d_right, d_seed_ext, d_chain_first,
            d_chain_win);
    }
    return cudaGetLastError();
}

}  // namespace fa
