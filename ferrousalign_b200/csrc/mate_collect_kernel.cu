// mate_collect_kernel.cu -- mate-rescue jobs from anchors and a 2-bit packed reference (sm_100a).
//
// collect_rescue_jobs_for_read_soa (src/pipelines/linear/paired/mate_rescue.rs:1804-2045):
// per rescue attempt -- a read whose mate (the anchor) aligned -- no jobs unless some of the
// read's alignments score at least best - pen_unpaired (at most max_matesw counted) and its
// primary one does; otherwise every orientation not marked failed by the insert-size
// statistics and not already covered by one of the read's alignments at a consistent
// distance (mem_infer_dir, mate_rescue.rs:537-551) gets a reference window from the
// anchor's position and the orientation's insert-size bounds, cut to the anchor's
// reference sequence (bns_fetch_seq, bntseq.rs:700-739, with bns_pos2rid's binary search,
// :535-559); a window on that sequence of at least min_seed_len bases is a job: the read
// (reverse complemented for orientations 1 and 2) against the window's bases.
//
// Each attempt's (at most four) windows are computed twice: by one thread to size its
// output (target bytes, jobs, query bytes, scanned over the attempts with the job
// collection's scan), then by one warp whose lanes write the read and window bases of its
// jobs side by side.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

namespace {

constexpr int kMateCollectThreads = 128;

struct Win {
    int64_t beg, end;
    int32_t rid;
    bool ok;
};

// bns_pos2rid (bntseq.rs:535-559), its binary search as written
__device__ int pos2rid(const RescueRef &R, int64_t pos_f) {
    if (pos_f >= (int64_t)R.l_pac) return -1;
    uint32_t left = 0, right = R.n_chr, mid = 0;
    while (left < right) {
        mid = (left + right) >> 1;
        if (pos_f >= (int64_t)R.chr_off[mid]) {
            if (mid == R.n_chr - 1) break;
            if (pos_f < (int64_t)R.chr_off[mid + 1]) break;
            left = mid + 1;
        } else {
            right = mid;
        }
    }
    return (int)mid;
}

// FM-index start of an alignment on its strand (mate_rescue.rs:1897-1904, 1921-1928)
__device__ __forceinline__ int64_t aln_rb(const RescueRef &R, const fa_rescue_aln &a, int64_t chr_offset) {
    const int64_t g = chr_offset + a.pos;
    return a.is_rev ? ((int64_t)R.l_pac << 1) - 1 - (g + a.ref_len - 1) : g;
}

// the windows of one attempt; returns how many are jobs
__device__ int rescue_windows(const fa_rescue_opts &opt, const fa_insert_bounds *bd, const RescueRef &R,
                              const fa_rescue_aln *__restrict__ alns, const fa_rescue_cand &c, int qlen, Win w[4])
{
#pragma unroll
    for (int r = 0; r < 4; ++r) w[r].ok = false;
    // mate_rescue.rs:1822-1870: score threshold
    int best = 0;
    for (uint32_t k = 0; k < c.aln_count; ++k) {
        const int s = alns[c.aln_first + k].score;
        best = k == 0 || s > best ? s : best;
    }
    const long long t64 = (long long)best - opt.pen_unpaired;
    const int thr = t64 < INT32_MIN ? INT32_MIN : (t64 > INT32_MAX ? INT32_MAX : (int)t64);
    uint32_t above = 0;
    for (uint32_t k = 0; k < c.aln_count; ++k) above += alns[c.aln_first + k].score >= thr;
    if (opt.max_matesw >= 0 && above > (uint32_t)opt.max_matesw) above = (uint32_t)opt.max_matesw;
    if (above == 0 || alns[c.primary].score < thr) return 0;
    // mate_rescue.rs:1894-1940: orientations still to try
    const int64_t l_pac = (int64_t)R.l_pac;
    const int64_t chr_offset = (int64_t)R.chr_off[c.anchor.ref_id];
    const int64_t a_rb = aln_rb(R, c.anchor, chr_offset);
    bool skip[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) skip[r] = bd[r].failed != 0;
    for (uint32_t k = 0; k < c.aln_count; ++k) {
        const fa_rescue_aln &m = alns[c.aln_first + k];
        if (m.ref_id != c.anchor.ref_id) continue;
        const int64_t m_rb = aln_rb(R, m, chr_offset);
        // mem_infer_dir (mate_rescue.rs:537-551)
        const int r1 = a_rb >= l_pac, r2 = m_rb >= l_pac;
        const int64_t p2 = r1 == r2 ? m_rb : (l_pac << 1) - 1 - m_rb;
        const int64_t dist = p2 > a_rb ? p2 - a_rb : a_rb - p2;
        const int dir = (r1 == r2 ? 0 : 1) ^ (p2 > a_rb ? 0 : 3);
        if (dist >= bd[dir].low && dist <= bd[dir].high) skip[dir] = true;
    }
    int n = 0;
    for (int r = 0; r < 4; ++r) {   // mate_rescue.rs:1956-2044
        if (skip[r]) continue;
        const bool is_rev = (r >> 1) != (r & 1), is_larger = (r >> 1) == 0;
        int64_t rb, re;
        if (!is_rev) {
            rb = is_larger ? a_rb + bd[r].low : a_rb - bd[r].high;
            re = (is_larger ? a_rb + bd[r].high : a_rb - bd[r].low) + qlen;
        } else {
            rb = (is_larger ? a_rb + bd[r].low : a_rb - bd[r].high) - qlen;
            re = is_larger ? a_rb + bd[r].high : a_rb - bd[r].low;
        }
        rb = rb > 0 ? rb : 0;
        re = re < (l_pac << 1) ? re : (l_pac << 1);
        if (rb >= re) continue;
        // bns_fetch_seq: the reference sequence under the window's midpoint
        const int64_t mid = (rb + re) >> 1;
        const bool mrev = mid >= l_pac;
        const int64_t pos_f = mrev ? (l_pac << 1) - 1 - mid : mid;
        const int rid = pos2rid(R, pos_f);
        if (rid < 0 || rid != c.anchor.ref_id) continue;
        int64_t fb = (int64_t)R.chr_off[rid], fe = fb + (int64_t)R.chr_len[rid];
        if (mrev) {
            const int64_t t = fb;
            fb = (l_pac << 1) - fe;
            fe = (l_pac << 1) - t;
        }
        const int64_t beg = rb > fb ? rb : fb, end = re < fe ? re : fe;
        if (end - beg < opt.min_seed_len) continue;
        // a window on one strand of one sequence never straddles l_pac, so bns_get_seq
        // returns its end - beg bases
        w[r].beg = beg;
        w[r].end = end;
        w[r].rid = rid;
        w[r].ok = true;
        ++n;
    }
    return n;
}

__global__ void __launch_bounds__(kMateCollectThreads)
mate_collect_plan_kernel(fa_rescue_opts opt, fa_insert_bounds b0, fa_insert_bounds b1, fa_insert_bounds b2,
                         fa_insert_bounds b3, RescueRef R, const uint64_t *__restrict__ read_off,
                         const fa_rescue_aln *__restrict__ alns, const fa_rescue_cand *__restrict__ cands,
                         uint32_t n_cand, CollectPlan *__restrict__ plan)
{
    const uint32_t i = blockIdx.x * kMateCollectThreads + threadIdx.x;
    if (i >= n_cand) return;
    const fa_insert_bounds bd[4] = {b0, b1, b2, b3};
    const fa_rescue_cand c = cands[i];
    const int qlen = (int)(read_off[c.read + 1] - read_off[c.read]);
    Win w[4];
    const int n = rescue_windows(opt, bd, R, alns, c, qlen, w);
    CollectPlan pl{};
    for (int r = 0; r < 4; ++r)
        if (w[r].ok) pl.v[0] += (unsigned long long)(w[r].end - w[r].beg);
    pl.v[1] = (unsigned long long)n;
    pl.v[2] = (unsigned long long)n * (unsigned long long)qlen;
    plan[i] = pl;
}

__global__ void __launch_bounds__(kMateCollectThreads)
mate_collect_fill_kernel(fa_rescue_opts opt, fa_insert_bounds b0, fa_insert_bounds b1, fa_insert_bounds b2,
                         fa_insert_bounds b3, RescueRef R, const uint8_t *__restrict__ reads,
                         const uint64_t *__restrict__ read_off, const fa_rescue_aln *__restrict__ alns,
                         const fa_rescue_cand *__restrict__ cands, uint32_t n_cand,
                         const CollectPlan *__restrict__ plan, fa_mate_job *__restrict__ jobs,
                         fa_rescue_job_info *__restrict__ info, uint8_t *__restrict__ qbuf,
                         uint8_t *__restrict__ tbuf)
{
    const uint32_t i = (blockIdx.x * kMateCollectThreads + threadIdx.x) >> 5;   // one warp per attempt
    const int lane = threadIdx.x & 31;
    if (i >= n_cand) return;
    const CollectPlan pl = plan[i];
    if (pl.v[1] == 0) return;
    const fa_insert_bounds bd[4] = {b0, b1, b2, b3};
    const fa_rescue_cand c = cands[i];
    const uint64_t ro = read_off[c.read];
    const int qlen = (int)(read_off[c.read + 1] - ro);
    Win w[4];
    rescue_windows(opt, bd, R, alns, c, qlen, w);   // every lane: the same windows
    uint64_t ji = pl.off[1], qo = pl.off[2], to = pl.off[0];
    // mate_rescue.rs:314-321: the xtra word of every job of this read
    uint32_t xtra = 0x40000u | 0x80000u | (uint32_t)(opt.min_seed_len * opt.match_score);
    if (qlen * opt.match_score < 250) xtra |= 0x10000u;
    for (int r = 0; r < 4; ++r) {
        if (!w[r].ok) continue;
        const bool is_rev = (r >> 1) != (r & 1);
        for (int k = lane; k < qlen; k += 32) {   // the read, reverse complemented for 1 and 2
            const uint8_t b = is_rev ? reads[ro + qlen - 1 - k] : reads[ro + k];
            qbuf[qo + k] = is_rev ? (uint8_t)(b < 4 ? 3 - b : 4) : b;
        }
        const uint64_t L = (uint64_t)(w[r].end - w[r].beg);
        for (uint64_t p = lane; p < L; p += 32) tbuf[to + p] = pac_base(R.pac, R.l_pac, (uint64_t)w[r].beg + p);
        if (lane == 0) {
            fa_mate_job j;
            j.q_off = qo;
            j.t_off = to;
            j.qlen = qlen;
            j.tlen = (int32_t)L;
            j.xtra = xtra;
            j._pad = 0;
            jobs[ji] = j;
            fa_rescue_job_info f;
            f.cand = i;
            f.orientation = r;
            f.is_rev = is_rev;
            f.rid = w[r].rid;
            f.adj_rb = w[r].beg;
            f.adj_re = w[r].end;
            info[ji] = f;
        }
        ++ji;
        qo += (uint64_t)qlen;
        to += L;
    }
}

}  // namespace

cudaError_t launch_mate_collect_plan(const fa_rescue_opts &opt, const fa_insert_bounds *bd, RescueRef ref,
                                     const uint64_t *d_read_off, const fa_rescue_aln *d_alns,
                                     const fa_rescue_cand *d_cands, uint32_t n_cand, CollectPlan *d_plan,
                                     cudaStream_t s)
{
    if (n_cand == 0) return cudaSuccess;
    mate_collect_plan_kernel<<<(n_cand + kMateCollectThreads - 1) / kMateCollectThreads, kMateCollectThreads, 0,
                               s>>>(opt, bd[0], bd[1], bd[2], bd[3], ref, d_read_off, d_alns, d_cands, n_cand,
                                    d_plan);
    return cudaGetLastError();
}

cudaError_t launch_mate_collect_fill(const fa_rescue_opts &opt, const fa_insert_bounds *bd, RescueRef ref,
                                     const uint8_t *d_reads, const uint64_t *d_read_off, const fa_rescue_aln *d_alns,
                                     const fa_rescue_cand *d_cands, uint32_t n_cand, const CollectPlan *d_plan,
                                     fa_mate_job *d_jobs, fa_rescue_job_info *d_info, uint8_t *d_qbuf,
                                     uint8_t *d_tbuf, cudaStream_t s)
{
    if (n_cand == 0) return cudaSuccess;
    const uint64_t threads = 32ull * n_cand;
    mate_collect_fill_kernel<<<(unsigned)((threads + kMateCollectThreads - 1) / kMateCollectThreads),
                               kMateCollectThreads, 0, s>>>(opt, bd[0], bd[1], bd[2], bd[3], ref, d_reads, d_read_off, d_alns, d_cands,
                                    n_cand, d_plan, d_jobs, d_info, d_qbuf, d_tbuf);
    return cudaGetLastError();
}

}  // namespace fa
