// region_kernel.cu -- alignment regions from left/right extension results (sm_100a).
//
// merge_scores_to_regions (src/pipelines/linear/region.rs:737-890), the consumer of the
// extension batch: for every seed of a chain, the region the seed's extensions reach,
// with bwa-mem2's clip decision per side (local bounds qle/tle unless the end-to-end
// score gscore is positive and within the clipping penalty of the local score, then the
// query end with gtle), the seed coverage of that region, and per chain the region of the
// first seed with the strictly highest total score.  One thread per chain: a chain holds
// a handful of seeds, and the work is a few integer compares per seed pair, so the kernel
// is bound by the gathers of seed records and extension results from HBM.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

namespace {

constexpr int kRegionThreads = 128;

__global__ void __launch_bounds__(kRegionThreads)
merge_regions_kernel(fa_region_opts opt, const uint32_t *__restrict__ chain_first, uint32_t n_chains,
                     const int32_t *__restrict__ query_len, const fa_seed_ext *__restrict__ seeds,
                     uint32_t n_seeds, const fa_ext_result *__restrict__ left, uint32_t n_left,
                     const fa_ext_result *__restrict__ right, uint32_t n_right, fa_region *__restrict__ out,
                     uint32_t *__restrict__ status)
{
    const uint32_t c = blockIdx.x * kRegionThreads + threadIdx.x;
    if (c >= n_chains) return;
    const uint32_t s0 = chain_first[c], s1 = chain_first[c + 1];
    fa_region best;
    best.rb = best.re = 0;
    best.qb = best.qe = best.score = best.truesc = best.seedcov = best.seedlen0 = 0;
    best.w = opt.w;
    best.seed = -1;
    if (s1 < s0 || s1 > n_seeds) {   // malformed chain range: no region, reported
        atomicOr(status, ST_RANGE);
        out[c] = best;
        return;
    }
    const int32_t qlen = query_len[c];
    int32_t best_score = INT32_MIN;
    for (uint32_t k = s0; k < s1; ++k) {
        const fa_seed_ext sd = seeds[k];
        // region.rs:772-781: bounds from the seed, seed score len * a
        int32_t qb = sd.query_pos, qe = sd.query_pos + sd.len;
        uint64_t rb = sd.ref_pos, re = sd.ref_pos + (uint64_t)(int64_t)sd.len;
        int32_t truesc = 0;
        int32_t total = sd.len * opt.a;
        if (sd.left_job >= 0) {
            // region.rs:784-809: an index past the left results leaves the seed's bounds
            if ((uint32_t)sd.left_job < n_left) {
                const fa_ext_result L = left[sd.left_job];
                total = L.score;
                if (L.gscore <= 0 || L.gscore <= L.score - opt.pen_clip5) {   // local
                    qb = sd.query_pos - L.qle;
                    rb = sd.ref_pos - (uint64_t)(int64_t)L.tle;
                    truesc = L.score;
                } else {                                                       // to the query start
                    qb = 0;
                    rb = sd.ref_pos - (uint64_t)(int64_t)L.gtle;
                    truesc = L.gscore;
                }
            }
        } else if (sd.query_pos == 0) {
            truesc = sd.len * opt.a;   // region.rs:810-813
        }
        if (sd.right_job >= 0 && (uint32_t)sd.right_job < n_right) {   // region.rs:816-836
            const fa_ext_result R = right[sd.right_job];
            total += R.score;
            const uint64_t seed_end = sd.ref_pos + (uint64_t)(int64_t)sd.len;
            if (R.gscore <= 0 || R.gscore <= R.score - opt.pen_clip3) {
                qe = sd.query_pos + sd.len + R.qle;
                re = seed_end + (uint64_t)(int64_t)R.tle;
            } else {
                qe = qlen;
                re = seed_end + (uint64_t)(int64_t)R.gtle;
            }
        }
        if (truesc == 0) truesc = total;   // region.rs:842-845
        // region.rs:847-858: seeds of the chain inside the region, both axes
        int32_t cov = 0;
        for (uint32_t o = s0; o < s1; ++o) {
            const fa_seed_ext so = seeds[o];
            if (so.query_pos >= qb && so.query_pos + so.len <= qe && so.ref_pos >= rb &&
                so.ref_pos + (uint64_t)(int64_t)so.len <= re)
                cov += so.len;
        }
        if (total > best_score) {   // region.rs:868-872: first strict maximum of the chain
            best_score = total;
            best.rb = rb;
            best.re = re;
            best.qb = qb;
            best.qe = qe;
            best.score = total;
            best.truesc = truesc;
            best.seedcov = cov;
            best.seedlen0 = sd.len;
            best.seed = (int32_t)k;
        }
    }
    out[c] = best;
}

}  // namespace

cudaError_t launch_merge_regions(const fa_region_opts &opt, const uint32_t *d_chain_first, uint32_t n_chains,
                                 const int32_t *d_query_len, const fa_seed_ext *d_seeds, uint32_t n_seeds,
                                 const fa_ext_result *d_left, uint32_t n_left, const fa_ext_result *d_right,
                                 uint32_t n_right, fa_region *d_out, uint32_t *d_status, cudaStream_t s)
{
    if (n_chains == 0) return cudaSuccess;
    const uint32_t blocks = (n_chains + kRegionThreads - 1) / kRegionThreads;
    merge_regions_kernel<<<blocks, kRegionThreads, 0, s>>>(opt, d_chain_first, n_chains, d_query_len, d_seeds,
                                                           n_seeds, d_left, n_left, d_right, n_right, d_out,
                                                           d_status);
    return cudaGetLastError();
}

}  // namespace fa
