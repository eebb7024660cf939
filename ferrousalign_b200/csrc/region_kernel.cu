// region_kernel.cu -- alignment regions from left/right extension results (sm_100a).
//
// merge_scores_to_regions (src/pipelines/linear/region.rs:737-890), the consumer of the
// extension batch: for every seed of a chain, the region the seed's extensions reach,
// with bwa-mem2's clip decision per side (local bounds qle/tle unless the end-to-end
// score gscore is positive and within the clipping penalty of the local score, then the
// query end with gtle), the seed coverage of that region, and per chain the region of the
// first seed with the strictly highest total score.  One thread per chain: a chain holds
// a handful of seeds, and the work is a few integer compares per seed pair, so the kernel
// is bound by moving seed records and extension results from HBM: each block stages its
// chains' seed records in shared memory with coalesced copies, each thread fetches the
// results of four seeds at a time so their loads are in flight together, and the seed
// coverage (a pass over the chain's seeds) is computed for the chosen region only, the one
// whose coverage the reference keeps.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

namespace {

constexpr int kRegionThreads = 128;
constexpr int kStageSeeds = 8 * kRegionThreads;   // seed records a block stages (24 KB)
constexpr int kSeedGroup = 4;                     // seeds whose results are fetched together

// One extension result: as three 8-byte loads when the array is 8-byte aligned (V8), else
// field by field.
template <bool V8>
__device__ __forceinline__ fa_ext_result load_result(const fa_ext_result *__restrict__ base, int32_t k) {
    if (!V8) return base[k];
    const uint2 *p = reinterpret_cast<const uint2 *>(base + k);
    const uint2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    fa_ext_result r;
    r.score = (int32_t)a.x;
    r.qle = (int32_t)a.y;
    r.tle = (int32_t)b.x;
    r.gtle = (int32_t)b.y;
    r.gscore = (int32_t)c.x;
    r.max_off = (int32_t)c.y;
    return r;
}

template <bool V8>
__global__ void __launch_bounds__(kRegionThreads)
merge_regions_kernel(fa_region_opts opt, const uint32_t *__restrict__ chain_first, uint32_t n_chains,
                     const int32_t *__restrict__ query_len, const fa_seed_ext *__restrict__ seeds,
                     uint32_t n_seeds, const fa_ext_result *__restrict__ left, uint32_t n_left,
                     const fa_ext_result *__restrict__ right, uint32_t n_right, fa_region *__restrict__ out,
                     uint32_t *__restrict__ status)
{
    // The block's chains own one contiguous run of seed records: staged in shared memory
    // with coalesced 8-byte copies (when the run is well formed and fits), so each thread
    // then reads its chain's seeds -- once per region and once per coverage test -- from
    // there instead of with scattered 24-byte global loads.
    __shared__ uint2 stage[kStageSeeds * 3];
    const uint32_t cb0 = blockIdx.x * kRegionThreads;
    const uint32_t cb1 = min(cb0 + kRegionThreads, n_chains);
    const uint32_t b_lo = chain_first[cb0], b_hi = chain_first[cb1];
    const bool staged = b_lo <= b_hi && b_hi <= n_seeds && b_hi - b_lo <= (uint32_t)kStageSeeds;
    if (staged) {
        const uint2 *src = reinterpret_cast<const uint2 *>(seeds + b_lo);
        for (uint32_t i = threadIdx.x; i < 3 * (b_hi - b_lo); i += kRegionThreads) stage[i] = src[i];
    }
    __syncthreads();
    const uint32_t c = cb0 + threadIdx.x;
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
    const bool local = staged && s0 >= b_lo && s1 <= b_hi;
    const fa_seed_ext *sv = local ? reinterpret_cast<const fa_seed_ext *>(stage) : seeds;
    const uint32_t sbase = local ? b_lo : 0u;   // sv[k - sbase] is seed k
    const int32_t qlen = query_len[c];
    int32_t best_score = INT32_MIN;
    for (uint32_t k0 = s0; k0 < s1; k0 += kSeedGroup) {
        // the group's seeds and the extension results they index, all loads issued first
        fa_seed_ext sd[kSeedGroup];
        fa_ext_result L[kSeedGroup], R[kSeedGroup];
        bool has_l[kSeedGroup], has_r[kSeedGroup];
#pragma unroll
        for (int u = 0; u < kSeedGroup; ++u) {
            has_l[u] = has_r[u] = false;
            if (k0 + u < s1) {
                sd[u] = sv[k0 + u - sbase];
                has_l[u] = sd[u].left_job >= 0 && (uint32_t)sd[u].left_job < n_left;
                has_r[u] = sd[u].right_job >= 0 && (uint32_t)sd[u].right_job < n_right;
                if (has_l[u]) L[u] = load_result<V8>(left, sd[u].left_job);
                if (has_r[u]) R[u] = load_result<V8>(right, sd[u].right_job);
            }
        }
#pragma unroll
        for (int u = 0; u < kSeedGroup; ++u) {
            if (k0 + u >= s1) break;
            const fa_seed_ext &s = sd[u];
            // region.rs:772-781: bounds from the seed, seed score len * a
            int32_t qb = s.query_pos, qe = s.query_pos + s.len;
            uint64_t rb = s.ref_pos, re = s.ref_pos + (uint64_t)(int64_t)s.len;
            int32_t truesc = 0;
            int32_t total = s.len * opt.a;
            if (has_l[u]) {
                // region.rs:784-809 (an index past the left results leaves the seed's bounds)
                total = L[u].score;
                if (L[u].gscore <= 0 || L[u].gscore <= L[u].score - opt.pen_clip5) {   // local
                    qb = s.query_pos - L[u].qle;
                    rb = s.ref_pos - (uint64_t)(int64_t)L[u].tle;
                    truesc = L[u].score;
                } else {                                                             // to the query start
                    qb = 0;
                    rb = s.ref_pos - (uint64_t)(int64_t)L[u].gtle;
                    truesc = L[u].gscore;
                }
            } else if (s.left_job < 0 && s.query_pos == 0) {
                truesc = s.len * opt.a;   // region.rs:810-813
            }
            if (has_r[u]) {   // region.rs:816-836
                total += R[u].score;
                const uint64_t seed_end = s.ref_pos + (uint64_t)(int64_t)s.len;
                if (R[u].gscore <= 0 || R[u].gscore <= R[u].score - opt.pen_clip3) {
                    qe = s.query_pos + s.len + R[u].qle;
                    re = seed_end + (uint64_t)(int64_t)R[u].tle;
                } else {
                    qe = qlen;
                    re = seed_end + (uint64_t)(int64_t)R[u].gtle;
                }
            }
            if (truesc == 0) truesc = total;   // region.rs:842-845
            if (total > best_score) {   // region.rs:868-872: first strict maximum of the chain
                best_score = total;
                best.rb = rb;
                best.re = re;
                best.qb = qb;
                best.qe = qe;
                best.score = total;
                best.truesc = truesc;
                best.seedlen0 = s.len;
                best.seed = (int32_t)(k0 + u);
            }
        }
    }
    // region.rs:847-858: seeds of the chain inside the region, both axes -- computed for
    // the chosen region only, the one whose coverage the reference keeps
    if (best.seed >= 0) {
        int32_t cov = 0;
        for (uint32_t o = s0; o < s1; ++o) {
            const fa_seed_ext so = sv[o - sbase];
            if (so.query_pos >= best.qb && so.query_pos + so.len <= best.qe && so.ref_pos >= best.rb &&
                so.ref_pos + (uint64_t)(int64_t)so.len <= best.re)
                cov += so.len;
        }
        best.seedcov = cov;
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
    const bool v8 = (((uintptr_t)d_left | (uintptr_t)d_right) & 7u) == 0;
    if (v8)
        merge_regions_kernel<true><<<blocks, kRegionThreads, 0, s>>>(opt, d_chain_first, n_chains, d_query_len,
                                                                     d_seeds, n_seeds, d_left, n_left, d_right,
                                                                     n_right, d_out, d_status);
    else
        merge_regions_kernel<false><<<blocks, kRegionThreads, 0, s>>>(opt, d_chain_first, n_chains, d_query_len,
                                                                      d_seeds, n_seeds, d_left, n_left, d_right,
                                                                      n_right, d_out, d_status);
    return cudaGetLastError();
}

}  // namespace fa
