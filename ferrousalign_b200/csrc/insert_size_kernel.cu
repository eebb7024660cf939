// insert_size_kernel.cu -- insert-size statistics of read pairs (sm_100a).
//
// calculate_insert_size_stats (src/pipelines/linear/paired/insert_size.rs:73-243): per
// orientation (mem_infer_dir, :34-51) the pairs' distances in (0, 10000], their 25th, 50th
// and 75th percentiles (sorted-order indices trunc(q n + 0.499)), the mean and standard
// deviation of the distances within 2 IQR of the quartiles, and the proper-pair bounds
// (3 IQR, widened to 4 standard deviations, at least 1); an orientation with fewer than 10
// pairs, or fewer than 5% of the largest orientation's, is marked failed.
//
// The sort is a histogram: distances are integers in [1, 10000], so one counter per value
// and orientation gives every order statistic and the in-bound sums exactly.  The squared
// deviations are added one sample at a time in ascending order with explicitly rounded
// double operations (no contraction into FMAs), the order and rounding of the reference's
// loop over the sorted vector, so the statistics are bit-identical.

#include <climits>

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

namespace {

constexpr int kMaxIns = 10000;   // insert_size.rs:19
constexpr int kBins = kMaxIns + 1;
constexpr int kHistThreads = 256;

__global__ void __launch_bounds__(kHistThreads)
insert_hist_kernel(int64_t l_pac, const int64_t *__restrict__ pairs, uint32_t n, uint32_t *__restrict__ hist)
{
    const uint32_t i = blockIdx.x * kHistThreads + threadIdx.x;
    if (i >= n) return;
    const int64_t pos1 = pairs[2 * i], pos2 = pairs[2 * i + 1];
    const int r1 = pos1 >= l_pac, r2 = pos2 >= l_pac;
    const int64_t p2 = r1 == r2 ? pos2 : (l_pac << 1) - 1 - pos2;
    const int64_t dist = p2 > pos1 ? p2 - pos1 : pos1 - p2;
    const int o = (r1 == r2 ? 0 : 1) ^ (p2 > pos1 ? 0 : 3);
    if (dist > 0 && dist <= kMaxIns) atomicAdd(&hist[o * kBins + (int)dist], 1u);
}

// Rust's saturating `f64 as i32`
__device__ __forceinline__ int32_t as_i32(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT_MAX;
    if (x <= -2147483648.0) return INT_MIN;
    return (int32_t)x;
}

// the k-th smallest distance (0-based) of orientation o
__device__ int order_stat(const uint32_t *h, uint64_t k) {
    uint64_t cum = 0;
    for (int v = 1; v <= kMaxIns; ++v) {
        cum += h[v];
        if (cum > k) return v;
    }
    return kMaxIns;
}

__global__ void insert_stats_kernel(const uint32_t *__restrict__ hist, fa_insert_stats *__restrict__ out)
{
    __shared__ uint64_t count_of[4];
    const int o = threadIdx.x;
    const uint32_t *h = hist + o * kBins;
    uint64_t n = 0;
    for (int v = 1; v <= kMaxIns; ++v) n += h[v];
    count_of[o] = n;
    fa_insert_stats st;
    st.avg = 0.0;
    st.std = 0.0;
    st.low = st.high = 0;
    st.failed = 1;
    st._pad = 0;
    if (n >= 10) {   // MIN_DIR_CNT, insert_size.rs:13
        const double dn = (double)n;
        const int p25 = order_stat(h, (uint64_t)__dadd_rn(__dmul_rn(0.25, dn), 0.499));
        const int p75 = order_stat(h, (uint64_t)__dadd_rn(__dmul_rn(0.75, dn), 0.499));
        const double iqr = (double)(p75 - p25);
        int low = as_i32(__dadd_rn(__dsub_rn((double)p25, __dmul_rn(2.0, iqr)), 0.499));   // OUTLIER_BOUND
        if (low < 1) low = 1;
        const int high_o = as_i32(__dadd_rn(__dadd_rn((double)p75, __dmul_rn(2.0, iqr)), 0.499));
        long long sum = 0;
        unsigned long long cnt = 0;
        for (int v = low > 1 ? low : 1; v <= high_o && v <= kMaxIns; ++v) {
            sum += (long long)v * h[v];
            cnt += h[v];
        }
        if (cnt > 0) {
            const double avg = __ddiv_rn((double)sum, (double)cnt);
            double ss = 0.0;
            for (int v = low > 1 ? low : 1; v <= high_o && v <= kMaxIns; ++v) {
                const double d = __dsub_rn((double)v, avg), dd = __dmul_rn(d, d);
                for (uint32_t c = 0; c < h[v]; ++c) ss = __dadd_rn(ss, dd);
            }
            const double sd = __dsqrt_rn(__ddiv_rn(ss, (double)cnt));
            int lo = as_i32(__dadd_rn(__dsub_rn((double)p25, __dmul_rn(3.0, iqr)), 0.499));    // MAPPING_BOUND
            int hi = as_i32(__dadd_rn(__dadd_rn((double)p75, __dmul_rn(3.0, iqr)), 0.499));
            const int lo_sd = as_i32(__dadd_rn(__dsub_rn(avg, __dmul_rn(4.0, sd)), 0.499));     // MAX_STDDEV
            const int hi_sd = as_i32(__dadd_rn(__dadd_rn(avg, __dmul_rn(4.0, sd)), 0.499));
            if (lo > lo_sd) lo = lo_sd;
            if (hi < hi_sd) hi = hi_sd;
            if (lo < 1) lo = 1;
            st.avg = avg;
            st.std = sd;
            st.low = lo;
            st.high = hi;
            st.failed = 0;
        }
    }
    __syncthreads();
    uint64_t mx = 0;
    for (int k = 0; k < 4; ++k) mx = count_of[k] > mx ? count_of[k] : mx;
    // MIN_DIR_RATIO (insert_size.rs:14, 228-236)
    if (!st.failed && n < (uint64_t)__dmul_rn((double)mx, 0.05)) st.failed = 1;
    out[o] = st;
}

}  // namespace

cudaError_t launch_insert_stats(int64_t l_pac, const int64_t *d_pairs, uint32_t n, uint32_t *d_hist,
                                fa_insert_stats *d_out, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * 4 * kBins, s);
    if (e != cudaSuccess) return e;
    if (n) insert_hist_kernel<<<(n + kHistThreads - 1) / kHistThreads, kHistThreads, 0, s>>>(l_pac, d_pairs, n, d_hist);
    insert_stats_kernel<<<1, 4, 0, s>>>(d_hist, d_out);
    return cudaGetLastError();
}

size_t insert_hist_bytes() { return sizeof(uint32_t) * 4 * kBins; }

}  // namespace fa
