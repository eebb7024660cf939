// order_kernel.cu -- device-side length ordering of extension jobs.
//
// Jobs of similar query length share a warp, so the 32 lanes of a warp run similar
// row counts and the shared-memory class of a launch fits its jobs.  A histogram of
// query lengths sizes the launches; a scatter with warp-aggregated atomics writes the
// longest-first processing order.

#include "fa_kernels.h"

namespace fa {

constexpr int kHistBins = FA_MAX_QLEN + 1;

__global__ void qlen_hist_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint32_t *__restrict__ hist)
{
    __shared__ uint32_t h[kHistBins];
    for (int b = threadIdx.x; b < kHistBins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int q = jobs[i].qlen;
        q = q < 0 ? 0 : (q > FA_MAX_QLEN ? FA_MAX_QLEN : q);
        atomicAdd(&h[q], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kHistBins; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

__global__ void qlen_scatter_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ order)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    int q = live ? jobs[i].qlen : -1;
    q = q < -1 ? 0 : (q > FA_MAX_QLEN ? FA_MAX_QLEN : q);
    const unsigned peers = __match_any_sync(0xffffffffu, q);
    if (!live) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cursor[q], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    order[base + __popc(peers & ((1u << lane) - 1u))] = i;
}

cudaError_t launch_qlen_hist(const fa_job *d_jobs, uint32_t n, uint32_t *d_hist, int sm_count, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(d_hist, 0, sizeof(uint32_t) * kHistBins, s);
    if (e != cudaSuccess || n == 0) return e;
    uint32_t blocks = (n + 1023) / 1024;
    if (blocks > (uint32_t)sm_count * 4) blocks = sm_count * 4;
    qlen_hist_kernel<<<blocks, 1024, 0, s>>>(d_jobs, n, d_hist);
    return cudaGetLastError();
}

cudaError_t launch_qlen_scatter(const fa_job *d_jobs, uint32_t n, uint32_t *d_cursor, uint32_t *d_order,
                                cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    qlen_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, d_cursor, d_order);
    return cudaGetLastError();
}

}  // namespace fa

namespace fa {

// Splits mate-rescue jobs by lane width (KSW_XBYTE: 16 u8 lanes, else 8 i16 lanes) into
// two order lists and records, per kind, the job count and the longest query, plus the
// longest target: info = {n_byte, n_word, max_q_byte, max_q_word, max_t}.
__global__ void mate_split_kernel(const fa_mate_job *__restrict__ jobs, uint32_t n, uint32_t *__restrict__ order_b,
                                  uint32_t *__restrict__ order_w, uint32_t *__restrict__ info)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    fa_mate_job jb;
    if (live) jb = jobs[i];
    const bool byte = live && (jb.xtra & FA_KSW_XBYTE);
    const unsigned mb = __ballot_sync(0xffffffffu, byte);
    const unsigned mw = __ballot_sync(0xffffffffu, live && !byte);
    const int lane = threadIdx.x & 31;
    uint32_t base_b = 0, base_w = 0;
    if (lane == 0) {
        if (mb) base_b = atomicAdd(&info[0], (uint32_t)__popc(mb));
        if (mw) base_w = atomicAdd(&info[1], (uint32_t)__popc(mw));
    }
    base_b = __shfl_sync(0xffffffffu, base_b, 0);
    base_w = __shfl_sync(0xffffffffu, base_w, 0);
    if (!live) return;
    const unsigned below = (1u << lane) - 1u;
    if (byte) {
        order_b[base_b + __popc(mb & below)] = i;
        atomicMax(&info[2], (uint32_t)max(jb.qlen, 0));
    } else {
        order_w[base_w + __popc(mw & below)] = i;
        atomicMax(&info[3], (uint32_t)max(jb.qlen, 0));
    }
    atomicMax(&info[4], (uint32_t)max(jb.tlen, 0));
    if (jb.qlen <= 0 || jb.tlen < 0) atomicOr(&info[5], 1u);
}

cudaError_t launch_mate_split(const fa_mate_job *d_jobs, uint32_t n, uint32_t *d_order_b, uint32_t *d_order_w,
                              uint32_t *d_info, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(d_info, 0, 8 * sizeof(uint32_t), s);
    if (e != cudaSuccess || n == 0) return e;
    mate_split_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, d_order_b, d_order_w, d_info);
    return cudaGetLastError();
}

}  // namespace fa
