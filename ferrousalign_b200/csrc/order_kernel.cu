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
