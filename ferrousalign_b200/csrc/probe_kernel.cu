// probe_kernel.cu -- integer / DPX instruction-throughput probe.
//
// The roofline of the DP kernels is the SM integer pipe, for which no measured peak
// exists on this hardware; this probe measures it.  Each thread keeps 32 independent
// accumulator chains and applies one instruction kind to all of them four times per loop
// iteration (128 instructions of the measured kind against one add, compare and branch
// of loop control), with no other ALU work in the loop, so the issue rate of that one
// instruction kind, not latency or bookkeeping, bounds the run.

#include <cstdio>
#include <cuda_fp16.h>

#include "fa_kernels.h"

namespace fa {

constexpr int kProbeChains = 32;

__device__ __forceinline__ __half2 u2h(uint32_t x) {
    __half2 h;
    memcpy(&h, &x, 4);
    return h;
}
__device__ __forceinline__ uint32_t h2u(__half2 h) {
    uint32_t x;
    memcpy(&x, &h, 4);
    return x;
}
constexpr int kProbeUnroll = 4;

template <int KIND>
__global__ void __launch_bounds__(256) probe_kernel(uint32_t b, uint32_t c, int iters, uint32_t *sink)
{
    uint32_t acc[kProbeChains];
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) acc[k] = threadIdx.x * 2654435761u + k * 40503u + blockIdx.x;
#pragma unroll 1
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < kProbeUnroll; ++u) {
#pragma unroll
            for (int k = 0; k < kProbeChains; ++k) {
                if (KIND == 0) acc[k] = __viaddmax_s16x2_relu(acc[k], b, c);
                else if (KIND == 1) acc[k] = __vimax3_s16x2_relu(acc[k], b, c);
                else if (KIND == 2) acc[k] = (uint32_t)__viaddmax_s32_relu((int)acc[k], (int)b, (int)c);
                else if (KIND == 3) acc[k] = (uint32_t)__vimax3_s32((int)acc[k], (int)b, (int)c);
                else if (KIND == 4) acc[k] = (uint32_t)max((int)acc[k] + (int)b, (int)c);
                else if (KIND == 5) acc[k] = h2u(__hmax2(u2h(acc[k]), u2h(b)));
                else if (KIND == 6) acc[k] = h2u(__hadd2(u2h(acc[k]), u2h(b)));
                else if (KIND == 7) acc[k] = acc[k] * b + c;                         // IMAD
                else if (KIND == 8) {   // half the chains on DPX, half on half2 max: shared pipe or not
                    if (k & 1) acc[k] = h2u(__hmax2(u2h(acc[k]), u2h(b)));
                    else acc[k] = __viaddmax_s16x2_relu(acc[k], b, c);
                } else {                // KIND 9: DPX and IMAD interleaved
                    if (k & 1) acc[k] = acc[k] * b + c;
                    else acc[k] = __viaddmax_s16x2_relu(acc[k], b, c);
                }
            }
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) x ^= acc[k];
    if (x == 0x9e3779b9u) sink[0] = x;
}

// ops/s for one instruction kind (0: viaddmax_s16x2_relu, 1: vimax3_s16x2_relu,
// 2: viaddmax_s32_relu, 3: vimax3_s32, 4: add+max as two plain instructions, 5: half2 max,
// 6: half2 add, 7: integer multiply-add, 8: DPX and half2 max on alternate chains, 9: DPX and
// integer multiply-add on alternate chains -- the last two tell whether the kinds share a pipe).
double probe_int_peak(int kind, int sm_count, cudaStream_t s, float *ms_out)
{
    uint32_t *sink = nullptr;
    if (cudaMalloc(&sink, 4) != cudaSuccess) return -1.0;
    const int iters = 1024, threads = 256, blocks = sm_count * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&]() {
        switch (kind) {
            case 0: probe_kernel<0><<<blocks, threads, 0, s>>>(0x00010001u, 0x00020002u, iters, sink); break;
            case 1: probe_kernel<1><<<blocks, threads, 0, s>>>(0x00010001u, 0x00020002u, iters, sink); break;
            case 2: probe_kernel<2><<<blocks, threads, 0, s>>>(1u, 2u, iters, sink); break;
            case 3: probe_kernel<3><<<blocks, threads, 0, s>>>(1u, 2u, iters, sink); break;
            case 5: probe_kernel<5><<<blocks, threads, 0, s>>>(0x64006400u, 0x64016401u, iters, sink); break;
            case 6: probe_kernel<6><<<blocks, threads, 0, s>>>(0x00010001u, 0u, iters, sink); break;
            case 7: probe_kernel<7><<<blocks, threads, 0, s>>>(3u, 1u, iters, sink); break;
            case 8: probe_kernel<8><<<blocks, threads, 0, s>>>(0x00010001u, 0x00020002u, iters, sink); break;
            case 9: probe_kernel<9><<<blocks, threads, 0, s>>>(0x00010001u, 0x00020002u, iters, sink); break;
            default: probe_kernel<4><<<blocks, threads, 0, s>>>(1u, 2u, iters, sink); break;
        }
    };
    for (int w = 0; w < 3; ++w) launch();
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    if (ms_out) *ms_out = best;
    const double ops = (double)blocks * threads * iters * (kProbeChains * kProbeUnroll) * (kind == 4 ? 2.0 : 1.0);
    return ops / (best * 1e-3);
}

}  // namespace fa
