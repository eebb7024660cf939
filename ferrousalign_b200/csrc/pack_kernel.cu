// pack_kernel.cu -- byte codes to the 2-bit packed form with its N runs, on the device
// (sm_100a), for outputs that the job-collection kernels write as bytes.
//
// Packed layout (fa_packed_seq): base k in bits 2*(k % 4) of byte k / 4; a code of 4 (N) is
// stored as 0 and listed in a sorted run list of (pos, len).  The packing is one thread per
// 16 bases (one 16-byte load, one 32-bit store); the runs come from three launches: run
// starts counted per block, the block counts scanned by one block, then each thread writes
// its starts' runs at its place in position order.  HBM-bound passes over the bytes.

#include "fa_device.cuh"
#include "fa_kernels.h"
#include "fa_packed.cuh"

namespace fa {

namespace {

constexpr int kPackThreads = 256;
constexpr int kRunChunk = 64;                          // bytes a thread scans for run starts
constexpr int kRunBlockBytes = kRunChunk * kPackThreads;

// four byte codes -> 8 bits (code & 3 each: N, code 4, becomes 0)
__device__ __forceinline__ uint32_t pack4(uint32_t v) {
    v &= 0x03030303u;
    return (v | v >> 6 | v >> 12 | v >> 18) & 0xFFu;
}

__global__ void __launch_bounds__(kPackThreads)
pack2_kernel(const uint8_t *__restrict__ src, uint64_t n, uint32_t *__restrict__ dst)
{
    const uint64_t w = (uint64_t)blockIdx.x * kPackThreads + threadIdx.x;
    const uint64_t b0 = w * 16;
    if (b0 >= n) return;
    const uint4 x = *reinterpret_cast<const uint4 *>(src + b0);   // the source is 16-byte aligned and padded
    uint32_t r = pack4(x.x) | pack4(x.y) << 8 | pack4(x.z) << 16 | pack4(x.w) << 24;
    if (b0 + 16 > n) r &= (1u << (2 * (uint32_t)(n - b0))) - 1u;   // bases past the end: 0
    dst[w] = r;
}

// starts of N runs among bytes [k0, k1) (the byte before k0 decides a start at k0): a full
// chunk as four 16-byte loads, each word's N bytes found with one SIMD compare (a start is an
// N byte whose lower neighbour is not N); a partial one byte by byte
__device__ __forceinline__ uint32_t count_starts(const uint8_t *__restrict__ src, uint64_t k0, uint64_t k1) {
    uint32_t c = 0;
    uint32_t prev = k0 > 0 && src[k0 - 1] == 4u ? 0xFF000000u : 0u;   // the previous N mask's top byte
    if (k1 - k0 == kRunChunk) {
        const uint4 *q = reinterpret_cast<const uint4 *>(src + k0);
#pragma unroll
        for (int v = 0; v < kRunChunk / 16; ++v) {
            const uint4 x = q[v];
            const uint32_t w[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const uint32_t nm = __vcmpeq4(w[m], 0x04040404u);
                c += __popc(nm & ~(nm << 8 | prev >> 24)) >> 3;
                prev = nm;
            }
        }
        return c;
    }
    uint32_t pb = prev ? 4u : 0u;
    for (uint64_t k = k0; k < k1; ++k) {
        const uint32_t v = src[k];
        c += v == 4u && pb != 4u;
        pb = v;
    }
    return c;
}

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *tot) {
    __shared__ uint32_t warp_sums[kPackThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < kPackThreads / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kPackThreads / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (wid > 0 ? warp_sums[wid - 1] : 0u) + x - v;
    if (tot) *tot = warp_sums[kPackThreads / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kPackThreads)
runs_count_kernel(const uint8_t *__restrict__ src, uint64_t n, uint32_t *__restrict__ block_counts)
{
    const uint64_t k0 = (uint64_t)blockIdx.x * kRunBlockBytes + (uint64_t)threadIdx.x * kRunChunk;
    const uint64_t k1 = k0 + kRunChunk < n ? k0 + kRunChunk : n;
    const uint32_t c = k0 < n ? count_starts(src, k0, k1) : 0u;
    uint32_t tot;
    block_exclusive_scan(c, &tot);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = tot;
}

// exclusive prefix of the block counts (one block); the total at [nblocks]
__global__ void __launch_bounds__(1024)
runs_scan_kernel(uint32_t *__restrict__ block_counts, uint32_t nblocks)
{
    __shared__ uint32_t part[1024];
    const uint32_t per = (nblocks + 1023) / 1024;
    const uint32_t a = threadIdx.x * per, b = min(a + per, nblocks);
    uint32_t s = 0;
    for (uint32_t i = a; i < b; ++i) s += block_counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t y = threadIdx.x >= (uint32_t)o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += y;
        __syncthreads();
    }
    uint32_t run = threadIdx.x > 0 ? part[threadIdx.x - 1] : 0u;
    for (uint32_t i = a; i < b; ++i) {
        const uint32_t v = block_counts[i];
        block_counts[i] = run;
        run += v;
    }
    if (threadIdx.x == 1023) block_counts[nblocks] = part[1023];
}

__global__ void __launch_bounds__(kPackThreads)
runs_write_kernel(const uint8_t *__restrict__ src, uint64_t n, const uint32_t *__restrict__ block_first,
                  fa_nrun *__restrict__ runs, uint64_t cap)
{
    const uint64_t k0 = (uint64_t)blockIdx.x * kRunBlockBytes + (uint64_t)threadIdx.x * kRunChunk;
    const uint64_t k1 = k0 + kRunChunk < n ? k0 + kRunChunk : n;
    const uint32_t c = k0 < n ? count_starts(src, k0, k1) : 0u;
    uint64_t slot = (uint64_t)block_first[blockIdx.x] + block_exclusive_scan(c, nullptr);
    if (c == 0) return;
    uint32_t prev = k0 > 0 ? src[k0 - 1] : 0u;
    for (uint64_t k = k0; k < k1; ++k) {
        const uint32_t v = src[k];
        if (v == 4u && prev != 4u) {
            uint64_t e = k + 1;
            while (e < n && src[e] == 4u) ++e;
            if (slot < cap) runs[slot] = fa_nrun{k, e - k};
            ++slot;
        }
        prev = v;
    }
}

// 2-bit packed -> byte codes, one thread per 16 bases (one 32-bit load, one 16-byte store)
__global__ void __launch_bounds__(kPackThreads)
unpack2_kernel(const uint32_t *__restrict__ src, uint64_t n, uint8_t *__restrict__ dst)
{
    const uint64_t w = (uint64_t)blockIdx.x * kPackThreads + threadIdx.x;
    if (w * 16 >= n) return;
    const uint32_t x = src[w];
    uint4 o;
    o.x = spread4(x & 0xFFu);
    o.y = spread4((x >> 8) & 0xFFu);
    o.z = spread4((x >> 16) & 0xFFu);
    o.w = spread4(x >> 24);
    *reinterpret_cast<uint4 *>(dst + w * 16) = o;   // the destination is padded to 16 bytes
}

// one thread per N run: its bases in [lo, hi) back to code 4
__global__ void __launch_bounds__(kPackThreads)
apply_runs_kernel(const fa_nrun *__restrict__ runs, uint32_t nr, uint64_t lo, uint64_t hi, uint8_t *__restrict__ dst)
{
    const uint32_t k = blockIdx.x * kPackThreads + threadIdx.x;
    if (k >= nr) return;
    const fa_nrun r = runs[k];
    const uint64_t e = r.pos + r.len < hi ? r.pos + r.len : hi;
    for (uint64_t q = r.pos > lo ? r.pos : lo; q < e; ++q) dst[q] = 4;
}

}  // namespace

cudaError_t launch_unpack2_range(const uint8_t *d_src, uint64_t p0, uint64_t p1, const fa_nrun *d_runs,
                                 uint32_t n_runs, uint8_t *d_dst, cudaStream_t s)
{
    if (p1 <= p0) return cudaSuccess;
    if (p0 % 16) return cudaErrorInvalidValue;
    const uint64_t words = (p1 - p0 + 15) / 16;
    unpack2_kernel<<<(unsigned)((words + kPackThreads - 1) / kPackThreads), kPackThreads, 0, s>>>(
        reinterpret_cast<const uint32_t *>(d_src) + p0 / 16, p1 - p0, d_dst + p0);
    if (n_runs)
        apply_runs_kernel<<<(n_runs + kPackThreads - 1) / kPackThreads, kPackThreads, 0, s>>>(d_runs, n_runs, p0, p1,
                                                                                          d_dst);
    return cudaGetLastError();
}

cudaError_t launch_unpack2(const uint8_t *d_src, uint64_t n, const fa_nrun *d_runs, uint32_t n_runs, uint8_t *d_dst,
                           cudaStream_t s)
{
    return launch_unpack2_range(d_src, 0, n, d_runs, n_runs, d_dst, s);
}

size_t pack_runs_scratch_words(uint64_t n) { return (n + kRunBlockBytes - 1) / kRunBlockBytes + 1; }

cudaError_t launch_pack2(const uint8_t *d_src, uint64_t n, uint8_t *d_dst, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const uint64_t words = (n + 15) / 16;
    pack2_kernel<<<(unsigned)((words + kPackThreads - 1) / kPackThreads), kPackThreads, 0, s>>>(
        d_src, n, reinterpret_cast<uint32_t *>(d_dst));
    return cudaGetLastError();
}

cudaError_t launch_nruns(const uint8_t *d_src, uint64_t n, fa_nrun *d_runs, uint64_t cap, uint32_t *d_scratch,
                         cudaStream_t s)
{
    const uint32_t nb = (uint32_t)((n + kRunBlockBytes - 1) / kRunBlockBytes);
    if (nb == 0) return cudaMemsetAsync(d_scratch, 0, sizeof(uint32_t), s);
    runs_count_kernel<<<nb, kPackThreads, 0, s>>>(d_src, n, d_scratch);
    runs_scan_kernel<<<1, 1024, 0, s>>>(d_scratch, nb);
    runs_write_kernel<<<nb, kPackThreads, 0, s>>>(d_src, n, d_scratch, d_runs, cap);
    return cudaGetLastError();
}

}  // namespace fa
