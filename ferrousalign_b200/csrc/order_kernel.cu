// order_kernel.cu -- device-side length ordering of extension jobs.
//
// Jobs of similar query length share a warp, so the 32 lanes of a warp run similar
// row counts and the shared-memory class of a launch fits its jobs.  A histogram of
// query lengths sizes the launches; a scatter with warp-aggregated atomics writes the
// longest-first processing order.

#include "fa_kernels.h"

namespace fa {

constexpr int kHistBins = FA_MAX_QLEN + 1;

// Histogram bin of a job's query length: [0, FA_MAX_QLEN], lengths outside clamped to the
// nearer end.  The histogram and the scatter both use it, so every job has the same bin in
// both and each order slot is written exactly once.
__host__ __device__ __forceinline__ int qlen_bin(int qlen) {
    return qlen < 0 ? 0 : (qlen > FA_MAX_QLEN ? FA_MAX_QLEN : qlen);
}

__global__ void qlen_hist_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint32_t *__restrict__ hist)
{
    __shared__ uint32_t h[kHistBins];
    for (int b = threadIdx.x; b < kHistBins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&h[qlen_bin(jobs[i].qlen)], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kHistBins; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

__global__ void qlen_scatter_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ order)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    // a live job lands in the same bin as in qlen_hist_kernel (negative lengths in bin 0);
    // -1 marks only the lanes past n, which leave before touching the cursors
    const int q = live ? qlen_bin(jobs[i].qlen) : -1;
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
// longest target and the shortest u8 query: info = {n_byte, n_word, max_q_byte, max_q_word,
// max_t, bad, ~min_q_byte}.
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
        atomicMax(&info[6], 0xFFFFFFFFu - (uint32_t)max(jb.qlen, 0));   // the shortest, complemented
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

namespace fa {

// ------------------------------------------------------------- pipelined host batches
// A host batch is uploaded in K byte slices of the query and target buffers; a job can
// run once the slices holding its sequences have arrived, so jobs are grouped by that
// slice ("chunk", the larger of the query's and the target's last slice) and, inside a
// chunk, by decreasing query length.  Bin = chunk * (FA_MAX_QLEN + 1) + (FA_MAX_QLEN - qlen).
// The prep kernel also validates every job against the buffer lengths and the kernel
// limits (the same rules as the host-side checks), keeping the first bad job's index,
// and reduces the longest query and the widest configured band.  info = {status, first bad
// job, longest query, widest band}.

constexpr int kChunkBins = FA_MAX_QLEN + 1;

// the chunk of a job: the one holding the later of its query's and its target's last byte
__device__ __forceinline__ int chunk_of(const fa_job &jb, const ChunkEnds &ends, int nchunks) {
    const uint64_t lq = (jb.q_off + (uint64_t)jb.qlen - 1) >> ends.shift;
    const uint64_t lt = jb.tlen > 0 ? (jb.t_off + (uint64_t)jb.tlen - 1) >> ends.shift : 0;
    // the ends are increasing, so the count of ends at or below a byte is its chunk; the
    // later of the two chunks is the larger count
    int cq = 0, ct = 0;
    for (int k = 0; k < nchunks - 1; ++k) {
        cq += ends.q[k] <= lq;
        ct += ends.t[k] <= lt;
    }
    return cq > ct ? cq : ct;
}

__global__ void chunk_prep_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint64_t qbytes, uint64_t tbytes,
                                  const ChunkEnds ends, int nchunks, int max_score, int h0_min, int qcap_limit,
                                  uint32_t *__restrict__ hist, uint32_t *__restrict__ info)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    int bin = -1, qlen = 0, band = 0;
    if (live) {
        const fa_job jb = jobs[i];
        qlen = jb.qlen;
        band = max(jb.w, 0);
        uint32_t st = 0;
        if (jb.qlen <= 0 || jb.tlen < 0 || jb.h0 < h0_min) st |= ST_ARG;
        else if (jb.qlen > FA_MAX_QLEN || jb.tlen > FA_MAX_TLEN) st |= ST_CAPACITY;
        else if (jb.q_off + (uint64_t)jb.qlen > qbytes || jb.t_off + (uint64_t)jb.tlen > tbytes) st |= ST_ARG;
        else if ((int64_t)jb.h0 + (int64_t)max_score * jb.qlen > kPackedHMax || jb.qlen > qcap_limit)
            st |= ST_CAPACITY;
        if (st) {
            atomicOr(&info[0], st);
            atomicMin(&info[1], i);
            qlen = 0;
        } else {
            bin = chunk_of(jb, ends, nchunks) * kChunkBins + (FA_MAX_QLEN - jb.qlen);
        }
    }
    {
        // each chunk's lowest and highest job index (a chunk whose jobs form one index range
        // can return its results as soon as it has run)
        const int chunk = bin >= 0 ? bin / kChunkBins : -1;
        const unsigned same = __match_any_sync(0xffffffffu, chunk);
        const int lane = threadIdx.x & 31, lo_lane = __ffs(same) - 1, hi_lane = 31 - __clz(same);
        if (chunk >= 0 && lane == lo_lane) {
            atomicMin(&info[4 + nchunks + 1 + chunk], i);
            atomicMax(&info[4 + 2 * nchunks + 1 + chunk], i - lane + hi_lane);
        }
    }
    const int mq = __reduce_max_sync(0xffffffffu, qlen);
    if ((threadIdx.x & 31) == 0 && mq > 0) atomicMax(&info[2], (uint32_t)mq);
    const int mw = __reduce_max_sync(0xffffffffu, band);
    if ((threadIdx.x & 31) == 0 && mw > 0) atomicMax(&info[3], (uint32_t)mw);
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (bin >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
}

// Exclusive prefix over the bins (one block), and the chunk bounds: bounds[k] = first
// order position of chunk k, bounds[nchunks] = the number of valid jobs.
__global__ void __launch_bounds__(1024) chunk_scan_kernel(const uint32_t *__restrict__ hist, int nbins,
                                                          uint32_t *__restrict__ base, int nchunks,
                                                          uint32_t *__restrict__ bounds)
{
    __shared__ uint32_t part[1024];
    const int per = (nbins + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    uint32_t s = 0;
    for (int b = b0; b < min(b0 + per, nbins); ++b) s += hist[b];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {      // inclusive Hillis-Steele scan
        const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t acc = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (int b = b0; b < min(b0 + per, nbins); ++b) {
        base[b] = acc;
        acc += hist[b];
    }
    __syncthreads();
    if (threadIdx.x <= nchunks) {
        const int b = threadIdx.x * kChunkBins;
        bounds[threadIdx.x] = threadIdx.x == nchunks ? part[1023] : base[b];
    }
}

__global__ void chunk_scatter_kernel(const fa_job *__restrict__ jobs, uint32_t n, const ChunkEnds ends,
                                     int nchunks, const uint32_t *__restrict__ base, uint32_t *__restrict__ cursor,
                                     uint32_t *__restrict__ order)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int bin = -1;
    if (i < n) {
        const fa_job jb = jobs[i];
        bin = chunk_of(jb, ends, nchunks) * kChunkBins + (FA_MAX_QLEN - jb.qlen);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (bin < 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (lane == leader) pos = atomicAdd(&cursor[bin], (uint32_t)__popc(peers));
    pos = __shfl_sync(peers, pos, leader);
    order[base[bin] + pos + __popc(peers & ((1u << lane) - 1u))] = i;
}

size_t chunk_scratch_bytes(int nchunks) { return sizeof(uint32_t) * (3 * (size_t)nchunks * kChunkBins + 64); }

// scratch layout: hist[nbins] | base[nbins] | cursor[nbins] | info[4] | bounds[nchunks+1] |
// lowest job index per chunk[nchunks] | highest[nchunks]
cudaError_t launch_chunk_prep(const fa_job *d_jobs, uint32_t n, uint64_t qbytes, uint64_t tbytes, const ChunkEnds &ends,
                              int nchunks, int max_score, int h0_min, int qcap_limit, uint32_t *d_scratch,
                              cudaStream_t s)
{
    if (nchunks < 1 || nchunks > kMaxChunks) return cudaErrorInvalidValue;
    const size_t nbins = (size_t)nchunks * kChunkBins;
    uint32_t *hist = d_scratch, *cursor = d_scratch + 2 * nbins, *info = d_scratch + 3 * nbins;
    if (4 + 3 * (size_t)nchunks + 1 > 64) return cudaErrorInvalidValue;   // the 64 words past the bins
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * nbins, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * nbins, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(info, 0, sizeof(uint32_t) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(info + 1, 0xFF, sizeof(uint32_t), s);   // first bad job: none
    if (e == cudaSuccess) e = cudaMemsetAsync(info + 4 + nchunks + 1, 0xFF, sizeof(uint32_t) * nchunks, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(info + 4 + 2 * nchunks + 1, 0, sizeof(uint32_t) * nchunks, s);
    if (e != cudaSuccess || n == 0) return e;
    chunk_prep_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, qbytes, tbytes, ends, nchunks, max_score,
                                                      h0_min, qcap_limit, hist, info);
    chunk_scan_kernel<<<1, 1024, 0, s>>>(hist, (int)nbins, d_scratch + nbins, nchunks, info + 4);
    return cudaGetLastError();
}

cudaError_t launch_chunk_scatter(const fa_job *d_jobs, uint32_t n, const ChunkEnds &ends, int nchunks,
                                 uint32_t *d_scratch, uint32_t *d_order, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const size_t nbins = (size_t)nchunks * kChunkBins;
    if (nchunks < 1 || nchunks > kMaxChunks) return cudaErrorInvalidValue;
    chunk_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, ends, nchunks, d_scratch + nbins,
                                                         d_scratch + 2 * nbins, d_order);
    return cudaGetLastError();
}

}  // namespace fa

namespace fa {

// ------------------------------------------------------------- streamed host batches
// A streamed host batch is cut by job index: slice k is jobs [J_k, J_k+1), uploaded with
// the sequence bytes up to its resident ends, so a slice can start as soon as its own
// records and bytes have arrived.  Per slice, on the device: every job validated (the rules
// of chunk_prep_kernel), a valid job whose query or target ends past the resident ends
// counted as not resident (the host then takes the batch to another path), the rest
// ordered longest query first (local indices).  info = {status, first bad job (local),
// longest query, widest band, 0, listed jobs, jobs not resident, 0}.

// bin of a job in the slice's length order, or -1 (invalid, or not resident); *st gets the
// job's status bits
__device__ __forceinline__ int slice_bin(const fa_job &jb, uint64_t qpos, uint64_t tpos, uint64_t q_res,
                                         uint64_t t_res, int max_score, int h0_min, int qcap_limit, uint32_t *st,
                                         bool *resident) {
    uint32_t s = 0;
    if (jb.qlen <= 0 || jb.tlen < 0 || jb.h0 < h0_min) s |= ST_ARG;
    else if (jb.qlen > FA_MAX_QLEN || jb.tlen > FA_MAX_TLEN) s |= ST_CAPACITY;
    else if (jb.q_off + (uint64_t)jb.qlen > qpos || jb.t_off + (uint64_t)jb.tlen > tpos) s |= ST_ARG;
    else if ((int64_t)jb.h0 + (int64_t)max_score * jb.qlen > kPackedHMax || jb.qlen > qcap_limit)
        s |= ST_CAPACITY;
    *st = s;
    *resident = jb.q_off + (uint64_t)jb.qlen <= q_res && jb.t_off + (uint64_t)jb.tlen <= t_res;
    return s || !*resident ? -1 : FA_MAX_QLEN - jb.qlen;
}

__global__ void slice_prep_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint64_t qpos, uint64_t tpos,
                                  uint64_t q_res, uint64_t t_res, int max_score, int h0_min, int qcap_limit,
                                  uint32_t *__restrict__ hist, uint32_t *__restrict__ info)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int bin = -1, qlen = 0, band = 0;
    bool away = false;
    if (i < n) {
        const fa_job jb = jobs[i];
        uint32_t st = 0;
        bool resident = true;
        bin = slice_bin(jb, qpos, tpos, q_res, t_res, max_score, h0_min, qcap_limit, &st, &resident);
        if (st) {
            atomicOr(&info[0], st);
            atomicMin(&info[1], i);
        } else {
            qlen = jb.qlen;
            band = max(jb.w, 0);
            away = !resident;
        }
    }
    const unsigned aw = __ballot_sync(0xffffffffu, away);
    if ((threadIdx.x & 31) == 0 && aw) atomicAdd(&info[6], (uint32_t)__popc(aw));
    const int mq = __reduce_max_sync(0xffffffffu, qlen);
    if ((threadIdx.x & 31) == 0 && mq > 0) atomicMax(&info[2], (uint32_t)mq);
    const int mw = __reduce_max_sync(0xffffffffu, band);
    if ((threadIdx.x & 31) == 0 && mw > 0) atomicMax(&info[3], (uint32_t)mw);
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (bin >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
}

__global__ void slice_scatter_kernel(const fa_job *__restrict__ jobs, uint32_t n, uint64_t qpos, uint64_t tpos,
                                     uint64_t q_res, uint64_t t_res, int max_score, int h0_min, int qcap_limit,
                                     const uint32_t *__restrict__ base, uint32_t *__restrict__ cursor,
                                     uint32_t *__restrict__ order)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    int bin = -1;
    if (i < n) {
        uint32_t st = 0;
        bool resident = true;
        bin = slice_bin(jobs[i], qpos, tpos, q_res, t_res, max_score, h0_min, qcap_limit, &st, &resident);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (bin < 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (lane == leader) pos = atomicAdd(&cursor[bin], (uint32_t)__popc(peers));
    pos = __shfl_sync(peers, pos, leader);
    order[base[bin] + pos + __popc(peers & ((1u << lane) - 1u))] = i;
}

size_t slice_scratch_words(int nslices) { return (size_t)nslices * (3 * (size_t)kChunkBins + 8); }

// scratch (slice_scratch_words(1) words): hist | base | cursor (kChunkBins each) | info[8]
cudaError_t launch_slice_prep(const fa_job *d_jobs, uint32_t n, uint64_t qpos, uint64_t tpos, uint64_t q_res,
                              uint64_t t_res, int max_score, int h0_min, int qcap_limit, uint32_t *d_scratch,
                              uint32_t *d_order, cudaStream_t s)
{
    uint32_t *hist = d_scratch, *base = d_scratch + kChunkBins, *cursor = d_scratch + 2 * kChunkBins;
    uint32_t *info = d_scratch + 3 * kChunkBins;
    cudaError_t e = cudaMemsetAsync(d_scratch, 0, sizeof(uint32_t) * slice_scratch_words(1), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(info + 1, 0xFF, sizeof(uint32_t), s);   // first bad job: none
    if (e != cudaSuccess || n == 0) return e;
    slice_prep_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, qpos, tpos, q_res, t_res, max_score, h0_min,
                                                      qcap_limit, hist, info);
    // one bin group: bounds = {0, listed jobs} at info[4], info[5]
    chunk_scan_kernel<<<1, 1024, 0, s>>>(hist, kChunkBins, base, 1, info + 4);
    slice_scatter_kernel<<<(n + 255) / 256, 256, 0, s>>>(d_jobs, n, qpos, tpos, q_res, t_res, max_score, h0_min,
                                                         qcap_limit, base, cursor, d_order);
    return cudaGetLastError();
}

}  // namespace fa
