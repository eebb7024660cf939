// noalloc.cu -- device-resident seed extension that allocates no device memory.
//
// fa_ext_batch_device needs scratch memory besides its inputs and outputs: the
// query-length histogram, the longest-first job order and a status word.  It keeps
// them in buffers its context allocates with cudaMalloc.  Some callers cannot let a
// library do that: processes whose device memory is owned by a pool allocator (a
// framework's caching allocator, RMM) that must see every allocation, services that run
// under a fixed device-memory budget, and latency-critical paths where an allocation
// (and the implicit synchronisation of cudaFree) is not allowed.  This entry point keeps
// that scratch in one file-scope __device__ array instead, so it needs neither a context
// nor any allocation; the caller still passes the inputs and the output buffer.
//
// The array holds at most FA_NOALLOC_MAX_JOBS job indices (about 1 MiB in total) and
// stays resident on every GPU that loads the library until the process exits.

#include <cstdio>
#include <cstring>
#include <mutex>

#include "fa_kernels.h"

namespace fa {
namespace {

constexpr int kHistWords = FA_MAX_QLEN + 1;

// Layout of the scratch array.
struct NoAllocScratch {
    uint32_t status[64];                 // [0] = kernel status word; padded to 256 bytes
    uint32_t hist[(kHistWords + 63) / 64 * 64];
    uint32_t order[FA_NOALLOC_MAX_JOBS];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
NoAllocScratch *g_scratch[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};
int g_smem_optin[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The host-side symbol
// is only a stand-in, so the address comes from cudaGetSymbolAddress, once per device
// with that device current.
int scratch_for_current_device(NoAllocScratch **out, int *sm_count, int *smem_optin) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_last_error(FA_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_last_error(FA_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_last_error(FA_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch array failed");
        int sms = 0, optin = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            return set_last_error(FA_ERR_CUDA, "device attribute query failed");
        g_sm_count[dev] = sms;
        g_smem_optin[dev] = optin;
        g_scratch[dev] = static_cast<NoAllocScratch *>(p);
    }
    *out = g_scratch[dev];
    *sm_count = g_sm_count[dev];
    *smem_optin = g_smem_optin[dev];
    return FA_OK;
}

#define NA_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            char m_[256];                                                              \
            snprintf(m_, sizeof(m_), "%s failed: %s", #call, cudaGetErrorString(e_));  \
            return set_last_error(FA_ERR_CUDA, m_);                                    \
        }                                                                              \
    } while (0)

}  // namespace
}  // namespace fa

using namespace fa;

extern "C" int fa_ext_batch_device_noalloc(const fa_params *p, const fa_job *d_jobs, uint32_t n,
                                           const uint8_t *d_qseq, const uint8_t *d_tseq,
                                           fa_ext_result *d_out, void *stream)
{
    if (!p) return set_last_error(FA_ERR_ARG, "null params");
    if (p->m != 5) return set_last_error(FA_ERR_ARG, "alphabet size must be 5");
    if (p->o_del < 0 || p->e_del < 0 || p->o_ins < 0 || p->e_ins < 0)
        return set_last_error(FA_ERR_ARG, "negative gap penalties are not supported");
    if (n == 0) return FA_OK;
    if (n > FA_NOALLOC_MAX_JOBS) {
        char m[160];
        snprintf(m, sizeof(m), "fa_ext_batch_device_noalloc: %u jobs exceed the limit of %u per call "
                 "(split the batch)", n, (unsigned)FA_NOALLOC_MAX_JOBS);
        return set_last_error(FA_ERR_CAPACITY, m);
    }
    if (!d_jobs || !d_qseq || !d_tseq || !d_out) return set_last_error(FA_ERR_ARG, "null buffer");

    NoAllocScratch *sc = nullptr;
    int sm_count = 0, smem_optin = 0;
    if (int rc = scratch_for_current_device(&sc, &sm_count, &smem_optin)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    ExtParams kp;
    memcpy(kp.mat, p->mat, 25);
    kp.m = p->m;
    kp.o_del = p->o_del; kp.e_del = p->e_del; kp.o_ins = p->o_ins; kp.e_ins = p->e_ins;
    kp.zdrop = p->zdrop; kp.end_bonus = p->end_bonus;
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (p->mat[i] > (int8_t)ms) ms = p->mat[i];
    kp.max_score = ms;
    kp.flags = p->flags;

    // Every call reuses the array: clear the status word.  The histogram is cleared by its
    // launcher, and the scatter rewrites the first n order slots, each exactly once: the
    // histogram and the scatter put every job in the same bin (qlen_bin, invalid lengths
    // included), so no slot keeps an index left by an earlier, larger call.
    NA_CUDA(cudaMemsetAsync(sc->status, 0, sizeof(uint32_t), s));
    NA_CUDA(launch_qlen_hist(d_jobs, n, sc->hist, sm_count, s));
    uint32_t hist[kHistWords];
    NA_CUDA(cudaMemcpyAsync(hist, sc->hist, sizeof(hist), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));

    const int qlimit = (int)(smem_optin / (kExtThreads * sizeof(uint32_t))) - 1;
    uint32_t start[kHistWords];
    uint32_t seg_end[kHistWords / 32 + 2];
    int seg_cap[kHistWords / 32 + 2];
    int nseg = 0, cap = -1;
    uint32_t acc = 0;
    for (int q = FA_MAX_QLEN; q >= 0; --q) {
        start[q] = acc;
        if (!hist[q]) continue;
        if (q > qlimit) {
            char m[128];
            snprintf(m, sizeof(m), "a job has qlen=%d > %d", q, qlimit);
            return set_last_error(FA_ERR_CAPACITY, m);
        }
        if (cap < 0 || q <= ((cap + 31) / 32 - 1) * 32) {
            if (cap >= 0) { seg_cap[nseg] = cap; ++nseg; }
            cap = q;
        }
        acc += hist[q];
        seg_end[nseg] = acc;
    }
    if (cap >= 0) { seg_cap[nseg] = cap; ++nseg; }

    NA_CUDA(cudaMemcpyAsync(sc->hist, start, sizeof(start), cudaMemcpyHostToDevice, s));
    NA_CUDA(launch_qlen_scatter(d_jobs, n, sc->hist, sc->order, s));
    uint32_t b = 0;
    for (int k = 0; k < nseg; ++k) {
        NA_CUDA(launch_ext_packed(d_jobs, sc->order + b, seg_end[k] - b, nullptr, nullptr,
                                  SeqBuf{d_qseq, ~0ull, nullptr, 0, 0}, SeqBuf{d_tseq, ~0ull, nullptr, 0, 0}, kp,
                                  seg_cap[k], 0, nullptr, d_out, nullptr, false, nullptr, nullptr, sc->status, s));
        b = seg_end[k];
    }
    uint32_t st = 0;
    NA_CUDA(cudaMemcpyAsync(&st, sc->status, sizeof(st), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    if (st & ST_BAD_CODE) return set_last_error(FA_ERR_ARG, "a sequence byte is outside the alphabet (codes 0-4)");
    if (st & ST_ARG)
        return set_last_error(FA_ERR_ARG, "a job has h0 <= 0 (h0 < 0 with FA_PARAM_H0_ZERO), qlen <= 0 or tlen < 0");
    if (st & ST_CAPACITY) return set_last_error(FA_ERR_CAPACITY, "a job exceeded the kernel capacity");
    return FA_OK;
}
