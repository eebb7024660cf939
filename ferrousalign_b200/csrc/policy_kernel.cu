// policy_kernel.cu -- device-side band-retry decisions between extension rounds.
//
// Plain policy (bwa-mem2 mem_chain2aln): try band w << k for k < max_tries; stop when
// the score equals the previous try's (initially 0 for a left extension, h0 for a
// right one) or max_off < (w>>1) + (w>>2).  The reference itself runs a single
// ksw_extend2 per job (src/pipelines/linear/batch_extension/dispatch.rs:31-86), which
// is the max_tries = 1 case.
//
// Learned policy: start at a predicted narrow band and double it while it is below
// the configured band.  A narrow run is accepted when its band clamp never bound
// (then every wider band reproduces it exactly) or, with FA_JUDGE_MAXOFF, when it
// also passes the bwa-mem2 max_off test; otherwise the job continues on the ladder
// and finally falls back to the plain policy at the configured band.
//
// The decisions compact the jobs that need another run into a list whose length
// stays on the device, so a retry round needs no host round trip.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

__global__ void policy_init_kernel(const fa_job *__restrict__ jobs, uint32_t n,
                                   const int32_t *__restrict__ w_first, int w_min, int learned,
                                   PolicyState st)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const fa_job jb = jobs[i];
    int w = jb.w, k = 0;
    if (learned) {
        w = w_first ? w_first[i] : jb.w;
        if (w < w_min) w = w_min;
        if (w < jb.w) k = -1; else w = jb.w;
    }
    st.w_cur[i] = w;
    st.k[i] = k;
    st.prev[i] = jb.dir == FA_DIR_RIGHT ? jb.h0 : 0;
    st.w_final[i] = w;
    st.tries[i] = 0;
    if (st.missed) st.missed[i] = 0;
}

__global__ void policy_step_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ list,
                                   const uint32_t *__restrict__ count, uint32_t n_max,
                                   const fa_ext_result *__restrict__ out,
                                   const uint8_t *__restrict__ clamped, PolicyState st, int max_tries,
                                   int judge, uint32_t *__restrict__ next, uint32_t *__restrict__ next_count)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = count ? min(*count, n_max) : n_max;
    bool again = false;
    uint32_t jid = 0;
    if (t < n) {
        jid = list[t];
        const fa_job jb = jobs[jid];
        const fa_ext_result r = out[jid];
        int w = st.w_cur[jid], k = st.k[jid];
        st.tries[jid] += 1;
        st.w_final[jid] = w;
        if (k < 0) {   // learned narrow ladder
            bool ok = !clamped[jid];
            if (!ok && (judge & FA_JUDGE_MAXOFF)) ok = r.max_off < (w >> 1) + (w >> 2);
            if (!ok) {
                if (st.missed && st.tries[jid] == 1) st.missed[jid] = 1;
                w <<= 1;
                if (w >= jb.w) { w = jb.w; k = 0; }
                st.w_cur[jid] = w;
                st.k[jid] = k;
                again = true;
            }
        } else {       // bwa-mem2 ladder at w << k
            const bool stop = r.score == st.prev[jid] || r.max_off < (w >> 1) + (w >> 2);
            if (!stop && k + 1 < max_tries) {
                st.prev[jid] = r.score;
                st.k[jid] = k + 1;
                st.w_cur[jid] = jb.w << (k + 1);
                again = true;
            }
        }
    }
    // warp-aggregated append to the next list
    const unsigned mask = __ballot_sync(0xffffffffu, again);
    if (mask) {
        const int lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == __ffs(mask) - 1) base = atomicAdd(next_count, (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
        if (again) next[base + __popc(mask & ((1u << lane) - 1u))] = jid;
    }
}

cudaError_t launch_policy_init(const fa_job *d_jobs, uint32_t n, const int32_t *d_w_first, int w_min,
                               int learned, PolicyState st, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    policy_init_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_jobs, n, d_w_first, w_min, learned, st);
    return cudaGetLastError();
}

cudaError_t launch_policy_step(const fa_job *d_jobs, const uint32_t *d_list, const uint32_t *d_count,
                               uint32_t n_max, const fa_ext_result *d_out, const uint8_t *d_clamped,
                               PolicyState st, int max_tries, int judge, uint32_t *d_next,
                               uint32_t *d_next_count, cudaStream_t stream)
{
    if (n_max == 0) return cudaSuccess;
    policy_step_kernel<<<(n_max + 255) / 256, 256, 0, stream>>>(d_jobs, d_list, d_count, n_max, d_out,
                                                               d_clamped, st, max_tries, judge, d_next,
                                                               d_next_count);
    return cudaGetLastError();
}

}  // namespace fa
