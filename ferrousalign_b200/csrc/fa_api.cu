// fa_api.cu -- C ABI of the B200 seed-extension / mate-rescue library.
//
// Host side of the drop-in for execute_batch_simd_scoring
// (src/pipelines/linear/batch_extension/dispatch.rs:31-86) and for the ksw_align2
// calls of execute_mate_rescue_batch_with_engine
// (src/pipelines/linear/paired/mate_rescue.rs:595-685): validation (the reference's
// panics become FA_ERR_ARG), length ordering, device buffers, the band-retry rounds
// and the copies in and out.  There is no CPU fallback: every result comes from the
// CUDA kernels of this library.

#include <algorithm>
#include <chrono>
#include <functional>
#include <map>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <tuple>
#include <vector>

#include "fa_kernels.h"

using namespace fa;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define FA_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(FA_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max(bytes, (size_t)256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Largest query a packed-column launch can hold: (qcap+1) words per thread.
int packed_qcap_limit(size_t smem_optin) {
    return (int)(smem_optin / (kExtThreads * sizeof(uint32_t))) - 1;
}

}  // namespace

int fa::set_last_error(int code, const char *msg) {
    g_err = msg ? msg : "";
    return code;
}

struct fa_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf jobs, order, qseq, tseq, out, clamped, cells_job, misc;
    DevBuf ovf;   // two-row kernel: jobs handed on to the int32 kernel
    DevBuf reg_in, reg_out;   // region merge of host buffers: inputs, regions
    DevBuf col_in, col_plan, col_out;   // job collection: inputs, chain plans + scan sums, outputs
    DevBuf col_pk;                      // packed collection outputs: bases, N runs, run-scan scratch
    DevBuf cg_in, cg_scratch, cg_out;   // CIGAR regeneration: inputs, row state + traceback, outputs
    DevBuf mc_in, mc_plan, mc_out;      // mate-rescue jobs: inputs, plans + scan sums, outputs
    DevBuf is_buf;                      // insert-size statistics: pairs, histogram, results
    DevBuf w_first, w_cur, prev, kk, w_final, tries, missed, list_a, list_b, hist, feat, wbf, part_n, part_w;
    DevBuf part_blk[4];   // band partition scratch (per-block bucket offsets), one per lane
    DevBuf qruns, truns;                // N runs of packed host batches
    DevBuf ref_pac;                     // the resident packed reference (fa_ctx_set_reference)
    uint64_t ref_l_pac = 0;
    // the sequences of the current host call on the device (byte codes or packed bases)
    SeqBuf cq{}, ct{};
    uint32_t last_launches = 0;
    bool timing = false;
    int kernel = FA_KERNEL_AUTO;
    cudaStream_t last_stream = nullptr;   // stream of the last device-resident call
    cudaEvent_t kev0 = nullptr, kev1 = nullptr;   // bracket the extension kernels of a device call
    // learned rounds run their band groups on forked streams: fork on `stream`, join back
    cudaStream_t aux[2] = {nullptr, nullptr};
    cudaEvent_t fork_ev = nullptr, join_ev[2] = {nullptr, nullptr};
    // side streams for the int32 work of two-row launches (the jobs past the 8-bit bound, and
    // classes past the two-row kernel's columns): side[0] takes a multi-class sequence's
    // overflow passes and a retry round's, side[k] learned band group k's; one overflow count
    // per capacity class
    static constexpr int kSides = 3;
    cudaStream_t side[kSides] = {};
    cudaEvent_t side_fork[kSides] = {}, side_join[kSides] = {};
    DevBuf class_ovf_n;
    // a second lane for sliced host batches (alternate slices run concurrently): its own
    // stream, band-group streams and events, and scratch counters
    // (lane 0 is `stream` with misc, aux, fork_ev and join_ev; lanes 1 .. kLanes-1 here)
    static constexpr int kLanes = 4;
    cudaStream_t lane_s[kLanes] = {}, lane_aux[kLanes][2] = {};
    cudaEvent_t lane_fork[kLanes] = {}, lane_join[kLanes][2] = {}, lane_done[kLanes] = {};
    cudaEvent_t lane_ev[2] = {nullptr, nullptr};
    DevBuf lane_misc;   // kMiscBytes per lane
    // paired batches: the mate-rescue half's own buffers, stream and events
    DevBuf pm_jobs, pm_order, pm_q, pm_t, pm_out, pm_misc, pm_rev;
    DevBuf mate_rev;   // the mate SW reverse-pass list (launch_mate_sw)
    DevBuf mate_pk;    // packed mate input: bases and N runs before the unpack
    uint64_t q_bases = 0, t_bases = 0;   // bases of the host call's sequence buffers (cq / ct)
    cudaStream_t pm_stream = nullptr, pm_copy = nullptr;   // the mate half's kernels and uploads
    cudaEvent_t pm_ev0 = nullptr, pm_ev1 = nullptr, pm_fork = nullptr, pm_slice_ev[4] = {};
    // pipelined host batches: slice uploads on their own stream, one event per slice; the
    // same stream then returns each finished slice's results, after its done event
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t slice_ev[8] = {}, done_ev[8] = {}, jobs_ev = nullptr;
    cudaEvent_t span_ev[8][2] = {};   // sliced rounds: each slice's kernels, start and end
    // streamed host batches: the slices' validation on their own stream, one event per slice
    // for its job records uploaded and one for its summary back in pinned host words
    cudaStream_t prep_stream = nullptr;
    cudaEvent_t job_ev[8] = {}, info_ev[8] = {};
    uint32_t *h_slice_info = nullptr;
    void *h_stage = nullptr;   // page-locked staging of host-built arrays (sliced mate orders)
    size_t h_stage_cap = 0;
    // upload slices of pipelined / sliced host batches (0: chosen per batch, auto_slices)
    int slices_single = 0, slices_rounds = 0;
    DevBuf chunk_scratch;
    // kernel choice: fixed, or (FA_KERNEL_AUTO) tuned per (query capacity class, band)
    struct Choice { int kernel; int tpb; };
    int threads = kExtThreads;   // threads per block of the int32 kernel when fixed
    std::map<std::tuple<int, int, int>, Choice> tuned;   // (capacity class, band, packed)
    Choice last_choice{FA_KERNEL_INT32, kExtThreads};
    std::vector<std::pair<Choice, float>> last_tuning;
    // graph mode: the rounds of a call recorded once as a CUDA graph and replayed while the
    // call's shape (key) stays the same
    bool graph = false;
    cudaGraphExec_t gexec = nullptr;
    std::vector<uint64_t> gkey;
    uint32_t glaunches = 0;
};

int fa::fa_ctx_device(const fa_ctx *c) { return c->device; }

namespace {

// misc buffer layout (bytes): [0] status u32, [8] cells u64, [16] count A, [20] count B,
// [232] three u64 statistics sums (kStatsOff),
// [24..35] two-row kernel overflow counts (one per concurrent band group), [40..51] persistent
// two-row launches' job counters (one per overflow slot), [64] band-bucket
// histogram u32[kBandBuckets],
// [128] band-bucket cursors u32[kBandBuckets], [192] band-group bounds u32[3] and the end of
// the configured-band bucket u32
constexpr size_t kMiscBytes = 256;
constexpr size_t kStatsOff = 232;   // 3 x u64, after the band-group bounds at [192, 208)
struct Misc {
    uint32_t *status;
    unsigned long long *cells;
    uint32_t *cnt_a, *cnt_b, *ovf_n, *bucket_hist, *group_bounds;
    uint32_t *work;   // persistent two-row launches' job counters, one per overflow slot
};
Misc misc_at(char *b, char *shared) {
    return Misc{(uint32_t *)shared, (unsigned long long *)(shared + 8), (uint32_t *)(b + 16), (uint32_t *)(b + 20),
                (uint32_t *)(b + 24), (uint32_t *)(b + 64), (uint32_t *)(b + 192), (uint32_t *)(b + 40)};
}
Misc misc_of(fa_ctx *c) {
    char *b = c->misc.as<char>();
    return Misc{(uint32_t *)b, (unsigned long long *)(b + 8), (uint32_t *)(b + 16), (uint32_t *)(b + 20),
                (uint32_t *)(b + 24), (uint32_t *)(b + 64), (uint32_t *)(b + 192), (uint32_t *)(b + 40)};
}

// Lanes 1 .. nl-1 of sliced and streamed host batches: their misc blocks share the status
// word and the cell counter of lane 0 (misc_of), the rest is their own; ms[0] is lane 0's.
int ensure_lanes(fa_ctx *c, int nl, Misc *ms) {
    if (!c->lane_ev[0])
        for (auto &e : c->lane_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    FA_CUDA(c->lane_misc.ensure(kMiscBytes * fa_ctx::kLanes));
    ms[0] = misc_of(c);
    for (int l = 1; l < nl; ++l) {
        if (!c->lane_s[l]) {
            FA_CUDA(cudaStreamCreateWithFlags(&c->lane_s[l], cudaStreamNonBlocking));
            for (int k = 0; k < 2; ++k) {
                FA_CUDA(cudaStreamCreateWithFlags(&c->lane_aux[l][k], cudaStreamNonBlocking));
                FA_CUDA(cudaEventCreateWithFlags(&c->lane_join[l][k], cudaEventDisableTiming));
            }
            FA_CUDA(cudaEventCreateWithFlags(&c->lane_fork[l], cudaEventDisableTiming));
            FA_CUDA(cudaEventCreateWithFlags(&c->lane_done[l], cudaEventDisableTiming));
        }
        ms[l] = misc_at(c->lane_misc.as<char>() + l * kMiscBytes, c->misc.as<char>());
    }
    return FA_OK;
}

cudaStream_t lane_stream(fa_ctx *c, int l) { return l ? c->lane_s[l] : c->stream; }

int ensure_aux_streams(fa_ctx *c) {
    if (c->fork_ev) return FA_OK;
    for (int k = 0; k < 2; ++k) {
        FA_CUDA(cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking));
        FA_CUDA(cudaEventCreateWithFlags(&c->join_ev[k], cudaEventDisableTiming));
    }
    FA_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    return FA_OK;
}

// Extension launch: the int32 one-job-per-thread kernel, the two-rows-per-thread
// int16x2 kernel (bwa-form matrices, queries up to 254 columns; jobs whose scores can pass
// 255 go on to the int32 kernel in the same call), or the two-jobs-per-thread int16x2
// kernel.  All are exact.  With `cert` the int32 kernel also evaluates the exit-bound
// certificate (flag bit 1), which only the int32 kernel implements.
using Choice = fa_ctx::Choice;

// The two-row kernel's overflow list (`words` entries), its count and the persistent
// launch's job counter.
// side / side_ev (optional): the stream the int32 work runs on (the two-row launch's
// overflow jobs, listed ahead of it, or the whole launch when the capacity is past the
// two-row kernel's columns), forked from the launch stream by side_ev.
struct OvfRes {
    uint32_t *list, *count, *work;
    size_t words;
    cudaStream_t side = nullptr;
    cudaEvent_t side_ev = nullptr;
    bool early = true;   // the overflow jobs listed and started ahead of the two-row launch
};

cudaError_t launch_ext_res(fa_ctx *c, Choice kc, const fa_job *d_jobs, const uint32_t *d_order, uint32_t n,
                           const uint32_t *d_n, const SeqBuf &d_q, const SeqBuf &d_t, const ExtParams &kp, int qcap,
                           const int32_t *d_w_try, fa_ext_result *d_out, uint8_t *d_clamped, bool cert,
                           uint32_t *d_cells_job, unsigned long long *d_cells, uint32_t *d_status, cudaStream_t s,
                           const OvfRes &r) {
    if (kc.kernel == FA_KERNEL_ROWS2 && !cert && ext_rows2_eligible(kp, qcap) &&
        ext_rows2_smem_bytes(qcap, kc.tpb, 0) <= c->smem_optin && r.words >= (size_t)n && r.list)
        return launch_ext_rows2(d_jobs, d_order, n, nullptr, d_n, d_q, d_t, kp, qcap, 0, false, d_w_try, d_out,
                                d_clamped, d_cells_job, d_cells, d_status, r.list, r.count, s, kc.tpb, r.work,
                                r.side, r.side_ev, r.early);
    if (kc.kernel == FA_KERNEL_INT16X2 && ext_pair_eligible(kp) && !cert && !d_q.packed)
        return launch_ext_pair(d_jobs, d_order, n, d_n, d_q, d_t, kp, qcap, d_w_try, d_out, d_clamped,
                               d_cells_job, d_cells, d_status, s);
    if (r.side && qcap > kRows2MaxQ) {
        cudaError_t e = cudaEventRecord(r.side_ev, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(r.side, r.side_ev, 0);
        if (e != cudaSuccess) return e;
        s = r.side;
    }
    return launch_ext_packed(d_jobs, d_order, n, nullptr, d_n, d_q, d_t, kp, qcap, 0, d_w_try, d_out, d_clamped,
                             cert, d_cells_job, d_cells, d_status, s, kc.tpb);
}

// `slot` (0-2) picks the two-row kernel's overflow list and count, so launches that may run
// concurrently use different ones; each list holds a third of the buffer.
// `side`: the int32 work on the first side stream (ensure_side), joined back before the return.
cudaError_t launch_ext(fa_ctx *c, Choice kc, const fa_job *d_jobs, const uint32_t *d_order, uint32_t n,
                       const uint32_t *d_n, const SeqBuf &d_q, const SeqBuf &d_t, const ExtParams &kp, int qcap,
                       const int32_t *d_w_try, fa_ext_result *d_out, uint8_t *d_clamped, bool cert,
                       uint32_t *d_cells_job, unsigned long long *d_cells, uint32_t *d_status, cudaStream_t s,
                       int slot = 0, bool side = false) {
    const size_t ovf_words = c->ovf.cap / (3 * sizeof(uint32_t));
    OvfRes r{c->misc.p ? c->ovf.as<uint32_t>() + slot * ovf_words : nullptr,
             c->misc.p ? misc_of(c).ovf_n + slot : nullptr, c->misc.p ? misc_of(c).work + slot : nullptr, ovf_words};
    side = side && c->side[0];
    if (side) {
        r.side = c->side[0];
        r.side_ev = c->side_fork[0];
        cudaError_t e = cudaEventRecord(c->side_fork[0], s);   // the side stream joins any capture here
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->side[0], c->side_fork[0], 0);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = launch_ext_res(c, kc, d_jobs, d_order, n, d_n, d_q, d_t, kp, qcap, d_w_try, d_out, d_clamped,
                                   cert, d_cells_job, d_cells, d_status, s, r);
    if (e != cudaSuccess || !side) return e;
    e = cudaEventRecord(c->side_join[0], c->side[0]);
    return e == cudaSuccess ? cudaStreamWaitEvent(s, c->side_join[0], 0) : e;
}

// Kernel launches one launch_ext call makes (the two-row kernel adds its overflow pass).
uint32_t ext_kernels_of(fa_ctx *c, Choice kc, const ExtParams &kp, int qcap) {
    return kc.kernel == FA_KERNEL_ROWS2 && ext_rows2_eligible(kp, qcap) &&
                   ext_rows2_smem_bytes(qcap, kc.tpb, 0) <= c->smem_optin ? 2u : 1u;
}

// The side stream, its events and one overflow count per capacity class (outside any
// capture: it may allocate).
int ensure_side(fa_ctx *c, size_t classes) {
    for (int k = 0; k < fa_ctx::kSides; ++k)
        if (!c->side[k]) {
            FA_CUDA(cudaStreamCreateWithFlags(&c->side[k], cudaStreamNonBlocking));
            FA_CUDA(cudaEventCreateWithFlags(&c->side_fork[k], cudaEventDisableTiming));
            FA_CUDA(cudaEventCreateWithFlags(&c->side_join[k], cudaEventDisableTiming));
        }
    FA_CUDA(c->class_ovf_n.ensure(sizeof(uint32_t) * std::max<size_t>(classes, 64)));
    return FA_OK;
}

// Forks (join = false) or joins the side streams to / from s.
cudaError_t side_link(fa_ctx *c, cudaStream_t s, bool join) {
    for (int k = 0; k < fa_ctx::kSides; ++k) {
        cudaEvent_t ev = join ? c->side_join[k] : c->side_fork[k];
        cudaError_t e = cudaEventRecord(ev, join ? c->side[k] : s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(join ? s : c->side[k], ev, 0);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The capacity classes of a length-sorted order (segs: each class's end and capacity, longest
// first), one launch each on stream s.  With several classes the int32 work -- each two-row
// launch's overflow pass (its own list in the overflow buffer at the class's offset, its own
// count) and every class past the two-row kernel's columns -- runs on one side stream, so the
// longest jobs, a few warps per SM whose time is set by their own latency, overlap the shorter
// classes' launches instead of following each of them; the side stream joins s at the end.
// The passes follow their two-row launches (not listed ahead) and take one stream in turn: a
// persistent launch sharing the GPU with early or concurrent passes cannot finish, and so
// start the next class, before those passes free its slots (13.8 against 13.4 ms on 2M
// 50-300 bp jobs).
cudaError_t launch_classes(fa_ctx *c, const std::vector<std::pair<uint32_t, int>> &segs,
                           const std::function<Choice(size_t)> &kc_of, const fa_job *d_jobs,
                           const uint32_t *d_order, const SeqBuf &d_q, const SeqBuf &d_t, const ExtParams &kp,
                           const int32_t *d_w_try, fa_ext_result *d_out, uint8_t *d_flags, bool cert,
                           uint32_t *d_cells_job, unsigned long long *d_cells, uint32_t *d_status, cudaStream_t s,
                           uint32_t *launches) {
    const bool side = segs.size() > 1 && c->side[0] && c->misc.p &&
                      c->class_ovf_n.cap >= sizeof(uint32_t) * segs.size() &&
                      c->ovf.cap >= sizeof(uint32_t) * (size_t)segs.back().first;
    if (side) {
        // the side streams join the launch sequence (and any capture) from the start
        cudaError_t e = side_link(c, s, false);
        if (e != cudaSuccess) return e;
    }
    const size_t ovf_words = c->ovf.cap / (3 * sizeof(uint32_t));
    uint32_t b = 0;
    for (size_t k = 0; k < segs.size(); ++k) {
        const auto &sg = segs[k];
        const Choice kc = kc_of(k);
        OvfRes r{c->misc.p ? c->ovf.as<uint32_t>() : nullptr, c->misc.p ? misc_of(c).ovf_n : nullptr,
                 c->misc.p ? misc_of(c).work : nullptr, ovf_words};
        if (side) {
            r.list = c->ovf.as<uint32_t>() + b;
            r.count = c->class_ovf_n.as<uint32_t>() + k;
            r.words = sg.first - b;
            r.side = c->side[0];
            r.side_ev = c->side_fork[0];
            r.early = false;   // the next class's launch waits for this one's to finish
        }
        cudaError_t e = launch_ext_res(c, kc, d_jobs, d_order + b, sg.first - b, nullptr, d_q, d_t, kp, sg.second,
                                       d_w_try, d_out, d_flags, cert, d_cells_job, d_cells, d_status, s, r);
        if (e != cudaSuccess) return e;
        if (launches) *launches += ext_kernels_of(c, kc, kp, sg.second);
        b = sg.first;
    }
    return side ? side_link(c, s, true) : cudaSuccess;
}

// The kernel a call runs.  A fixed setting is used as is.  FA_KERNEL_AUTO is an
// autotuner: the first time a (query capacity class of 32 columns, configured band) pair
// is seen, every exact candidate -- the int32 one-job-per-thread kernel with 64, 128 or
// 256 threads per block, and where the scoring allows them the two-rows-per-thread
// kernel with 64 or 128 and the two-jobs-per-thread kernel -- runs twice on the first
// (longest) 393,216 jobs of the call's order, and the fastest is kept for that pair.  All
// candidates give identical results.
// The kernel a fixed setting names (false for FA_KERNEL_AUTO).
bool fixed_choice(fa_ctx *c, Choice *kc) {
    if (c->kernel == FA_KERNEL_INT16X2) *kc = Choice{FA_KERNEL_INT16X2, kPairThreads};
    else if (c->kernel == FA_KERNEL_INT32) *kc = Choice{FA_KERNEL_INT32, c->threads};
    else if (c->kernel == FA_KERNEL_ROWS2) *kc = Choice{FA_KERNEL_ROWS2, c->threads == 128 ? 128 : 64};
    else return false;
    c->last_choice = *kc;
    return true;
}

Choice resolve_choice(fa_ctx *c, const ExtParams &kp, const fa_job *d_jobs, const uint32_t *d_order, uint32_t n,
                      const SeqBuf &d_q, const SeqBuf &d_t, int qcap, int band, fa_ext_result *d_out,
                      uint32_t *d_status, cudaStream_t s, int *rc) {
    *rc = FA_OK;
    Choice fixed;
    if (fixed_choice(c, &fixed)) return fixed;
    const std::tuple<int, int, int> key{(qcap + 31) / 32, band, (int)d_q.packed};
    auto it = c->tuned.find(key);
    if (it != c->tuned.end()) return c->last_choice = it->second;
    std::vector<Choice> cands{{FA_KERNEL_INT32, 64}, {FA_KERNEL_INT32, kExtThreads}, {FA_KERNEL_INT32, 256}};
    if (ext_rows2_eligible(kp, qcap)) {
        cands.push_back({FA_KERNEL_ROWS2, 64});
        cands.push_back({FA_KERNEL_ROWS2, 128});
    }
    if (ext_pair_eligible(kp) && !d_q.packed) cands.push_back({FA_KERNEL_INT16X2, kPairThreads});
    // a sample of several claim rounds of the persistent launch (about 2,700 resident warps of
    // 32 jobs), so the partly used last round does not decide between 64 and 128 threads
    const uint32_t ns = std::min<uint32_t>(n, 393216);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Choice best{FA_KERNEL_INT32, kExtThreads};
    float best_ms = 1e30f;
    c->last_tuning.clear();
    auto bail = [&](cudaError_t e) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        *rc = fail(FA_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
        return best;
    };
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) return bail(e);
    for (const Choice &kc : cands) {
        if (kc.kernel == FA_KERNEL_INT32 && ext_packed_smem_bytes(qcap, 0, kc.tpb) > c->smem_optin) continue;
        if (kc.kernel == FA_KERNEL_INT16X2 && ext_pair_smem_bytes(qcap) > c->smem_optin) continue;
        if (kc.kernel == FA_KERNEL_ROWS2 && (ext_rows2_smem_bytes(qcap, kc.tpb, 0) > c->smem_optin ||
                                             c->ovf.cap < 3 * sizeof(uint32_t) * (size_t)ns))
            continue;
        for (int rep = 0; rep < 3; ++rep) {           // one warm-up, two timed
            if (rep == 1 && (e = cudaEventRecord(e0, s)) != cudaSuccess) return bail(e);
            e = launch_ext(c, kc, d_jobs, d_order, ns, nullptr, d_q, d_t, kp, qcap, nullptr, d_out, nullptr, false,
                           nullptr, nullptr, d_status, s);
            if (e != cudaSuccess) return bail(e);
        }
        if ((e = cudaEventRecord(e1, s)) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess)
            return bail(e);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
        c->last_tuning.push_back({kc, ms});
        if (ms < best_ms) { best_ms = ms; best = kc; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tuned[key] = best;
    return c->last_choice = best;
}

// The kernel of one slice of a streamed host batch: the fixed one, the one tuned for the
// slice's (capacity class, band, form), or one tuned for the same band and form -- the
// nearest capacity class at or above the slice's, else the nearest below (every choice is
// exact; launch_ext falls back where a kernel does not fit).  False when nothing is tuned
// for that band and form.
bool slice_choice(fa_ctx *c, int qcap, int band, bool packed, Choice *kc) {
    if (fixed_choice(c, kc)) return true;
    const int cls = (qcap + 31) / 32;
    auto it = c->tuned.find({cls, band, (int)packed});
    if (it == c->tuned.end()) {
        int best = -1;
        for (auto jt = c->tuned.begin(); jt != c->tuned.end(); ++jt) {
            if (std::get<1>(jt->first) != band || std::get<2>(jt->first) != (int)packed) continue;
            const int kcls = std::get<0>(jt->first);
            const int d = kcls >= cls ? kcls - cls : 1000 + cls - kcls;
            if (best < 0 || d < best) {
                best = d;
                it = jt;
            }
        }
        if (best < 0) return false;
    }
    *kc = c->last_choice = it->second;
    return true;
}

// One learned round over a band-partitioned list: configured-band and wide narrow jobs
// in the full-row kernel, bands 13-24 in the 64-column ring kernel, bands <= 12 in the
// 32-column ring kernel; the three run concurrently on forked streams.  Their launches are
// not persistent: three persistent grids each take every resident slot and so run one
// after the other (measured 5.69 against 5.59 ms for the learned bench batch).  The two-row
// kernels run them where the scoring allows (each group with its own overflow list), the
// int32 kernels otherwise or when int32 is the fixed choice.
// lane 1 (sliced host batches): the second lane's group streams and events, and the overflow
// lists from ovf_off words on.
int launch_learned_round(fa_ctx *c, const fa_job *d_jobs, const uint32_t *d_list, uint32_t n_max,
                         const SeqBuf &d_q, const SeqBuf &d_t, const ExtParams &kp, int qcap,
                         const int32_t *d_w_cur, fa_ext_result *d_out, uint8_t *d_flags, bool cert, Misc &m,
                         cudaStream_t s, uint32_t *launches, int lane = 0, size_t ovf_off = 0,
                         bool narrow_only = false, uint32_t *cells_job = nullptr, bool sides = false) {
    // narrow_only: the configured-band bucket is left out (its jobs run in a later round)
    // sides: each group's int32 jobs, listed ahead of its two-row launch, on a side stream of
    // its own (ensure_side) from the group's start, joined back at the group's end
    if (int rc = ensure_aux_streams(c)) return rc;
    cudaStream_t *aux = lane ? c->lane_aux[lane] : c->aux;
    cudaEvent_t fork_ev = lane ? c->lane_fork[lane] : c->fork_ev, *join_ev = lane ? c->lane_join[lane] : c->join_ev;
    const uint32_t *g = m.group_bounds;
    const bool rows2 = c->kernel != FA_KERNEL_INT32 && ext_rows2_eligible(kp, qcap) &&
                       ext_rows2_smem_bytes(qcap, 64, 0) <= c->smem_optin &&
                       c->ovf.cap >= sizeof(uint32_t) * (ovf_off + 3 * (size_t)n_max);
    if (!cells_job) cells_job = c->cells_job.as<uint32_t>();
    sides = sides && rows2 && c->side[0];
    auto group = [&](int k, int ring, cudaStream_t st) -> cudaError_t {
        // narrow_only: group 0 starts after the configured-band bucket (g[3])
        const uint32_t *first = k == 0 ? (narrow_only ? g + 3 : nullptr) : g + k - 1;
        if (rows2 && sides) {
            cudaError_t e = cudaEventRecord(c->side_fork[k], st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(c->side[k], c->side_fork[k], 0);
            if (e == cudaSuccess)
                e = launch_ext_rows2(d_jobs, d_list, n_max, first, g + k, d_q, d_t, kp, qcap, ring, cert, d_w_cur,
                                     d_out, d_flags, cells_job, m.cells, m.status,
                                     c->ovf.as<uint32_t>() + ovf_off + (size_t)k * n_max, m.ovf_n + k, st, 64,
                                     nullptr, c->side[k], c->side_fork[k]);
            if (e == cudaSuccess) e = cudaEventRecord(c->side_join[k], c->side[k]);
            return e == cudaSuccess ? cudaStreamWaitEvent(st, c->side_join[k], 0) : e;
        }
        if (rows2)
            return launch_ext_rows2(d_jobs, d_list, n_max, first, g + k, d_q, d_t, kp, qcap, ring, cert, d_w_cur,
                                    d_out, d_flags, cells_job, m.cells, m.status,
                                    c->ovf.as<uint32_t>() + ovf_off + (size_t)k * n_max, m.ovf_n + k, st, 64);
        return launch_ext_packed(d_jobs, d_list, n_max, first, g + k, d_q, d_t, kp, qcap, ring, d_w_cur, d_out,
                                 d_flags, cert, cells_job, m.cells, m.status, st);
    };
    FA_CUDA(cudaEventRecord(fork_ev, s));
    FA_CUDA(group(0, 0, s));
    const int rings[2] = {64, 32};
    for (int k = 0; k < 2; ++k) {
        FA_CUDA(cudaStreamWaitEvent(aux[k], fork_ev, 0));
        FA_CUDA(group(k + 1, rings[k], aux[k]));
        FA_CUDA(cudaEventRecord(join_ev[k], aux[k]));
        FA_CUDA(cudaStreamWaitEvent(s, join_ev[k], 0));
    }
    *launches += rows2 ? (sides ? 9 : 6) : 3;
    return FA_OK;
}

int check_params(const fa_params *p) {
    if (!p) return fail(FA_ERR_ARG, "null params");
    if (p->m != 5) return fail(FA_ERR_ARG, "alphabet size m=%d unsupported (must be 5)", p->m);
    if (p->o_del < 0 || p->e_del < 0 || p->o_ins < 0 || p->e_ins < 0)
        return fail(FA_ERR_ARG, "negative gap penalties are not supported");
    return FA_OK;
}

ExtParams ext_params_of(const fa_params *p) {
    ExtParams k;
    memset(&k, 0, sizeof(k));   // padding too: graph keys compare the raw words
    memcpy(k.mat, p->mat, 25);
    k.m = p->m;
    k.o_del = p->o_del; k.e_del = p->e_del; k.o_ins = p->o_ins; k.e_ins = p->e_ins;
    k.zdrop = p->zdrop; k.end_bonus = p->end_bonus;
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (p->mat[i] > (int8_t)ms) ms = p->mat[i];
    k.max_score = ms;
    k.flags = p->flags;
    return k;
}

// Validation mirrors the reference's panics (h0 <= 0 asserts at ksw_affine_gap.rs:968,
// unless FA_PARAM_H0_ZERO lifts the assert for h0 == 0; out-of-range slices) and this
// library's limits.
int check_jobs(const fa_job *jobs, uint32_t n, uint64_t qlen_buf, uint64_t tlen_buf,
               const ExtParams &k, int qcap_limit, int *max_qlen) {
    int mq = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const fa_job &j = jobs[i];
        if (j.qlen <= 0) return fail(FA_ERR_ARG, "job %u: qlen=%d must be > 0", i, j.qlen);
        if (j.tlen < 0) return fail(FA_ERR_ARG, "job %u: tlen=%d must be >= 0", i, j.tlen);
        if (j.h0 < 0 || (j.h0 == 0 && !(k.flags & FA_PARAM_H0_ZERO)))
            return fail(FA_ERR_ARG, "job %u: h0=%d must be > 0 (or 0 with FA_PARAM_H0_ZERO)", i, j.h0);
        if (j.qlen > FA_MAX_QLEN || j.tlen > FA_MAX_TLEN)
            return fail(FA_ERR_CAPACITY, "job %u: lengths %d/%d exceed %d/%d", i, j.qlen, j.tlen,
                        FA_MAX_QLEN, FA_MAX_TLEN);
        if (j.q_off + (uint64_t)j.qlen > qlen_buf || j.t_off + (uint64_t)j.tlen > tlen_buf)
            return fail(FA_ERR_ARG, "job %u: sequence range outside the buffers", i);
        if ((int64_t)j.h0 + (int64_t)k.max_score * j.qlen > kPackedHMax)
            return fail(FA_ERR_CAPACITY, "job %u: h0 + max(mat)*qlen = %lld exceeds %d", i,
                        (long long)j.h0 + (long long)k.max_score * j.qlen, kPackedHMax);
        if (j.qlen > qcap_limit)
            return fail(FA_ERR_CAPACITY, "job %u: qlen=%d exceeds %d", i, j.qlen, qcap_limit);
        mq = std::max(mq, j.qlen);
    }
    *max_qlen = mq;
    return FA_OK;
}

// Counting sort by query length, longest first; returns [begin,end) segments of
// the order that share a shared-memory capacity class.
void length_order(const fa_job *jobs, uint32_t n, std::vector<uint32_t> &order,
                  std::vector<std::pair<uint32_t, int>> &segs) {
    std::vector<uint32_t> cnt(FA_MAX_QLEN + 2, 0);
    for (uint32_t i = 0; i < n; ++i) cnt[jobs[i].qlen]++;
    std::vector<uint32_t> start(FA_MAX_QLEN + 2, 0);
    uint32_t acc = 0;
    for (int q = FA_MAX_QLEN; q >= 0; --q) { start[q] = acc; acc += cnt[q]; }
    order.resize(n);
    for (uint32_t i = 0; i < n; ++i) order[start[jobs[i].qlen]++] = i;
    // capacity classes: multiples of 32 columns
    segs.clear();
    uint32_t b = 0;
    while (b < n) {
        const int q = jobs[order[b]].qlen;
        const int cap = (q + 31) / 32 * 32;
        uint32_t e = b;
        while (e < n && jobs[order[e]].qlen > cap - 32) ++e;
        segs.push_back({e, std::min(cap, q)});
        b = e;
    }
}

int ensure_ext_buffers(fa_ctx *c, uint32_t n, uint64_t qb, uint64_t tb) {
    FA_CUDA(c->jobs.ensure(sizeof(fa_job) * (size_t)n));
    FA_CUDA(c->order.ensure(sizeof(uint32_t) * (size_t)n));
    FA_CUDA(c->qseq.ensure(qb + kSeqPad));
    FA_CUDA(c->tseq.ensure(tb + kSeqPad));
    FA_CUDA(c->out.ensure(sizeof(fa_ext_result) * (size_t)n));
    FA_CUDA(c->clamped.ensure(n));
    FA_CUDA(c->cells_job.ensure(sizeof(uint32_t) * (size_t)n));
    FA_CUDA(c->ovf.ensure(3 * sizeof(uint32_t) * (size_t)n));
    FA_CUDA(c->misc.ensure(kMiscBytes));
    return FA_OK;
}

int ensure_policy_buffers(fa_ctx *c, uint32_t n) {
    const size_t b = sizeof(int32_t) * (size_t)n;
    FA_CUDA(c->w_first.ensure(b));
    FA_CUDA(c->w_cur.ensure(b));
    FA_CUDA(c->prev.ensure(b));
    FA_CUDA(c->kk.ensure(b));
    FA_CUDA(c->w_final.ensure(b));
    FA_CUDA(c->tries.ensure(b));
    FA_CUDA(c->missed.ensure(n));
    FA_CUDA(c->list_a.ensure(b));
    FA_CUDA(c->list_b.ensure(b));
    FA_CUDA(c->part_n.ensure(b));
    FA_CUDA(c->part_w.ensure(b));
    for (DevBuf &pb : c->part_blk) FA_CUDA(pb.ensure(sizeof(uint32_t) * band_partition_scratch_words(n)));
    return FA_OK;
}

int read_status(fa_ctx *c, cudaStream_t s) {
    uint32_t st = 0;
    FA_CUDA(cudaMemcpyAsync(&st, misc_of(c).status, 4, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (st & ST_BAD_CODE) return fail(FA_ERR_ARG, "a sequence byte is outside the alphabet (codes 0-4)");
    if (st & ST_CAPACITY) return fail(FA_ERR_CAPACITY, "a job exceeded the launch capacity");
    if (st & ST_BLIST) return fail(FA_ERR_CAPACITY, "mate-SW run list overflow");
    if (st & ST_ARG) return fail(FA_ERR_ARG, "a job has h0 <= 0 (h0 < 0 with FA_PARAM_H0_ZERO), qlen <= 0 or tlen < 0");
    if (st & ST_RANGE) return fail(FA_ERR_ARG, "a chain's seed range is malformed");
    if (st & ST_RUNS)
        return fail(FA_ERR_ARG, "a packed buffer's N runs are empty, unsorted, overlapping or outside the bases");
    return FA_OK;
}

// Runs the extension rounds on device data.  order/segs describe the first round;
// retry rounds reuse the widest capacity class.
// Number of extension rounds a call may need: narrow rounds of the learned ladder
// (doubling from w_min up to the widest configured band, or one with FA_JUDGE_ONCE)
// plus the bwa-mem2 tries.
int max_rounds_of(const fa_policy *pol, int max_w) {
    const int mode = pol ? pol->mode : FA_POLICY_SINGLE;
    if (mode == FA_POLICY_SINGLE) return 1;
    const int max_tries = std::max(1, pol->max_tries);
    if (mode != FA_POLICY_LEARNED) return max_tries;
    int narrow = (pol->judge & FA_JUDGE_HINT) && (pol->judge & FA_JUDGE_BOUND) ? 2 : 1;
    if (!(pol->judge & FA_JUDGE_ONCE))
        for (long long w = std::max(1, pol->w_min); w * 2 < max_w && narrow < 13; w *= 2) ++narrow;
    return narrow + max_tries;
}

// Enqueues the extension rounds of one call on stream s.  Without `capture` the host
// reads each round's retry count and stops early when nothing is left; with `capture`
// (recording a CUDA graph) the rounds run a fixed number of times with every count on
// the device, so no round needs the host.  The first round launches once per capacity
// class of the length-sorted order either way.
int enqueue_ext(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, uint32_t n,
                const std::vector<std::pair<uint32_t, int>> &segs, int qcap_all, int max_w, const fa_job *d_jobs,
                const uint32_t *d_order, const SeqBuf &d_q, const SeqBuf &d_t, const int32_t *d_wfirst,
                fa_ext_result *d_out, cudaStream_t s, bool capture, uint32_t *launches, uint32_t *retries,
                Choice kc, const std::vector<Choice> *seg_kc = nullptr, int r_first = 0,
                const uint32_t *list0 = nullptr, const uint32_t *cnt0 = nullptr) {
    // r_first > 0: the rounds before it have run (policy state initialised, their retry list
    // in list0 / *cnt0, which is list_a / cnt_a); go on from round r_first
    Misc m = misc_of(c);
    if (r_first == 0) FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    const int mode = pol ? pol->mode : FA_POLICY_SINGLE;
    const std::vector<std::pair<uint32_t, int>> one_seg{{n, qcap_all}};
    const auto &segs0 = segs.empty() ? one_seg : segs;
    // first-round kernel of each capacity class (tuned per class); retries use kc
    auto kc_of = [&](size_t k) { return seg_kc && k < seg_kc->size() ? (*seg_kc)[k] : kc; };
    if (mode == FA_POLICY_SINGLE) {
        FA_CUDA(launch_classes(c, segs0, kc_of, d_jobs, d_order, d_q, d_t, kp, nullptr, d_out, nullptr, false,
                               c->cells_job.as<uint32_t>(), m.cells, m.status, s, launches));
        return FA_OK;
    }
    PolicyState st{c->w_cur.as<int32_t>(), c->prev.as<int32_t>(), c->kk.as<int32_t>(),
                   c->w_final.as<int32_t>(), c->tries.as<int32_t>(), c->missed.as<uint8_t>()};
    const int learned = mode == FA_POLICY_LEARNED;
    // flags feed the learned judge only; the certificate only its BOUND test
    uint8_t *d_flags = learned ? c->clamped.as<uint8_t>() : nullptr;
    const bool cert = learned && (pol->judge & FA_JUDGE_BOUND);
    if (r_first == 0) {
        FA_CUDA(launch_policy_init(d_jobs, n, d_wfirst, pol->w_min, learned, st, s));
        ++*launches;
    }
    const int max_tries = std::max(1, pol->max_tries);
    // the int32 jobs of every two-row launch start at once on side streams (run_ext and
    // run_ext_graph create them)
    const bool sides = c->side[0] != nullptr;
    const int max_rounds = capture ? max_rounds_of(pol, max_w) : (learned ? 13 : 0) + max_tries;
    const bool once = learned && (pol->judge & FA_JUDGE_ONCE);
    // rounds that can hold narrow runs: the first, and with hints also the second
    const int narrow_rounds = (learned && (pol->judge & FA_JUDGE_HINT) && (pol->judge & FA_JUDGE_BOUND)) ? 2 : 1;
    const uint32_t *list = r_first ? list0 : d_order;
    const uint32_t *cnt = r_first ? cnt0 : nullptr;
    uint32_t *next = c->list_a.as<uint32_t>(), *next_cnt = m.cnt_a;
    uint32_t *spare = c->list_b.as<uint32_t>(), *spare_cnt = m.cnt_b;
    if (r_first) {
        std::swap(next, spare);
        std::swap(next_cnt, spare_cnt);
    }
    for (int r = r_first; r < max_rounds; ++r) {
        // with one narrow try, rounds after the narrow ones hold only plain-policy runs
        const bool cert_r = cert && !(once && r >= narrow_rounds);
        if (r == 0 && !learned) {
            FA_CUDA(launch_classes(c, segs0, kc_of, d_jobs, d_order, d_q, d_t, kp, st.w_cur, d_out, d_flags, cert_r,
                                   c->cells_job.as<uint32_t>(), m.cells, m.status, s, launches));
        } else if (learned && !cert_r && c->kernel != FA_KERNEL_INT16X2) {
            // after the narrow tries every job left runs the plain policy: one launch of the
            // call's autotuned kernel over the compacted list
            FA_CUDA(launch_ext(c, kc, d_jobs, list, n, cnt, d_q, d_t, kp, qcap_all, st.w_cur, d_out, d_flags, false,
                               c->cells_job.as<uint32_t>(), m.cells, m.status, s, 0, sides));
            *launches += ext_kernels_of(c, kc, kp, qcap_all) * (sides ? 2u : 1u) - (sides ? 1u : 0u);
        } else if (learned) {
            // band buckets (configured band first, then narrow bands decreasing), then the
            // three band groups concurrently
            FA_CUDA(launch_band_partition(d_jobs, list, cnt, n, st.w_cur, c->part_n.as<uint32_t>(),
                                          m.bucket_hist, c->part_blk[0].as<uint32_t>(), m.group_bounds, s));
            if (c->kernel == FA_KERNEL_INT16X2) {
                FA_CUDA(launch_ext(c, kc, d_jobs, c->part_n.as<uint32_t>(), n, cnt, d_q, d_t, kp, qcap_all,
                                   st.w_cur, d_out, d_flags, cert_r, c->cells_job.as<uint32_t>(), m.cells,
                                   m.status, s));
                *launches += 3;
            } else {
                if (int rc = launch_learned_round(c, d_jobs, c->part_n.as<uint32_t>(), n, d_q, d_t, kp, qcap_all,
                                                  st.w_cur, d_out, d_flags, cert_r, m, s, launches, 0, 0, false,
                                                  nullptr, sides))
                    return rc;
                *launches += 2;   // band histogram and scatter
            }
        } else {
            FA_CUDA(launch_ext(c, kc, d_jobs, list, n, cnt, d_q, d_t, kp, qcap_all, st.w_cur, d_out,
                               d_flags, cert_r, c->cells_job.as<uint32_t>(), m.cells, m.status, s, 0, sides));
            *launches += cert_r ? 1u : ext_kernels_of(c, kc, kp, qcap_all) * (sides ? 2u : 1u) - (sides ? 1u : 0u);
        }
        FA_CUDA(cudaMemsetAsync(next_cnt, 0, 4, s));
        FA_CUDA(launch_policy_step(d_jobs, list, nullptr, cnt, n, d_out, d_flags, st, max_tries,
                                   pol->judge, next, next_cnt, s));
        ++*launches;
        if (!capture) {
            uint32_t h_cnt = 0;
            FA_CUDA(cudaMemcpyAsync(&h_cnt, next_cnt, 4, cudaMemcpyDeviceToHost, s));
            FA_CUDA(cudaStreamSynchronize(s));
            if (h_cnt == 0) break;
            if (retries) *retries += h_cnt;
        }
        list = next; cnt = next_cnt;
        std::swap(next, spare);
        std::swap(next_cnt, spare_cnt);
    }
    return FA_OK;
}

// Status word, statistics and final bands of the call whose work ev0..ev1 bracket.
// `retries_from_tries`: count retries from the per-job run counts (graph replays, where
// the host saw no round).
int finish_ext(fa_ctx *c, const fa_policy *pol, uint32_t n, cudaStream_t s, fa_ext_stats *stats,
               int32_t *h_wfinal, uint32_t launches, uint32_t retries, bool retries_from_tries) {
    Misc m = misc_of(c);
    const int mode = pol ? pol->mode : FA_POLICY_SINGLE;
    // the N runs of packed host buffers are checked on the device, after the rounds (which
    // read them without faulting whatever they hold): a bad list fails the call
    for (const auto &[buf, nb] : {std::pair<const SeqBuf *, uint64_t>{&c->cq, c->q_bases}, {&c->ct, c->t_bases}})
        if (buf->packed && buf->n_runs) FA_CUDA(launch_runs_check(buf->runs, buf->n_runs, nb, m.status, s));
    if (int rc = read_status(c, s)) return rc;
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        // the per-job counts summed on the device: one read of four words
        const bool tries = retries_from_tries && mode != FA_POLICY_SINGLE;
        const bool missed = mode == FA_POLICY_LEARNED;
        unsigned long long *d_sums = reinterpret_cast<unsigned long long *>(c->misc.as<char>() + kStatsOff);
        FA_CUDA(launch_stats_sum(c->cells_job.as<uint32_t>(), tries ? c->tries.as<int32_t>() : nullptr,
                                 missed ? c->missed.as<uint8_t>() : nullptr, n, d_sums, c->sm_count, s));
        unsigned long long h[4];
        FA_CUDA(cudaMemcpyAsync(h, m.cells, 8, cudaMemcpyDeviceToHost, s));
        FA_CUDA(cudaMemcpyAsync(h + 1, d_sums, 24, cudaMemcpyDeviceToHost, s));
        FA_CUDA(cudaStreamSynchronize(s));
        stats->cells_executed = h[0];
        stats->kernel_ms = ms;
        stats->kernel_launches = launches;
        stats->jobs = n;
        stats->cells = h[1];
        stats->retries = tries ? (uint32_t)(h[2] - n) : retries;
        if (missed) stats->misses = (uint32_t)h[3];
    }
    if (h_wfinal && mode != FA_POLICY_SINGLE)
        FA_CUDA(cudaMemcpy(h_wfinal, c->w_final.p, 4ull * n, cudaMemcpyDeviceToHost));
    return FA_OK;
}

// Runs the extension rounds on device data.  order/segs describe the first round;
// retry rounds reuse the widest capacity class.
int run_ext(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, uint32_t n,
            const std::vector<std::pair<uint32_t, int>> &segs, int qcap_all, int band, const fa_job *d_jobs,
            const uint32_t *d_order, const SeqBuf &d_q, const SeqBuf &d_t, const int32_t *d_wfirst,
            fa_ext_result *d_out, cudaStream_t s, fa_ext_stats *stats, int32_t *h_wfinal) {
    uint32_t launches = 0, retries = 0;
    if (pol && pol->mode != FA_POLICY_SINGLE)
        if (int rc = ensure_policy_buffers(c, n)) return rc;
    if (int rc = ensure_side(c, segs.size())) return rc;
    int rc0 = FA_OK;
    const Choice kc = resolve_choice(c, kp, d_jobs, d_order, n, d_q, d_t, qcap_all, band, d_out, misc_of(c).status, s,
                                     &rc0);
    if (rc0) return rc0;
    // each capacity class gets its own tuned choice (a class the two-row kernel cannot hold
    // does not decide for the others)
    std::vector<Choice> seg_kc;
    {
        uint32_t b = 0;
        for (auto &sg : segs) {
            seg_kc.push_back(resolve_choice(c, kp, d_jobs, d_order + b, sg.first - b, d_q, d_t, sg.second, band, d_out,
                                            misc_of(c).status, s, &rc0));
            if (rc0) return rc0;
            b = sg.first;
        }
        c->last_choice = kc;
    }
    FA_CUDA(cudaEventRecord(c->ev0, s));
    if (int rc = enqueue_ext(c, kp, pol, n, segs, qcap_all, 0, d_jobs, d_order, d_q, d_t, d_wfirst, d_out, s, false,
                             &launches, &retries, kc, &seg_kc))
        return rc;
    FA_CUDA(cudaEventRecord(c->ev1, s));
    return finish_ext(c, pol, n, s, stats, h_wfinal, launches, retries, false);
}

// Everything a recorded graph bakes in: the launch sequence's shape, every scalar passed
// by value, and every buffer address.
std::vector<uint64_t> graph_key(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, uint32_t n, int qcap, int max_w,
                                const std::vector<uint64_t> &extra) {
    std::vector<uint64_t> k{(uint64_t)(pol ? pol->mode : -1), (uint64_t)(pol ? pol->judge : 0),
                            (uint64_t)(pol ? pol->max_tries : 0), (uint64_t)(pol ? pol->w_min : 0), n,
                            (uint64_t)qcap, (uint64_t)max_w, (uint64_t)c->kernel};
    const uint32_t *kw = reinterpret_cast<const uint32_t *>(&kp);
    for (size_t i = 0; i < sizeof(ExtParams) / 4; ++i) k.push_back(kw[i]);
    for (DevBuf *b : {&c->jobs, &c->order, &c->qseq, &c->tseq, &c->out, &c->clamped, &c->cells_job, &c->misc,
                      &c->w_first, &c->w_cur, &c->prev, &c->kk, &c->w_final, &c->tries, &c->missed, &c->list_a,
                      &c->list_b, &c->feat, &c->wbf, &c->part_n, &c->ovf, &c->part_blk[0], &c->part_blk[1],
                      &c->part_blk[2], &c->part_blk[3], &c->class_ovf_n})
        k.push_back((uint64_t)(uintptr_t)b->p);
    for (const SeqBuf *b : {&c->cq, &c->ct}) {
        k.push_back(b->packed);
        k.push_back(b->nbytes);
        k.push_back(b->n_runs);
        k.push_back((uint64_t)(uintptr_t)b->runs);
    }
    k.insert(k.end(), extra.begin(), extra.end());
    return k;
}

// Graph mode: records `prologue` (if any) and the call's rounds as one CUDA graph the
// first time a key is seen, then replays it; ev0..ev1 bracket the replay.
int run_ext_graph(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, uint32_t n,
                  const std::vector<std::pair<uint32_t, int>> &segs, int qcap, int max_w,
                  const std::vector<uint64_t> &extra, const std::function<int(cudaStream_t, uint32_t *)> &prologue,
                  const int32_t *d_wfirst, cudaStream_t s, fa_ext_stats *stats, int32_t *h_wfinal) {
    if (pol && pol->mode != FA_POLICY_SINGLE)
        if (int rc = ensure_policy_buffers(c, n)) return rc;
    if (int rc = ensure_aux_streams(c)) return rc;
    if (int rc = ensure_side(c, segs.size())) return rc;
    int rc0 = FA_OK;
    const Choice kc = resolve_choice(c, kp, c->jobs.as<fa_job>(), c->order.as<uint32_t>(), n, c->cq, c->ct, qcap,
                                     max_w, c->out.as<fa_ext_result>(),
                                     misc_of(c).status, s, &rc0);
    if (rc0) return rc0;
    // each capacity class's kernel, tuned before recording (tuning cannot run in a capture);
    // the classes and their choices are part of the key, so a replay has the same ones
    std::vector<Choice> seg_kc;
    {
        uint32_t b = 0;
        for (auto &sg : segs) {
            seg_kc.push_back(resolve_choice(c, kp, c->jobs.as<fa_job>(), c->order.as<uint32_t>() + b, sg.first - b,
                                            c->cq, c->ct, sg.second, max_w,
                                            c->out.as<fa_ext_result>(), misc_of(c).status, s, &rc0));
            if (rc0) return rc0;
            b = sg.first;
        }
        c->last_choice = kc;
    }
    std::vector<uint64_t> extra2 = extra;
    extra2.push_back((uint64_t)kc.kernel << 32 | (uint32_t)kc.tpb);
    for (size_t k = 0; k < segs.size(); ++k) {
        extra2.push_back((uint64_t)segs[k].first << 32 | (uint32_t)segs[k].second);
        extra2.push_back((uint64_t)seg_kc[k].kernel << 32 | (uint32_t)seg_kc[k].tpb);
    }
    std::vector<uint64_t> key = graph_key(c, kp, pol, n, qcap, max_w, extra2);
    if (!c->gexec || key != c->gkey) {
        if (c->gexec) {
            cudaGraphExecDestroy(c->gexec);
            c->gexec = nullptr;
        }
        uint32_t launches = 0;
        FA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        int rc = prologue ? prologue(s, &launches) : FA_OK;
        if (!rc)
            rc = enqueue_ext(c, kp, pol, n, segs, qcap, max_w, c->jobs.as<fa_job>(), c->order.as<uint32_t>(),
                             c->cq, c->ct, d_wfirst, c->out.as<fa_ext_result>(), s,
                             true, &launches, nullptr, kc, &seg_kc);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (rc || ec != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (rc) return rc;
            FA_CUDA(ec);
        }
        const cudaError_t ei = cudaGraphInstantiate(&c->gexec, g, 0);
        cudaGraphDestroy(g);
        FA_CUDA(ei);
        c->gkey = key;
        c->glaunches = launches;
    }
    FA_CUDA(cudaEventRecord(c->ev0, s));
    FA_CUDA(cudaGraphLaunch(c->gexec, s));
    FA_CUDA(cudaEventRecord(c->ev1, s));
    return finish_ext(c, pol, n, s, stats, h_wfinal, c->glaunches, 0, true);
}

int max_band_of(const fa_job *jobs, uint32_t n) {
    int w = 0;
    for (uint32_t i = 0; i < n; ++i) w = std::max(w, jobs[i].w);
    return w;
}

// One host sequence buffer as a call receives it: byte codes, or 2-bit packed bases with
// their N runs.  npos: the positions jobs may address (bytes, or bases when packed).
struct HostSeq {
    const uint8_t *p;
    uint64_t nbytes;
    uint64_t npos;
    const fa_nrun *runs;
    uint64_t n_runs;
    bool packed;
};

HostSeq host_bytes(const uint8_t *p, uint64_t len) { return HostSeq{p, len, len, nullptr, 0, false}; }

// A packed host buffer, checked: bases present, N runs sorted, non-overlapping, non-empty and
// inside the buffer.
int host_packed(const fa_packed_seq *ps, const char *what, HostSeq *out) {
    if (!ps) return fail(FA_ERR_ARG, "null packed %s buffer", what);
    if (ps->n_bases && !ps->bases) return fail(FA_ERR_ARG, "packed %s buffer has no bases", what);
    if (ps->n_nruns && !ps->n_runs) return fail(FA_ERR_ARG, "packed %s buffer has no run array", what);
    if (ps->n_nruns >= (1ull << 32)) return fail(FA_ERR_CAPACITY, "packed %s buffer: too many N runs", what);
    // the runs themselves are checked on the device (finish_ext)
    *out = HostSeq{ps->bases, (ps->n_bases + 3) / 4, ps->n_bases, ps->n_runs, ps->n_nruns, true};
    return FA_OK;
}

// Device copies of a call's sequences (kSeqPad bytes of slack) and N runs, and the SeqBufs
// the kernels read them through.
int ensure_seq_buffers(fa_ctx *c, const HostSeq &q, const HostSeq &t) {
    FA_CUDA(c->qseq.ensure(q.nbytes + kSeqPad));
    FA_CUDA(c->tseq.ensure(t.nbytes + kSeqPad));
    if (q.n_runs) FA_CUDA(c->qruns.ensure(sizeof(fa_nrun) * q.n_runs));
    if (t.n_runs) FA_CUDA(c->truns.ensure(sizeof(fa_nrun) * t.n_runs));
    c->cq = SeqBuf{c->qseq.as<uint8_t>(), q.nbytes, q.n_runs ? c->qruns.as<fa_nrun>() : nullptr,
                   (uint32_t)q.n_runs, q.packed ? 1u : 0u};
    c->ct = SeqBuf{c->tseq.as<uint8_t>(), t.nbytes, t.n_runs ? c->truns.as<fa_nrun>() : nullptr,
                   (uint32_t)t.n_runs, t.packed ? 1u : 0u};
    c->q_bases = q.npos;
    c->t_bases = t.npos;
    return FA_OK;
}

int upload_runs(fa_ctx *c, const HostSeq &q, const HostSeq &t, cudaStream_t s) {
    if (q.n_runs) FA_CUDA(cudaMemcpyAsync(c->qruns.p, q.runs, sizeof(fa_nrun) * q.n_runs, cudaMemcpyHostToDevice, s));
    if (t.n_runs) FA_CUDA(cudaMemcpyAsync(c->truns.p, t.runs, sizeof(fa_nrun) * t.n_runs, cudaMemcpyHostToDevice, s));
    return FA_OK;
}

// Single-band host batch with the uploads pipelined under the kernels: the job records go
// first, the GPU validates them and orders them by (upload slice, query length) while the
// query and target buffers stream up in kSlices byte slices on a copy stream, and the
// jobs of each slice start as soon as that slice has arrived.  Same results, statistics
// and errors as the serial path (a rejected batch reports the first bad job through the
// host-side checks); with pageable host buffers the copies simply do not overlap.  Byte
// codes and packed bases alike: slices are cut in bytes, jobs placed by the byte holding
// their last base.
constexpr int kSlices = 8;   // at most this many upload slices (the event and scratch arrays)
constexpr uint32_t kPipeMinJobs = 32768;

int ensure_pipe_streams(fa_ctx *c) {
    FA_CUDA(c->chunk_scratch.ensure(std::max(chunk_scratch_bytes(kSlices),
                                             sizeof(uint32_t) * slice_scratch_words(kSlices))));
    if (!c->copy_stream) {
        FA_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (auto &e : c->slice_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto &e : c->done_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        FA_CUDA(cudaEventCreateWithFlags(&c->jobs_ev, cudaEventDisableTiming));
        FA_CUDA(cudaStreamCreateWithFlags(&c->prep_stream, cudaStreamNonBlocking));
        for (auto &e : c->job_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto &e : c->info_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        FA_CUDA(cudaMallocHost(&c->h_slice_info, sizeof(uint32_t) * kSliceInfoWords * kSlices));
        for (int k = 0; k < kSlices; ++k) {
            FA_CUDA(cudaEventCreate(&c->span_ev[k][0]));
            FA_CUDA(cudaEventCreate(&c->span_ev[k][1]));
        }
    }
    return ensure_aux_streams(c);
}

// graded slices (for 8: 1, 1, 2, 4, 6, 6, 6, 6 thirty-seconds of each buffer): the first jobs
// start after a small upload, and the uploads, faster than the kernels, stay ahead
constexpr int kGradedCum[kSlices + 1][kSlices] = {
    {32}, {32}, {4, 32}, {2, 10, 32}, {1, 4, 14, 32}, {1, 2, 6, 16, 32}, {1, 2, 4, 10, 20, 32},
    {1, 2, 4, 8, 14, 22, 32}, {1, 2, 4, 8, 14, 20, 26, 32}};
ChunkEnds graded_ends(const HostSeq &q, const HostSeq &t, int ns) {
    ChunkEnds ends;
    static_assert(kSlices <= kMaxChunks, "slice count");
    for (int k = 0; k < ns; ++k) {
        ends.q[k] = k == ns - 1 ? q.nbytes : q.nbytes / 32 * kGradedCum[ns][k];
        ends.t[k] = k == ns - 1 ? t.nbytes : t.nbytes / 32 * kGradedCum[ns][k];
    }
    ends.shift = q.packed ? 2 : 0;
    return ends;
}

// The sequence slices on the copy stream, one event per slice.
int upload_slices(fa_ctx *c, const HostSeq &q, const HostSeq &t, const ChunkEnds &ends, int ns) {
    cudaStream_t cs = c->copy_stream;
    for (int k = 0; k < ns; ++k) {
        const uint64_t q0 = k ? ends.q[k - 1] : 0, q1 = ends.q[k];
        const uint64_t t0 = k ? ends.t[k - 1] : 0, t1 = ends.t[k];
        if (q1 > q0) FA_CUDA(cudaMemcpyAsync(c->qseq.as<uint8_t>() + q0, q.p + q0, q1 - q0, cudaMemcpyHostToDevice, cs));
        if (t1 > t0) FA_CUDA(cudaMemcpyAsync(c->tseq.as<uint8_t>() + t0, t.p + t0, t1 - t0, cudaMemcpyHostToDevice, cs));
        FA_CUDA(cudaEventRecord(c->slice_ev[k], cs));
    }
    return FA_OK;
}

// Validation and (slice, length) histogram of the uploaded jobs; h_info as launch_chunk_prep
// lays it out: status, first bad job, longest query, widest band | slice bounds in the order |
// each slice's lowest and highest job index.  A rejected batch reports its first bad job
// with the host-side checks' message.
constexpr int kInfoWords = 4 + kSlices + 1 + 2 * kSlices;
inline int info_words(int ns) { return 4 + ns + 1 + 2 * ns; }
int prep_slices(fa_ctx *c, const ExtParams &kp, const fa_job *jobs, uint32_t n, const HostSeq &q, const HostSeq &t,
                const ChunkEnds &ends, int ns, uint32_t *h_info) {
    cudaStream_t s = c->stream;
    uint32_t *scratch = c->chunk_scratch.as<uint32_t>();
    const size_t nbins = (size_t)ns * (FA_MAX_QLEN + 1);
    FA_CUDA(launch_chunk_prep(c->jobs.as<fa_job>(), n, q.npos, t.npos, ends, ns, kp.max_score,
                              (kp.flags & FA_PARAM_H0_ZERO) ? 0 : 1, packed_qcap_limit(c->smem_optin), scratch, s));
    FA_CUDA(cudaMemcpyAsync(h_info, scratch + 3 * nbins, sizeof(uint32_t) * info_words(ns), cudaMemcpyDeviceToHost,
                            s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (h_info[0]) {
        FA_CUDA(cudaStreamSynchronize(c->copy_stream));   // the caller's buffers stay in use until then
        const uint32_t bad = h_info[1] < n ? h_info[1] : 0;
        int mq = 0;
        const int rc = check_jobs(jobs + bad, 1, q.npos, t.npos, kp, packed_qcap_limit(c->smem_optin), &mq);
        if (rc) return fail(rc, "job %u: %s", bad, g_err.c_str() + (g_err.compare(0, 7, "job 0: ") == 0 ? 7 : 0));
        return fail(FA_ERR_ARG, "job %u is invalid", bad);
    }
    return FA_OK;
}

// Whether every slice's jobs form one index range, together covering all n jobs (the
// sequences lie in job order).
bool slices_in_order(const uint32_t *h_info, uint32_t n, int ns) {
    uint32_t covered = 0;
    for (int k = 0; k < ns; ++k) {
        const uint32_t cnt = h_info[4 + k + 1] - h_info[4 + k];
        const uint32_t lo = h_info[4 + ns + 1 + k], hi = h_info[4 + 2 * ns + 1 + k];
        if (cnt && hi - lo + 1 != cnt) return false;
        covered += cnt;
    }
    return covered == n;
}

// Slice counts when the caller set none.  Byte-code batches are upload-bound (the
// sequences take longer to copy than the rounds to run), so eight slices let the kernels follow
// the copies closely; packed batches upload a quarter of the bytes, and the per-slice rounds
// then cost more than the overlap gains past two slices.  A single-band batch runs one kernel
// per slice and takes eight either way.
int auto_slices(bool rounds, const HostSeq &hq) { return rounds && hq.packed ? 2 : 8; }

// Slice counts of streamed host batches when the caller set none (measured on 1M 151-bp
// jobs): byte codes are upload-bound (four times the bytes), so eight slices follow the
// uploads; packed retry-policy slices each end in a few long retries, so three; packed
// single-band slices run one kernel each, six.
int auto_slices_streamed(bool rounds, const HostSeq &hq) { return !hq.packed ? 8 : rounds ? 3 : 6; }

// Whether a host batch streams.  A learned batch of byte codes does not: its uploads end
// after its kernels would, and a streamed slice's rounds -- the narrow round, then the
// retries at the configured band, about 1 ms of one-thread-per-job latency whatever the
// slice's size -- would follow the last upload; the pipelined path runs the retries of all
// slices once after the last slice instead (9.9 against 10.0-12.1 ms per 1M jobs).
bool streams(const fa_policy *pol, const HostSeq &hq) {
    return hq.packed || !pol || pol->mode != FA_POLICY_LEARNED;
}

int ext_batch_pipelined(fa_ctx *c, const ExtParams &kp, const fa_job *jobs, uint32_t n, const HostSeq &hq,
                        const HostSeq &ht, fa_ext_result *out, fa_ext_stats *stats) {
    if (int rc = ensure_ext_buffers(c, n, 0, 0)) return rc;
    if (int rc = ensure_seq_buffers(c, hq, ht)) return rc;
    if (int rc = ensure_pipe_streams(c)) return rc;
    cudaStream_t s = c->stream, cs = c->copy_stream;
    const int ns = c->slices_single ? c->slices_single : auto_slices(false, hq);
    const ChunkEnds ends = graded_ends(hq, ht, ns);
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    // the job records and N runs first, then the sequence slices, all on the copy stream
    // (one after another, so the records arrive at full bandwidth)
    FA_CUDA(cudaEventRecord(c->fork_ev, s));      // after all earlier work on the main stream
    FA_CUDA(cudaStreamWaitEvent(cs, c->fork_ev, 0));
    FA_CUDA(cudaMemcpyAsync(c->jobs.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice, cs));
    if (int rc = upload_runs(c, hq, ht, cs)) return rc;
    FA_CUDA(cudaEventRecord(c->jobs_ev, cs));
    FA_CUDA(cudaStreamWaitEvent(s, c->jobs_ev, 0));
    if (int rc = upload_slices(c, hq, ht, ends, ns)) return rc;
    uint32_t h_info[kInfoWords];
    if (int rc = prep_slices(c, kp, jobs, n, hq, ht, ends, ns, h_info)) return rc;
    const int max_q = (int)h_info[2];
    FA_CUDA(launch_chunk_scatter(c->jobs.as<fa_job>(), n, ends, ns, c->chunk_scratch.as<uint32_t>(),
                                 c->order.as<uint32_t>(), s));
    const int band = (int)h_info[3];   // widest configured band, reduced on the device
    if (c->kernel == FA_KERNEL_AUTO && !c->tuned.count({(max_q + 31) / 32, band, (int)hq.packed}))
        FA_CUDA(cudaStreamWaitEvent(s, c->slice_ev[ns - 1], 0));   // tuning reads every slice
    int rc0 = FA_OK;
    const Choice kc = resolve_choice(c, kp, c->jobs.as<fa_job>(), c->order.as<uint32_t>(), n, c->cq, c->ct, max_q,
                                     band, c->out.as<fa_ext_result>(), m.status, s, &rc0);
    if (rc0) return rc0;
    uint32_t launches = 2;
    // slices alternate between the main stream and an auxiliary one (each with its own
    // overflow list), so one slice's last, partly filled wave overlaps the next slice's start
    cudaStream_t sk[2] = {s, c->aux[0]};
    FA_CUDA(cudaEventRecord(c->ev0, s));
    FA_CUDA(cudaEventRecord(c->fork_ev, s));
    FA_CUDA(cudaStreamWaitEvent(sk[1], c->fork_ev, 0));
    // Results come back slice by slice on the upload stream, behind the uploads, each once
    // its kernels have run, when every slice's jobs form one index range (sequences laid
    // out in job order) and `out` is pinned (an asynchronous copy into pageable memory would
    // hold the host thread): only the last slice's results are left for the end.
    bool early = false;
    {
        cudaPointerAttributes pa;
        early = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        early = early && slices_in_order(h_info, n, ns);
    }
    for (int k = 0; k < ns; ++k) {
        const uint32_t cnt = h_info[4 + k + 1] - h_info[4 + k];
        cudaStream_t st = sk[k & 1];
        FA_CUDA(cudaStreamWaitEvent(st, c->slice_ev[k], 0));
        if (cnt == 0) continue;
        FA_CUDA(launch_ext(c, kc, c->jobs.as<fa_job>(), c->order.as<uint32_t>() + h_info[4 + k], cnt, nullptr, c->cq,
                           c->ct, kp, max_q, nullptr, c->out.as<fa_ext_result>(), nullptr, false,
                           c->cells_job.as<uint32_t>(), m.cells, m.status, st, k & 1));
        launches += ext_kernels_of(c, kc, kp, max_q);
        if (early) {
            const uint32_t lo = h_info[4 + ns + 1 + k];
            FA_CUDA(cudaEventRecord(c->done_ev[k], st));
            FA_CUDA(cudaStreamWaitEvent(cs, c->done_ev[k], 0));
            FA_CUDA(cudaMemcpyAsync(out + lo, c->out.as<fa_ext_result>() + lo, sizeof(fa_ext_result) * (size_t)cnt,
                                    cudaMemcpyDeviceToHost, cs));
        }
    }
    FA_CUDA(cudaEventRecord(c->join_ev[0], sk[1]));
    FA_CUDA(cudaStreamWaitEvent(s, c->join_ev[0], 0));
    FA_CUDA(cudaEventRecord(c->ev1, s));
    if (early) {
        FA_CUDA(cudaEventRecord(c->join_ev[1], cs));
        FA_CUDA(cudaStreamWaitEvent(s, c->join_ev[1], 0));
    } else {
        FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
    }
    if (int rc = finish_ext(c, nullptr, n, s, stats, nullptr, launches, 0, false)) return rc;
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

// Busy time of the slices whose bits `spans` sets: the union of their [start, end] events.
float busy_ms(fa_ctx *c, int spans, int ns) {
    int k0 = 0;
    while (!(spans & (1 << k0))) ++k0;
    std::vector<std::pair<float, float>> iv;
    for (int k = k0; k < ns; ++k) {
        if (!(spans & (1 << k))) continue;
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, c->span_ev[k0][0], c->span_ev[k][0]);
        cudaEventElapsedTime(&b, c->span_ev[k0][0], c->span_ev[k][1]);
        iv.push_back({a, b});
    }
    std::sort(iv.begin(), iv.end());
    float busy = 0.f, lo = iv[0].first, hi = iv[0].second;
    for (size_t i = 1; i < iv.size(); ++i) {
        if (iv[i].first > hi) {
            busy += hi - lo;
            lo = iv[i].first;
        }
        hi = std::max(hi, iv[i].second);
    }
    return busy + (hi - lo);
}

// A retry policy's rounds on a host batch whose jobs address their sequences in job order
// (FA_POLICY_BWA, or FA_POLICY_LEARNED with first bands from w_first or, given a model, from
// the band features and MLP on the device): the job records, hints, first bands and N runs
// go up first, then the sequences in kSlices graded slices on the copy stream.  As each
// slice arrives its jobs run prediction, policy set-up and the first extension round; the
// jobs that round rejects collect in one retry list across the slices, and the later rounds
// run over that list.  Results, bands and statistics are those of the serial path; the
// device time reported is the kernels' busy time (the waits for uploads left out).
// *done = false (nothing run) when the jobs' sequences are not in job order.
int ext_batch_sliced(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, const fa_band_model *model, float margin,
                     const fa_job *jobs, uint32_t n, const HostSeq &hq, const HostSeq &ht, const fa_band_hint *hints,
                     const int32_t *w_first, fa_ext_result *out, int32_t *w_first_out, int32_t *w_final,
                     fa_ext_stats *stats, bool *done) {
    *done = false;
    const bool learned = pol->mode == FA_POLICY_LEARNED;
    if (int rc = ensure_ext_buffers(c, n, 0, 0)) return rc;
    if (int rc = ensure_seq_buffers(c, hq, ht)) return rc;
    if (int rc = ensure_policy_buffers(c, n)) return rc;
    if (int rc = ensure_pipe_streams(c)) return rc;
    float *d_x = nullptr;
    fa_band_hint *d_h = nullptr;
    std::vector<__nv_bfloat16> wbf;
    float mean[16], sd[16];
    if (model) {
        FA_CUDA(c->feat.ensure(sizeof(float) * 16 * (size_t)n + sizeof(fa_band_hint) * (size_t)n));
        FA_CUDA(c->wbf.ensure(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS));
        d_x = c->feat.as<float>();
        d_h = hints ? reinterpret_cast<fa_band_hint *>(d_x + 16 * (size_t)n) : nullptr;
        band_model_export(model, wbf, mean, sd);
    }
    cudaStream_t s = c->stream, cs = c->copy_stream;
    const int ns = c->slices_rounds ? c->slices_rounds : auto_slices(true, hq);
    const ChunkEnds ends = graded_ends(hq, ht, ns);
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    FA_CUDA(cudaEventRecord(c->fork_ev, s));
    FA_CUDA(cudaStreamWaitEvent(cs, c->fork_ev, 0));
    FA_CUDA(cudaMemcpyAsync(c->jobs.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice, cs));
    if (int rc = upload_runs(c, hq, ht, cs)) return rc;
    if (model) {
        if (d_h) FA_CUDA(cudaMemcpyAsync(d_h, hints, sizeof(fa_band_hint) * (size_t)n, cudaMemcpyHostToDevice, cs));
        FA_CUDA(cudaMemcpyAsync(c->wbf.p, wbf.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS,
                                cudaMemcpyHostToDevice, cs));
    } else if (learned) {
        FA_CUDA(cudaMemcpyAsync(c->w_first.p, w_first, 4ull * n, cudaMemcpyHostToDevice, cs));
    }
    FA_CUDA(cudaEventRecord(c->jobs_ev, cs));
    FA_CUDA(cudaStreamWaitEvent(s, c->jobs_ev, 0));
    if (int rc = upload_slices(c, hq, ht, ends, ns)) return rc;
    uint32_t h_info[kInfoWords];
    if (int rc = prep_slices(c, kp, jobs, n, hq, ht, ends, ns, h_info)) return rc;
    if (!slices_in_order(h_info, n, ns)) {
        FA_CUDA(cudaStreamSynchronize(cs));
        return FA_OK;
    }
    *done = true;
    const int max_q = (int)h_info[2];
    const int band = (int)h_info[3];
    FA_CUDA(launch_chunk_scatter(c->jobs.as<fa_job>(), n, ends, ns, c->chunk_scratch.as<uint32_t>(),
                                 c->order.as<uint32_t>(), s));
    if (c->kernel == FA_KERNEL_AUTO && !c->tuned.count({(max_q + 31) / 32, band, (int)hq.packed}))
        FA_CUDA(cudaStreamWaitEvent(s, c->slice_ev[ns - 1], 0));   // tuning reads every slice
    int rc0 = FA_OK;
    const Choice kc = resolve_choice(c, kp, c->jobs.as<fa_job>(), c->order.as<uint32_t>(), n, c->cq, c->ct, max_q,
                                     band, c->out.as<fa_ext_result>(), m.status, s, &rc0);
    if (rc0) return rc0;
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));   // the tuner's runs leave their cells and status
    const fa_job *d_jobs = c->jobs.as<fa_job>();
    const uint32_t *order = c->order.as<uint32_t>();
    int32_t *d_wf = c->w_first.as<int32_t>();
    PolicyState st{c->w_cur.as<int32_t>(), c->prev.as<int32_t>(), c->kk.as<int32_t>(),
                   c->w_final.as<int32_t>(), c->tries.as<int32_t>(), c->missed.as<uint8_t>()};
    uint8_t *d_flags = learned ? c->clamped.as<uint8_t>() : nullptr;
    const bool cert = learned && (pol->judge & FA_JUDGE_BOUND);
    const int max_tries = std::max(1, pol->max_tries);
    uint32_t launches = 0, retries = 0;
    int spans = 0;
    // Alternate slices run on two lanes, so one slice's last, longest jobs overlap the next
    // slice's start: lane 0 is the main stream with misc_of(c), lane 1 its own stream, band-
    // group streams and counters (status, cells and the retry list's count are shared).
    Misc ms[2];
    if (int rc = ensure_lanes(c, 2, ms)) return rc;
    Misc &m1 = ms[1];
    uint32_t max_cnt = 0;
    for (int k = 0; k < ns; ++k) max_cnt = std::max(max_cnt, h_info[4 + k + 1] - h_info[4 + k]);
    FA_CUDA(c->ovf.ensure(sizeof(uint32_t) * std::max<size_t>(3 * (size_t)n, 6 * (size_t)max_cnt)));
    FA_CUDA(cudaMemsetAsync(c->lane_misc.as<char>() + kMiscBytes, 0, 64, s));
    FA_CUDA(cudaEventRecord(c->lane_ev[0], s));
    FA_CUDA(cudaStreamWaitEvent(c->lane_s[1], c->lane_ev[0], 0));
    for (int k = 0; k < ns; ++k) {
        const uint32_t b = h_info[4 + k], cnt = h_info[4 + k + 1] - b;
        const int lane = k & 1;
        cudaStream_t ls = lane ? c->lane_s[1] : s;
        Misc &ml = lane ? m1 : m;
        FA_CUDA(cudaStreamWaitEvent(ls, c->slice_ev[k], 0));
        if (cnt == 0) continue;
        const uint32_t lo = h_info[4 + ns + 1 + k];
        FA_CUDA(cudaEventRecord(c->span_ev[k][0], ls));
        if (model) {
            FA_CUDA(launch_band_features(d_jobs + lo, cnt, c->cq, c->ct, d_h ? d_h + lo : nullptr, kp.max_score,
                                         d_x + 16 * (size_t)lo, ls));
            FA_CUDA(launch_band_predict(c->wbf.as<__nv_bfloat16>(), mean, sd, d_x + 16 * (size_t)lo, d_jobs + lo, cnt,
                                        margin, pol->w_min, nullptr, d_wf + lo, ls));
            launches += 2;
        }
        const PolicyState sl{st.w_cur + lo, st.prev + lo, st.k + lo, st.w_final + lo, st.tries + lo,
                             st.missed + lo};
        FA_CUDA(launch_policy_init(d_jobs + lo, cnt, learned ? d_wf + lo : nullptr, pol->w_min, learned, sl, ls));
        const uint32_t *list = order + b;
        if (learned) {
            // the narrow bands now, each slice as it arrives; jobs whose first band is the
            // configured one join the retry list and run with the later round (same runs, same
            // policy state: the configured band goes straight to the bwa-mem2 rule either way)
            uint32_t *part = c->part_n.as<uint32_t>() + b;
            FA_CUDA(launch_band_partition(d_jobs, list, nullptr, cnt, st.w_cur, part, ml.bucket_hist,
                                          c->part_blk[lane].as<uint32_t>(), ml.group_bounds, ls));
            if (int rc = launch_learned_round(c, d_jobs, part, cnt, c->cq, c->ct, kp, max_q, st.w_cur,
                                              c->out.as<fa_ext_result>(), d_flags, cert, ml, ls, &launches, lane,
                                              (size_t)lane * 3 * max_cnt, true))
                return rc;
            FA_CUDA(launch_list_append(part, ml.group_bounds + 3, cnt, c->list_a.as<uint32_t>(), m.cnt_a, ls));
            FA_CUDA(launch_policy_step(d_jobs, part, ml.group_bounds + 3, ml.group_bounds + 2, cnt,
                                       c->out.as<fa_ext_result>(), d_flags, st, max_tries, pol->judge,
                                       c->list_a.as<uint32_t>(), m.cnt_a, ls));
            launches += 4;
        } else {
            FA_CUDA(launch_ext(c, kc, d_jobs, list, cnt, nullptr, c->cq, c->ct, kp, max_q, st.w_cur,
                               c->out.as<fa_ext_result>(), d_flags, false, c->cells_job.as<uint32_t>(), m.cells,
                               m.status, ls, lane));
            launches += ext_kernels_of(c, kc, kp, max_q);
            // the round's rejected jobs join one retry list (cnt_a counts across the slices)
            FA_CUDA(launch_policy_step(d_jobs, list, nullptr, nullptr, cnt, c->out.as<fa_ext_result>(), d_flags, st,
                                       max_tries, pol->judge, c->list_a.as<uint32_t>(), m.cnt_a, ls));
            launches += 2;
        }
        FA_CUDA(cudaEventRecord(c->span_ev[k][1], ls));
        spans |= 1 << k;
    }
    FA_CUDA(cudaEventRecord(c->lane_ev[1], c->lane_s[1]));
    FA_CUDA(cudaStreamWaitEvent(s, c->lane_ev[1], 0));
    FA_CUDA(cudaEventRecord(c->ev0, s));
    std::vector<std::pair<uint32_t, int>> segs{{n, max_q}};
    if (int rc = enqueue_ext(c, kp, pol, n, segs, max_q, band, d_jobs, order, c->cq, c->ct, d_wf,
                             c->out.as<fa_ext_result>(), s, false, &launches, &retries, kc, nullptr, 1,
                             c->list_a.as<uint32_t>(), m.cnt_a))
        return rc;
    FA_CUDA(cudaEventRecord(c->ev1, s));
    FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
    if (w_first_out && model) FA_CUDA(cudaMemcpyAsync(w_first_out, d_wf, 4ull * n, cudaMemcpyDeviceToHost, s));
    if (int rc = finish_ext(c, pol, n, s, stats, w_final, launches, retries, true)) return rc;
    if (stats && spans) stats->kernel_ms += busy_ms(c, spans, ns);   // plus the later rounds
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

// Streamed host batch (every policy): the batch is cut by job index into graded slices, and
// each slice's job records, hints or first bands, and the query and target bytes up to the
// slice's resident ends go up back to back on the copy stream, so the first slice starts
// after a small upload.  A prep stream validates each slice as its records arrive and
// orders its resident jobs by query length; the host reads the slice's summary (longest
// query, widest band, listed jobs), then enqueues the slice's whole work on one of two lanes
// -- band prediction, policy set-up, the first round and every retry round over the slice's
// own retry lists, with device-side counts -- and, into a pinned `out`, the copy of its
// results, which runs while the other lane computes.  Results, bands, statistics and errors
// are those of the serial path (a rejected batch reports its first bad job through the
// host-side checks).  *done = false when the jobs do not address their sequences in job
// order (nothing run, or, when a slice finds a job whose sequences lie past its resident
// ends, everything drained): the caller takes another path.
struct SliceSummary {
    uint32_t status, bad, max_q, band, listed, away;
};

bool jobs_in_sequence_order(const fa_job *jobs, uint32_t n) {
    constexpr uint32_t kProbes = 64;
    uint64_t q = 0, t = 0;
    for (uint32_t p = 0; p < kProbes; ++p) {
        const fa_job &j = jobs[(uint64_t)p * (n - 1) / (kProbes - 1)];
        if (j.q_off < q || j.t_off < t) return false;
        q = j.q_off;
        t = j.t_off;
    }
    return true;
}

int ext_batch_streamed(fa_ctx *c, const ExtParams &kp, const fa_policy *pol, const fa_band_model *model,
                       float margin, const fa_job *jobs, uint32_t n, const HostSeq &hq, const HostSeq &ht,
                       const fa_band_hint *hints, const int32_t *w_first, fa_ext_result *out, int32_t *w_first_out,
                       int32_t *w_final, fa_ext_stats *stats, bool *done) {
    *done = false;
    const int mode = pol ? pol->mode : FA_POLICY_SINGLE;
    const bool learned = mode == FA_POLICY_LEARNED;
    const int ns = mode == FA_POLICY_SINGLE ? (c->slices_single ? c->slices_single : auto_slices_streamed(false, hq))
                                            : (c->slices_rounds ? c->slices_rounds : auto_slices_streamed(true, hq));
    if (ns < 2 || ns > kSlices || !jobs_in_sequence_order(jobs, n)) return FA_OK;
    // slice bounds by job index, and each slice's resident ends (positions) and upload ends
    // (bytes): the bytes up to the later of the next slice's first sequence and this slice's
    // last job's end, never fewer than the slice before
    const uint64_t ppb = hq.packed ? 4 : 1;
    uint32_t J[kSlices + 1];
    uint64_t qres[kSlices], tres[kSlices], qend[kSlices], tend[kSlices];
    J[0] = 0;
    J[ns] = n;
    for (int k = 1; k < ns; ++k) J[k] = (uint32_t)((uint64_t)n * kGradedCum[ns][k - 1] / 32);
    for (int k = 0; k < ns; ++k) {
        if (k == ns - 1) {
            qend[k] = hq.nbytes;
            tend[k] = ht.nbytes;
        } else {
            const fa_job &a = jobs[J[k + 1]], &b = jobs[J[k + 1] - 1];
            const uint64_t eq = std::min<uint64_t>(std::max<uint64_t>(a.q_off, b.q_off + (uint64_t)std::max(b.qlen, 0)), hq.npos);
            const uint64_t et = std::min<uint64_t>(std::max<uint64_t>(a.t_off, b.t_off + (uint64_t)std::max(b.tlen, 0)), ht.npos);
            qend[k] = std::min<uint64_t>((eq + ppb - 1) / ppb, hq.nbytes);
            tend[k] = std::min<uint64_t>((et + ppb - 1) / ppb, ht.nbytes);
        }
        if (k) {
            qend[k] = std::max(qend[k], qend[k - 1]);
            tend[k] = std::max(tend[k], tend[k - 1]);
        }
        qres[k] = std::min<uint64_t>(qend[k] * ppb, hq.npos);
        tres[k] = std::min<uint64_t>(tend[k] * ppb, ht.npos);
    }
    uint32_t max_cnt = 0;
    for (int k = 0; k < ns; ++k) max_cnt = std::max(max_cnt, J[k + 1] - J[k]);
    if (int rc = ensure_ext_buffers(c, n, 0, 0)) return rc;
    if (int rc = ensure_seq_buffers(c, hq, ht)) return rc;
    if (mode != FA_POLICY_SINGLE)
        if (int rc = ensure_policy_buffers(c, n)) return rc;
    if (int rc = ensure_pipe_streams(c)) return rc;
    // one lane per slice, up to kLanes (slice k on lane k % nl), each with its own counters
    // and a third-of-its-slice overflow region per band group
    const int nl = std::min(ns, fa_ctx::kLanes);
    Misc ms[fa_ctx::kLanes];
    if (int rc = ensure_lanes(c, nl, ms)) return rc;
    FA_CUDA(c->ovf.ensure(sizeof(uint32_t) * std::max<size_t>(3 * (size_t)n, 3 * (size_t)nl * max_cnt)));
    float *d_x = nullptr;
    fa_band_hint *d_h = nullptr;
    std::vector<__nv_bfloat16> wbf;
    float mean[16], sd[16];
    if (model) {
        FA_CUDA(c->feat.ensure(sizeof(float) * 16 * (size_t)n + sizeof(fa_band_hint) * (size_t)n));
        FA_CUDA(c->wbf.ensure(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS));
        d_x = c->feat.as<float>();
        d_h = hints ? reinterpret_cast<fa_band_hint *>(d_x + 16 * (size_t)n) : nullptr;
        band_model_export(model, wbf, mean, sd);
    }
    cudaStream_t s = c->stream, cs = c->copy_stream, ps = c->prep_stream;
    Misc &m = ms[0];
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    FA_CUDA(cudaMemsetAsync(c->lane_misc.p, 0, kMiscBytes * fa_ctx::kLanes, s));
    FA_CUDA(cudaEventRecord(c->fork_ev, s));
    FA_CUDA(cudaStreamWaitEvent(cs, c->fork_ev, 0));
    FA_CUDA(cudaStreamWaitEvent(ps, c->fork_ev, 0));
    for (int l = 1; l < nl; ++l) FA_CUDA(cudaStreamWaitEvent(c->lane_s[l], c->fork_ev, 0));
    // uploads: N runs and model weights, then per slice its records and its bytes
    if (int rc = upload_runs(c, hq, ht, cs)) return rc;
    if (model)
        FA_CUDA(cudaMemcpyAsync(c->wbf.p, wbf.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS,
                                cudaMemcpyHostToDevice, cs));
    fa_job *d_jobs = c->jobs.as<fa_job>();
    int32_t *d_wf = mode != FA_POLICY_SINGLE ? c->w_first.as<int32_t>() : nullptr;
    for (int k = 0; k < ns; ++k) {
        const uint32_t j0 = J[k], cnt = J[k + 1] - j0;
        FA_CUDA(cudaMemcpyAsync(d_jobs + j0, jobs + j0, sizeof(fa_job) * (size_t)cnt, cudaMemcpyHostToDevice, cs));
        if (d_h) FA_CUDA(cudaMemcpyAsync(d_h + j0, hints + j0, sizeof(fa_band_hint) * cnt, cudaMemcpyHostToDevice, cs));
        if (learned && !model)
            FA_CUDA(cudaMemcpyAsync(d_wf + j0, w_first + j0, 4ull * cnt, cudaMemcpyHostToDevice, cs));
        FA_CUDA(cudaEventRecord(c->job_ev[k], cs));
        const uint64_t q0 = k ? qend[k - 1] : 0, t0 = k ? tend[k - 1] : 0;
        if (qend[k] > q0)
            FA_CUDA(cudaMemcpyAsync(c->qseq.as<uint8_t>() + q0, hq.p + q0, qend[k] - q0, cudaMemcpyHostToDevice, cs));
        if (tend[k] > t0)
            FA_CUDA(cudaMemcpyAsync(c->tseq.as<uint8_t>() + t0, ht.p + t0, tend[k] - t0, cudaMemcpyHostToDevice, cs));
        FA_CUDA(cudaEventRecord(c->slice_ev[k], cs));
    }
    // per slice: validation and length order as its records arrive, the summary to the host
    uint32_t *scratch = c->chunk_scratch.as<uint32_t>();
    uint32_t *order = c->order.as<uint32_t>();
    const size_t sw = slice_scratch_words(1);
    for (int k = 0; k < ns; ++k) {
        const uint32_t j0 = J[k], cnt = J[k + 1] - j0;
        FA_CUDA(cudaStreamWaitEvent(ps, c->job_ev[k], 0));
        FA_CUDA(launch_slice_prep(d_jobs + j0, cnt, hq.npos, ht.npos, qres[k], tres[k], kp.max_score,
                                  (kp.flags & FA_PARAM_H0_ZERO) ? 0 : 1, packed_qcap_limit(c->smem_optin),
                                  scratch + k * sw, order + j0, ps));
        FA_CUDA(cudaMemcpyAsync(c->h_slice_info + k * kSliceInfoWords, scratch + k * sw + 3 * (FA_MAX_QLEN + 1),
                                sizeof(uint32_t) * kSliceInfoWords, cudaMemcpyDeviceToHost, ps));
        FA_CUDA(cudaEventRecord(c->info_ev[k], ps));
    }
    auto drain = [&]() {
        cudaStreamSynchronize(cs);
        cudaStreamSynchronize(ps);
        for (int l = 0; l < nl; ++l) cudaStreamSynchronize(lane_stream(c, l));
    };
    auto summary = [&](int k, SliceSummary *f) -> int {
        FA_CUDA(cudaEventSynchronize(c->info_ev[k]));
        const uint32_t *w = c->h_slice_info + k * kSliceInfoWords;
        *f = SliceSummary{w[0], w[1], w[2], w[3], w[5], w[6]};
        return FA_OK;
    };
    // a slice with a bad job ends the call with that job's error; one with a job whose
    // sequences lie past its resident ends hands the batch to another path
    auto refuse = [&](int k, const SliceSummary &f) -> int {
        drain();
        if (f.status) {
            const uint32_t bad = J[k] + (f.bad < J[k + 1] - J[k] ? f.bad : 0);
            int mq = 0;
            const int rc = check_jobs(jobs + bad, 1, hq.npos, ht.npos, kp, packed_qcap_limit(c->smem_optin), &mq);
            if (rc) return fail(rc, "job %u: %s", bad, g_err.c_str() + (g_err.compare(0, 7, "job 0: ") == 0 ? 7 : 0));
            return fail(FA_ERR_ARG, "job %u is invalid", bad);
        }
        return FA_OK;   // *done stays false
    };
    SliceSummary f[kSlices];
    if (int rc = summary(0, &f[0])) return rc;
    if (f[0].status || f[0].away) return refuse(0, f[0]);
    // the kernel of every slice: fixed, or tuned; the first call for a (band, form) waits for
    // the whole batch and tunes on its largest slice
    Choice kc;
    if (!slice_choice(c, (int)f[0].max_q, (int)f[0].band, hq.packed, &kc)) {
        int kt = 0;
        for (int k = 1; k < ns; ++k) {
            if (int rc = summary(k, &f[k])) return rc;
            if (f[k].status || f[k].away) return refuse(k, f[k]);
            if (f[k].listed > f[kt].listed) kt = k;
        }
        FA_CUDA(cudaStreamWaitEvent(s, c->slice_ev[ns - 1], 0));
        FA_CUDA(cudaStreamWaitEvent(s, c->info_ev[ns - 1], 0));
        int rc0 = FA_OK;
        kc = resolve_choice(c, kp, d_jobs + J[kt], order + J[kt], f[kt].listed, c->cq, c->ct, (int)f[kt].max_q,
                       (int)f[kt].band, c->out.as<fa_ext_result>() + J[kt], m.status, s, &rc0);
        if (rc0) {
            drain();
            return rc0;
        }
        FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));   // the tuner's runs leave their cells and status
        FA_CUDA(cudaEventRecord(c->lane_ev[0], s));
        for (int l = 1; l < nl; ++l) FA_CUDA(cudaStreamWaitEvent(c->lane_s[l], c->lane_ev[0], 0));
    }
    // results back slice by slice only into page-locked memory (a copy into pageable memory
    // would hold the host thread until the slice had run)
    auto pinned = [](const void *p) {
        cudaPointerAttributes pa;
        const bool r = p && cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        return r;
    };
    const bool early = pinned(out);
    const bool wf_early = model && pinned(w_first_out);
    PolicyState st{c->w_cur.as<int32_t>(), c->prev.as<int32_t>(), c->kk.as<int32_t>(),
                   c->w_final.as<int32_t>(), c->tries.as<int32_t>(), c->missed.as<uint8_t>()};
    uint8_t *d_flags = learned ? c->clamped.as<uint8_t>() : nullptr;
    const bool cert = learned && (pol->judge & FA_JUDGE_BOUND);
    const bool once = learned && (pol->judge & FA_JUDGE_ONCE);
    const int narrow_rounds = learned && (pol->judge & FA_JUDGE_HINT) && (pol->judge & FA_JUDGE_BOUND) ? 2 : 1;
    const int max_tries = mode != FA_POLICY_SINGLE ? std::max(1, pol->max_tries) : 1;
    fa_ext_result *d_out = c->out.as<fa_ext_result>();
    uint32_t launches = 0;
    int spans = 0;
    for (int k = 0; k < ns; ++k) {
        if (k)
            if (int rc = summary(k, &f[k])) return rc;
        if (f[k].status || f[k].away) return refuse(k, f[k]);
        const int lane = k % nl;
        cudaStream_t ls = lane_stream(c, lane);
        Misc &ml = ms[lane];
        const uint32_t j0 = J[k], cnt = J[k + 1] - j0, listed = f[k].listed;
        const int qcap = (int)f[k].max_q;
        Choice kk = kc;
        slice_choice(c, qcap, (int)f[k].band, hq.packed, &kk);
        FA_CUDA(cudaStreamWaitEvent(ls, c->slice_ev[k], 0));
        FA_CUDA(cudaStreamWaitEvent(ls, c->info_ev[k], 0));
        FA_CUDA(cudaEventRecord(c->span_ev[k][0], ls));
        spans |= 1 << k;
        // the slice's views of the per-job arrays (its order and lists hold local indices)
        const fa_job *jb = d_jobs + j0;
        const uint32_t *ord = order + j0;
        fa_ext_result *o = d_out + j0;
        uint32_t *cj = c->cells_job.as<uint32_t>() + j0;
        const OvfRes ovr{c->ovf.as<uint32_t>() + (size_t)lane * 3 * max_cnt, ml.ovf_n, ml.work, 3 * (size_t)max_cnt};
        if (mode == FA_POLICY_SINGLE) {
            FA_CUDA(launch_ext_res(c, kk, jb, ord, listed, nullptr, c->cq, c->ct, kp, qcap, nullptr, o, nullptr, false,
                                   cj, ml.cells, ml.status, ls, ovr));
            launches += ext_kernels_of(c, kk, kp, qcap);
        } else {
            const PolicyState sl{st.w_cur + j0, st.prev + j0, st.k + j0, st.w_final + j0, st.tries + j0,
                                 st.missed + j0};
            uint8_t *fl = d_flags ? d_flags + j0 : nullptr;
            int32_t *wf = d_wf + j0;
            if (model) {
                FA_CUDA(launch_band_features(jb, cnt, c->cq, c->ct, d_h ? d_h + j0 : nullptr, kp.max_score,
                                             d_x + 16 * (size_t)j0, ls));
                FA_CUDA(launch_band_predict(c->wbf.as<__nv_bfloat16>(), mean, sd, d_x + 16 * (size_t)j0, jb, cnt,
                                            margin, pol->w_min, nullptr, wf, ls));
                launches += 2;
            }
            FA_CUDA(launch_policy_init(jb, cnt, learned ? wf : nullptr, pol->w_min, learned, sl, ls));
            ++launches;
            uint32_t *list = c->list_a.as<uint32_t>() + j0, *next = c->list_b.as<uint32_t>() + j0;
            uint32_t *lcnt = ml.cnt_a, *ncnt = ml.cnt_b;
            uint32_t *part = c->part_n.as<uint32_t>() + j0;
            uint32_t *blk = c->part_blk[lane].as<uint32_t>();
            const size_t ovf_off = (size_t)lane * 3 * max_cnt;
            FA_CUDA(cudaMemsetAsync(lcnt, 0, 4, ls));
            // first round: the narrow bands (the configured-band bucket joins the retry list),
            // or the policy's first band
            if (learned) {
                FA_CUDA(launch_band_partition(jb, ord, nullptr, listed, sl.w_cur, part, ml.bucket_hist, blk,
                                              ml.group_bounds, ls));
                if (int rc = launch_learned_round(c, jb, part, listed, c->cq, c->ct, kp, qcap, sl.w_cur, o, fl, cert,
                                                  ml, ls, &launches, lane, ovf_off, true, cj))
                    return rc;
                FA_CUDA(launch_list_append(part, ml.group_bounds + 3, listed, list, lcnt, ls));
                FA_CUDA(launch_policy_step(jb, part, ml.group_bounds + 3, ml.group_bounds + 2, listed, o, fl, sl,
                                           max_tries, pol->judge, list, lcnt, ls));
                launches += 5;   // partition (3), list append, policy step
            } else {
                FA_CUDA(launch_ext_res(c, kk, jb, ord, listed, nullptr, c->cq, c->ct, kp, qcap, sl.w_cur, o, fl,
                                       false, cj, ml.cells, ml.status, ls, ovr));
                launches += ext_kernels_of(c, kk, kp, qcap);
                FA_CUDA(launch_policy_step(jb, ord, nullptr, nullptr, listed, o, fl, sl, max_tries, pol->judge, list,
                                           lcnt, ls));
                ++launches;
            }
            // the later rounds over the slice's retry list, a fixed number with device-side
            // counts (an empty round's launches leave at once)
            const int rounds = max_rounds_of(pol, (int)f[k].band);
            for (int r = 1; r < rounds; ++r) {
                const bool cert_r = cert && !(once && r >= narrow_rounds);
                if (learned && cert_r) {
                    FA_CUDA(launch_band_partition(jb, list, lcnt, listed, sl.w_cur, part, ml.bucket_hist, blk,
                                                  ml.group_bounds, ls));
                    if (int rc = launch_learned_round(c, jb, part, listed, c->cq, c->ct, kp, qcap, sl.w_cur, o, fl,
                                                      true, ml, ls, &launches, lane, ovf_off, false, cj))
                        return rc;
                    launches += 3;   // partition
                } else {
                    FA_CUDA(launch_ext_res(c, kk, jb, list, listed, lcnt, c->cq, c->ct, kp, qcap, sl.w_cur, o, fl,
                                           cert_r, cj, ml.cells, ml.status, ls, ovr));
                    launches += cert_r ? 1u : ext_kernels_of(c, kk, kp, qcap);
                }
                FA_CUDA(cudaMemsetAsync(ncnt, 0, 4, ls));
                FA_CUDA(launch_policy_step(jb, list, nullptr, lcnt, listed, o, fl, sl, max_tries, pol->judge, next,
                                           ncnt, ls));
                ++launches;
                std::swap(list, next);
                std::swap(lcnt, ncnt);
            }
        }
        FA_CUDA(cudaEventRecord(c->span_ev[k][1], ls));
        if (early) FA_CUDA(cudaMemcpyAsync(out + j0, o, sizeof(fa_ext_result) * cnt, cudaMemcpyDeviceToHost, ls));
        if (wf_early) FA_CUDA(cudaMemcpyAsync(w_first_out + j0, d_wf + j0, 4ull * cnt, cudaMemcpyDeviceToHost, ls));
    }
    for (int l = 1; l < nl; ++l) {
        FA_CUDA(cudaEventRecord(c->lane_done[l], c->lane_s[l]));
        FA_CUDA(cudaStreamWaitEvent(s, c->lane_done[l], 0));
    }
    FA_CUDA(cudaEventRecord(c->ev0, s));
    FA_CUDA(cudaEventRecord(c->ev1, s));
    if (!early) FA_CUDA(cudaMemcpyAsync(out, d_out, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
    if (w_first_out && model && !wf_early)
        FA_CUDA(cudaMemcpyAsync(w_first_out, d_wf, 4ull * n, cudaMemcpyDeviceToHost, s));
    *done = true;
    if (int rc = finish_ext(c, pol, n, s, stats, w_final, launches, 0, mode != FA_POLICY_SINGLE)) {
        drain();
        return rc;
    }
    if (stats) stats->kernel_ms = busy_ms(c, spans, ns);
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

// fa_ext_batch_policy / fa_ext_batch_packed on host buffers of either form.
int ext_batch_host(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_job *jobs, uint32_t n,
                   const HostSeq &hq, const HostSeq &ht, const int32_t *w_first, fa_ext_result *out,
                   int32_t *w_final, fa_ext_stats *stats) {
    auto t0 = std::chrono::steady_clock::now();
    const ExtParams kp = ext_params_of(p);
    auto total = [&]() {
        if (stats)
            stats->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    const int mode = pol ? pol->mode : FA_POLICY_SINGLE;
    if (!c->graph && n >= kPipeMinJobs && (mode == FA_POLICY_SINGLE ? c->slices_single : c->slices_rounds) != 1 &&
        streams(pol, hq)) {
        bool done = false;
        int rc = ext_batch_streamed(c, kp, pol, nullptr, 0.f, jobs, n, hq, ht, nullptr, w_first, out, nullptr,
                                    w_final, stats, &done);
        if (rc) return rc;
        if (done) {
            if (w_final && mode == FA_POLICY_SINGLE)
                for (uint32_t i = 0; i < n; ++i) w_final[i] = jobs[i].w;
            total();
            return FA_OK;
        }
    }
    if (mode == FA_POLICY_SINGLE && !c->graph && n >= kPipeMinJobs && c->slices_single != 1) {
        int rc = ext_batch_pipelined(c, kp, jobs, n, hq, ht, out, stats);
        if (rc) return rc;
        if (w_final)
            for (uint32_t i = 0; i < n; ++i) w_final[i] = jobs[i].w;
        total();
        return FA_OK;
    }
    if (mode != FA_POLICY_SINGLE && !c->graph && n >= kPipeMinJobs && c->slices_rounds != 1) {
        bool done = false;
        int rc = ext_batch_sliced(c, kp, pol, nullptr, 0.f, jobs, n, hq, ht, nullptr, w_first, out, nullptr, w_final,
                                  stats, &done);
        if (rc) return rc;
        if (done) {
            total();
            return FA_OK;
        }
    }
    int max_q = 0;
    if (int rc = check_jobs(jobs, n, hq.npos, ht.npos, kp, packed_qcap_limit(c->smem_optin), &max_q)) return rc;
    std::vector<uint32_t> order;
    std::vector<std::pair<uint32_t, int>> segs;
    length_order(jobs, n, order, segs);
    if (int rc = ensure_ext_buffers(c, n, 0, 0)) return rc;
    if (int rc = ensure_seq_buffers(c, hq, ht)) return rc;
    cudaStream_t s = c->stream;
    FA_CUDA(cudaMemcpyAsync(c->jobs.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->order.p, order.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->qseq.p, hq.p, hq.nbytes, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->tseq.p, ht.p, ht.nbytes, cudaMemcpyHostToDevice, s));
    if (int rc = upload_runs(c, hq, ht, s)) return rc;
    if (mode == FA_POLICY_LEARNED) {
        if (int rc = ensure_policy_buffers(c, n)) return rc;
        FA_CUDA(cudaMemcpyAsync(c->w_first.p, w_first, 4ull * n, cudaMemcpyHostToDevice, s));
    }
    const int32_t *d_wf = mode == FA_POLICY_LEARNED ? c->w_first.as<int32_t>() : nullptr;
    int rc = c->graph
                 ? run_ext_graph(c, kp, pol, n, segs, max_q, max_band_of(jobs, n), {}, nullptr, d_wf, s, stats,
                                 w_final)
                 : run_ext(c, kp, pol, n, segs, max_q, max_band_of(jobs, n), c->jobs.as<fa_job>(),
                           c->order.as<uint32_t>(), c->cq, c->ct, d_wf, c->out.as<fa_ext_result>(), s, stats,
                           w_final);
    if (rc) return rc;
    FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (w_final && mode == FA_POLICY_SINGLE)
        for (uint32_t i = 0; i < n; ++i) w_final[i] = jobs[i].w;
    total();
    return FA_OK;
}

// fa_ext_batch_learned / fa_ext_batch_learned_packed on host buffers of either form.
int ext_learned_host(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_band_model *model, float margin,
                     const fa_job *jobs, uint32_t n, const HostSeq &hq, const HostSeq &ht, const fa_band_hint *hints,
                     fa_ext_result *out, int32_t *w_first_out, int32_t *w_final, fa_ext_stats *stats) {
    auto t0 = std::chrono::steady_clock::now();
    const ExtParams kp = ext_params_of(p);
    auto total = [&]() {
        if (stats)
            stats->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    if (!c->graph && n >= kPipeMinJobs && c->slices_rounds != 1) {
        bool done = false;
        int rc = FA_OK;
        if (streams(pol, hq)) {
            rc = ext_batch_streamed(c, kp, pol, model, margin, jobs, n, hq, ht, hints, nullptr, out, w_first_out,
                                    w_final, stats, &done);
            if (rc) return rc;
            if (done) {
                total();
                return FA_OK;
            }
        }
        rc = ext_batch_sliced(c, kp, pol, model, margin, jobs, n, hq, ht, hints, nullptr, out, w_first_out,
                              w_final, stats, &done);
        if (rc) return rc;
        if (done) {
            total();
            return FA_OK;
        }
    }
    int max_q = 0;
    if (int rc = check_jobs(jobs, n, hq.npos, ht.npos, kp, packed_qcap_limit(c->smem_optin), &max_q)) return rc;
    std::vector<uint32_t> order;
    std::vector<std::pair<uint32_t, int>> segs;
    length_order(jobs, n, order, segs);
    if (int rc = ensure_ext_buffers(c, n, 0, 0)) return rc;
    if (int rc = ensure_seq_buffers(c, hq, ht)) return rc;
    if (int rc = ensure_policy_buffers(c, n)) return rc;
    FA_CUDA(c->feat.ensure(sizeof(float) * 16 * (size_t)n + sizeof(fa_band_hint) * (size_t)n));
    FA_CUDA(c->wbf.ensure(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS));
    cudaStream_t s = c->stream;
    FA_CUDA(cudaMemcpyAsync(c->jobs.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->order.p, order.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->qseq.p, hq.p, hq.nbytes, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->tseq.p, ht.p, ht.nbytes, cudaMemcpyHostToDevice, s));
    if (int rc = upload_runs(c, hq, ht, s)) return rc;
    float *d_x = c->feat.as<float>();
    fa_band_hint *d_h = hints ? reinterpret_cast<fa_band_hint *>(d_x + 16 * (size_t)n) : nullptr;
    if (hints) FA_CUDA(cudaMemcpyAsync(d_h, hints, sizeof(fa_band_hint) * (size_t)n, cudaMemcpyHostToDevice, s));
    std::vector<__nv_bfloat16> wbf;
    float mean[16], sd[16];
    band_model_export(model, wbf, mean, sd);
    FA_CUDA(cudaMemcpyAsync(c->wbf.p, wbf.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice, s));
    auto predict = [&](cudaStream_t st, uint32_t *launches) -> int {
        FA_CUDA(launch_band_features(c->jobs.as<fa_job>(), n, c->cq, c->ct, d_h, kp.max_score, d_x, st,
                                     c->order.as<uint32_t>()));
        FA_CUDA(launch_band_predict(c->wbf.as<__nv_bfloat16>(), mean, sd, d_x, c->jobs.as<fa_job>(), n, margin,
                                    pol->w_min, nullptr, c->w_first.as<int32_t>(), st));
        *launches += 2;
        return FA_OK;
    };
    if (c->graph) {
        // features, prediction and every round in one graph
        std::vector<uint64_t> extra{hq.nbytes, ht.nbytes, (uint64_t)(uintptr_t)d_h};
        uint32_t mb;
        memcpy(&mb, &margin, 4);
        extra.push_back(mb);
        for (int k = 0; k < 16; ++k) {
            uint32_t a, b;
            memcpy(&a, &mean[k], 4);
            memcpy(&b, &sd[k], 4);
            extra.push_back((uint64_t)a << 32 | b);
        }
        int rc = run_ext_graph(c, kp, pol, n, segs, max_q, max_band_of(jobs, n), extra, predict,
                               c->w_first.as<int32_t>(), s, stats, w_final);
        if (rc) return rc;
        if (w_first_out) FA_CUDA(cudaMemcpy(w_first_out, c->w_first.p, 4ull * n, cudaMemcpyDeviceToHost));
        FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
        FA_CUDA(cudaStreamSynchronize(s));
        total();
        return FA_OK;
    }
    FA_CUDA(cudaEventRecord(c->ev0, s));
    {
        uint32_t pl = 0;
        if (int rc = predict(s, &pl)) return rc;
    }
    FA_CUDA(cudaEventRecord(c->ev1, s));
    float pred_ms = 0.f;
    FA_CUDA(cudaEventSynchronize(c->ev1));
    cudaEventElapsedTime(&pred_ms, c->ev0, c->ev1);
    if (w_first_out) FA_CUDA(cudaMemcpy(w_first_out, c->w_first.p, 4ull * n, cudaMemcpyDeviceToHost));
    int rc = run_ext(c, kp, pol, n, segs, max_q, max_band_of(jobs, n), c->jobs.as<fa_job>(), c->order.as<uint32_t>(),
                     c->cq, c->ct, c->w_first.as<int32_t>(), c->out.as<fa_ext_result>(), s, stats, w_final);
    if (rc) return rc;
    FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_ext_result) * (size_t)n, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        stats->kernel_ms += pred_ms;
        stats->kernel_launches += 2;
    }
    total();
    return FA_OK;
}

// Mate-rescue host batch: parameters, validation and the u8 / i16 lane split (the jobs of
// each kind in job order), as fa_mate_sw_batch and fa_pair_batch take them.
struct MateHostPlan {
    MateParams mp;
    std::vector<uint32_t> order;   // u8 jobs, then i16 jobs
    uint32_t n_byte = 0;
    int mq_b = 0, mq_w = 0, mt = 0, mn_b = INT_MAX;
    uint64_t q_end = 0, t_end = 0;   // the jobs' furthest query and target bytes
};

// jobs[0 .. n) checked and split by lane width; `base` numbers them in messages (a slice of a
// larger batch).
int plan_mate_host(const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n, uint64_t qseq_len,
                   uint64_t tseq_len, MateHostPlan *pl, uint32_t base = 0) {
    int mn = 127, mx = 0;
    for (int i = 0; i < 25; ++i) { mn = std::min<int>(mn, p->mat[i]); mx = std::max<int>(mx, p->mat[i]); }
    if (mx <= 0) return fail(FA_ERR_ARG, "scoring matrix needs a positive entry");
    MateParams &mp = pl->mp;
    memcpy(mp.mat, p->mat, 25);
    mp.m = 5;
    mp.o_del = p->o_del; mp.e_del = p->e_del; mp.o_ins = p->o_ins; mp.e_ins = p->e_ins;
    mp.shift = (uint8_t)(256 - mn);
    mp.max = mx;
    std::vector<uint32_t> word_list;
    pl->order.clear();
    for (uint32_t i = 0; i < n; ++i) {
        const fa_mate_job &j = jobs[i];
        if (j.qlen <= 0 || j.tlen < 0) return fail(FA_ERR_ARG, "mate job %u: bad lengths", base + i);
        if (j.tlen > FA_MAX_TLEN) return fail(FA_ERR_CAPACITY, "mate job %u: tlen too long", base + i);
        if (j.q_off + (uint64_t)j.qlen > qseq_len || j.t_off + (uint64_t)j.tlen > tseq_len)
            return fail(FA_ERR_ARG, "mate job %u: sequence range outside the buffers", base + i);
        const bool byte = (j.xtra & FA_KSW_XBYTE) != 0;
        if (byte ? j.qlen > 16 * 32 : j.qlen > 8 * 32)
            return fail(FA_ERR_CAPACITY, "mate job %u: qlen=%d exceeds the %s-lane limit", base + i, j.qlen,
                        byte ? "u8" : "i16");
        pl->q_end = std::max(pl->q_end, j.q_off + (uint64_t)j.qlen);
        pl->t_end = std::max(pl->t_end, j.t_off + (uint64_t)j.tlen);
        (byte ? pl->order : word_list).push_back(i);
        if (byte) {
            pl->mq_b = std::max(pl->mq_b, j.qlen);
            pl->mn_b = std::min(pl->mn_b, j.qlen);
        } else {
            pl->mq_w = std::max(pl->mq_w, j.qlen);
        }
        pl->mt = std::max(pl->mt, j.tlen);
    }
    pl->n_byte = (uint32_t)pl->order.size();
    pl->order.insert(pl->order.end(), word_list.begin(), word_list.end());
    return FA_OK;
}

// The mate SW kernels of a planned batch on device copies (jobs, order, sequences in d_*).
cudaError_t launch_mate_plan(const MateHostPlan &pl, const fa_mate_job *d_jobs, const uint32_t *d_order, uint32_t n,
                             const uint8_t *d_q, const uint8_t *d_t, fa_kswr *d_out, unsigned long long *d_cells,
                             uint32_t *d_status, uint32_t *d_rev, cudaStream_t s, uint32_t *launches) {
    if (pl.n_byte) {
        cudaError_t e = launch_mate_sw(true, d_jobs, d_order, pl.n_byte, d_q, d_t, pl.mp, pl.mn_b, pl.mq_b, pl.mt,
                                       d_out,
                                       d_cells, d_status, d_rev, s);
        if (e != cudaSuccess) return e;
        *launches += 2;
    }
    if (n > pl.n_byte) {
        cudaError_t e = launch_mate_sw(false, d_jobs, d_order + pl.n_byte, n - pl.n_byte, d_q, d_t, pl.mp, 1, pl.mq_w,
                                       pl.mt, d_out, d_cells, d_status, nullptr, s);
        if (e != cudaSuccess) return e;
        ++*launches;
    }
    return cudaSuccess;
}

// Argument checks shared by the host extension entry points.
int check_host_call(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_job *jobs, uint32_t n,
                    const void *out) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (int rc = check_params(p)) return rc;
    if (n == 0) return FA_OK;
    if (!jobs || !out) return fail(FA_ERR_ARG, "null buffer");
    if (pol && (pol->mode < FA_POLICY_SINGLE || pol->mode > FA_POLICY_LEARNED))
        return fail(FA_ERR_ARG, "unknown policy mode %d", pol->mode);
    return FA_OK;
}

int ext_batch_device(fa_ctx *c, const fa_params *p, const fa_job *d_jobs, uint32_t n, const SeqBuf &d_qseq,
                     const SeqBuf &d_tseq, const uint32_t *d_order, fa_ext_result *d_out, void *stream) {
    FA_CUDA(cudaSetDevice(c->device));
    const ExtParams kp = ext_params_of(p);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    FA_CUDA(c->misc.ensure(kMiscBytes));
    FA_CUDA(c->ovf.ensure(3 * sizeof(uint32_t) * (size_t)n));
    FA_CUDA(c->hist.ensure(sizeof(uint32_t) * (FA_MAX_QLEN + 1)));
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    // query-length histogram -> launch classes (one 16 KB read-back per batch)
    FA_CUDA(launch_qlen_hist(d_jobs, n, c->hist.as<uint32_t>(), c->sm_count, s));
    std::vector<uint32_t> hist(FA_MAX_QLEN + 1);
    FA_CUDA(cudaMemcpyAsync(hist.data(), c->hist.p, 4 * hist.size(), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    const int qlimit = packed_qcap_limit(c->smem_optin);
    std::vector<uint32_t> start(FA_MAX_QLEN + 1, 0);
    std::vector<std::pair<uint32_t, int>> segs;
    uint32_t acc = 0, seg_end = 0;
    int seg_cap = -1;
    for (int q = FA_MAX_QLEN; q >= 0; --q) {
        start[q] = acc;
        if (!hist[q]) continue;
        if (q > qlimit) return fail(FA_ERR_CAPACITY, "a job has qlen=%d > %d", q, qlimit);
        if (seg_cap < 0 || q <= ((seg_cap + 31) / 32 - 1) * 32) {
            if (seg_cap >= 0) segs.push_back({seg_end, seg_cap});
            seg_cap = q;
        }
        acc += hist[q];
        seg_end = acc;
    }
    if (seg_cap >= 0) segs.push_back({seg_end, seg_cap});
    const uint32_t *order = d_order;
    if (!order) {
        FA_CUDA(c->order.ensure(4ull * n));
        FA_CUDA(cudaMemcpyAsync(c->hist.p, start.data(), 4 * start.size(), cudaMemcpyHostToDevice, s));
        FA_CUDA(launch_qlen_scatter(d_jobs, n, c->hist.as<uint32_t>(), c->order.as<uint32_t>(), s));
        order = c->order.as<uint32_t>();
    } else {
        segs.assign(1, {n, std::max(0, segs.empty() ? 0 : segs.front().second)});
    }
    int rc0 = FA_OK;
    const Choice kc = resolve_choice(c, kp, d_jobs, order, n, d_qseq, d_tseq, segs.empty() ? 0 : segs.front().second,
                                     -1, d_out, m.status, s, &rc0);
    if (rc0) return rc0;
    std::vector<Choice> seg_kc;
    {
        uint32_t b = 0;
        for (auto &sg : segs) {
            seg_kc.push_back(resolve_choice(c, kp, d_jobs, order + b, sg.first - b, d_qseq, d_tseq, sg.second, -1,
                                            d_out, m.status, s, &rc0));
            if (rc0) return rc0;
            b = sg.first;
        }
        c->last_choice = kc;
    }
    if (segs.size() > 1)
        if (int rc = ensure_side(c, segs.size())) return rc;
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    FA_CUDA(launch_classes(c, segs, [&](size_t k) { return seg_kc[k]; }, d_jobs, order, d_qseq, d_tseq, kp, nullptr,
                           d_out, nullptr, false, nullptr, nullptr, m.status, s, nullptr));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = d_order ? 1u : 2u;
    for (size_t k = 0; k < segs.size(); ++k) c->last_launches += ext_kernels_of(c, seg_kc[k], kp, segs[k].second);
    c->last_stream = s;
    return FA_OK;
}

}  // namespace

// One host mate-SW batch: job checks and plan, the job upload, `upload` for the sequences
// (byte codes into c->qseq / c->tseq on stream s, after the status word is cleared), the SW
// kernels, the results and statistics.
template <class Upload>
int mate_host_batch(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n, uint64_t qseq_len,
                    uint64_t tseq_len, Upload upload, fa_kswr *out, fa_ext_stats *stats,
                    std::chrono::steady_clock::time_point t0) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!p || p->m != 5) return fail(FA_ERR_ARG, "alphabet size must be 5");
    if (n == 0) return FA_OK;
    if (!jobs || !out) return fail(FA_ERR_ARG, "null buffer");
    MateHostPlan pl;
    if (int rc = plan_mate_host(p, jobs, n, qseq_len, tseq_len, &pl)) return rc;
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    FA_CUDA(c->jobs.ensure(sizeof(fa_mate_job) * (size_t)n));
    FA_CUDA(c->order.ensure(4ull * n));
    FA_CUDA(c->out.ensure(sizeof(fa_kswr) * (size_t)n));
    FA_CUDA(c->misc.ensure(kMiscBytes));
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    FA_CUDA(cudaMemcpyAsync(c->jobs.p, jobs, sizeof(fa_mate_job) * (size_t)n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(c->order.p, pl.order.data(), 4ull * n, cudaMemcpyHostToDevice, s));
    if (int rc = upload(s)) return rc;
    FA_CUDA(cudaEventRecord(c->ev0, s));
    uint32_t launches = 0;
    FA_CUDA(c->mate_rev.ensure(4ull * (2 + (size_t)pl.n_byte)));
    FA_CUDA(launch_mate_plan(pl, c->jobs.as<fa_mate_job>(), c->order.as<uint32_t>(), n, c->qseq.as<uint8_t>(),
                             c->tseq.as<uint8_t>(), c->out.as<fa_kswr>(), m.cells, m.status,
                             c->mate_rev.as<uint32_t>(), s, &launches));
    FA_CUDA(cudaEventRecord(c->ev1, s));
    if (int rc = read_status(c, s)) return rc;
    FA_CUDA(cudaMemcpyAsync(out, c->out.p, sizeof(fa_kswr) * (size_t)n, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        unsigned long long cells = 0;
        FA_CUDA(cudaMemcpy(&cells, m.cells, 8, cudaMemcpyDeviceToHost));
        stats->cells = stats->cells_executed = cells;
        stats->kernel_ms = ms;
        stats->kernel_launches = launches;
        stats->jobs = n;
        stats->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return FA_OK;
}

int ensure_host_stage(fa_ctx *c, size_t bytes) {
    if (c->h_stage_cap >= bytes) return FA_OK;
    if (c->h_stage) cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_cap = 0;
    FA_CUDA(cudaMallocHost(&c->h_stage, bytes));
    c->h_stage_cap = bytes;
    return FA_OK;
}

bool host_pinned(const void *p) {
    cudaPointerAttributes pa;
    const bool r = p && cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return r;
}

// Device buffers, streams and events a sliced mate-SW batch runs on: kernels on s, uploads
// on cs, each slice's results (with an early-returned `out`) on ds.
struct MateSliceRes {
    cudaStream_t s, cs, ds;
    cudaEvent_t *slice_ev, *done_ev, ev0;
    fa_mate_job *jobs;
    uint32_t *order;
    uint8_t *q, *t;
    fa_kswr *out;
    unsigned long long *cells;
    uint32_t *status, *rev;
};
constexpr int kMateSlices = 4;

// The byte-code sequences of a sliced mate batch: each slice's new query and target bytes
// copied on the upload stream; nothing to prepare on the kernel stream.
struct MateBytesUp {
    const uint8_t *qseq, *tseq;
    uint8_t *d_q, *d_t;
    int upload(uint64_t qa, uint64_t qb, uint64_t ta, uint64_t tb, cudaStream_t cs) const {
        if (qb > qa) FA_CUDA(cudaMemcpyAsync(d_q + qa, qseq + qa, qb - qa, cudaMemcpyHostToDevice, cs));
        if (tb > ta) FA_CUDA(cudaMemcpyAsync(d_t + ta, tseq + ta, tb - ta, cudaMemcpyHostToDevice, cs));
        return FA_OK;
    }
    int prepare(uint64_t, uint64_t, uint64_t, uint64_t, cudaStream_t) const { return FA_OK; }
    int init(cudaStream_t, cudaStream_t, uint32_t *) const { return FA_OK; }
};

// The 2-bit packed sequences of a sliced mate batch: the N runs go up first and are checked on
// the kernel stream; each slice's new packed words go up on the upload stream and are unpacked
// to byte codes, its N runs applied, on the kernel stream before its kernels (the SW kernels
// read each base many times, from cache).  Slices start on 16-position words, one packed
// 32-bit word each.
struct MatePackedUp {
    HostSeq hq, ht;
    uint8_t *pq, *pt, *d_q, *d_t;
    fa_nrun *rq, *rt;
    uint32_t *status;
    int init(cudaStream_t cs, cudaStream_t, uint32_t *) const {
        if (hq.n_runs) FA_CUDA(cudaMemcpyAsync(rq, hq.runs, sizeof(fa_nrun) * hq.n_runs, cudaMemcpyHostToDevice, cs));
        if (ht.n_runs) FA_CUDA(cudaMemcpyAsync(rt, ht.runs, sizeof(fa_nrun) * ht.n_runs, cudaMemcpyHostToDevice, cs));
        return FA_OK;
    }
    static int up_range(const HostSeq &h, uint8_t *dst, uint64_t a, uint64_t b, cudaStream_t cs) {
        const uint64_t ba = a / 4, bb = std::min<uint64_t>((b + 3) / 4, h.nbytes);
        if (bb > ba) FA_CUDA(cudaMemcpyAsync(dst + ba, h.p + ba, bb - ba, cudaMemcpyHostToDevice, cs));
        return FA_OK;
    }
    int upload(uint64_t qa, uint64_t qb, uint64_t ta, uint64_t tb, cudaStream_t cs) const {
        if (int rc = up_range(hq, pq, qa, qb, cs)) return rc;
        return up_range(ht, pt, ta, tb, cs);
    }
    int prepare(uint64_t qa, uint64_t qb, uint64_t ta, uint64_t tb, cudaStream_t s) const {
        if (qa == 0) {   // the first slice: the runs, uploaded before it, are checked once
            FA_CUDA(launch_runs_check(rq, (uint32_t)hq.n_runs, hq.npos, status, s));
            FA_CUDA(launch_runs_check(rt, (uint32_t)ht.n_runs, ht.npos, status, s));
        }
        FA_CUDA(launch_unpack2_range(pq, qa, qb, rq, (uint32_t)hq.n_runs, d_q, s));
        FA_CUDA(launch_unpack2_range(pt, ta, tb, rt, (uint32_t)ht.n_runs, d_t, s));
        return FA_OK;
    }
};

// Graded job-index slices of a host mate-SW batch (n >= kPipeMinJobs): each slice is planned on
// the host (checks, lane split, its furthest query and target positions) while the GPU works on
// the earlier ones, then its job records and order (staged in the page-locked h_order) go up on
// r.cs with up.upload of the sequence positions up to its furthest job (rounded up to 16, so
// slices never share a 16-position word), up.prepare runs on r.s, and its kernels run on r.s,
// seeing the slice through views of the job and result arrays, so jobs out of sequence order
// only widen a slice's upload; with early_out its results go back on r.ds as soon as it has
// run.  A bad job returns its error (named by its index in the batch) with the earlier slices
// enqueued: the caller drains the streams.  r.rev holds 2 + the largest slice's job count.
template <class SeqUp>
int enqueue_mate_sliced(const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n, uint64_t qseq_len,
                        uint64_t tseq_len, const SeqUp &up, uint32_t *h_order, fa_kswr *early_out,
                        const MateSliceRes &r, uint32_t *launches) {
    uint32_t J[kMateSlices + 1];
    J[0] = 0;
    J[kMateSlices] = n;
    for (int k = 1; k < kMateSlices; ++k) J[k] = (uint32_t)((uint64_t)n * kGradedCum[kMateSlices][k - 1] / 32);
    uint64_t qe = 0, te = 0;
    MateHostPlan pl;
    for (int k = 0; k < kMateSlices; ++k) {
        const uint32_t j0 = J[k], cnt = J[k + 1] - j0;
        pl = MateHostPlan{};
        if (int rc = plan_mate_host(p, jobs + j0, cnt, qseq_len, tseq_len, &pl, j0)) return rc;
        memcpy(h_order + j0, pl.order.data(), 4ull * cnt);
        FA_CUDA(cudaMemcpyAsync(r.jobs + j0, jobs + j0, sizeof(fa_mate_job) * cnt, cudaMemcpyHostToDevice, r.cs));
        FA_CUDA(cudaMemcpyAsync(r.order + j0, h_order + j0, 4ull * cnt, cudaMemcpyHostToDevice, r.cs));
        auto up16 = [](uint64_t x, uint64_t cap) { return std::min(cap, (x + 15) & ~(uint64_t)15); };
        const uint64_t qn = std::max(qe, up16(pl.q_end, qseq_len)), tn = std::max(te, up16(pl.t_end, tseq_len));
        if (int rc = up.upload(qe, qn, te, tn, r.cs)) return rc;
        FA_CUDA(cudaEventRecord(r.slice_ev[k], r.cs));
        FA_CUDA(cudaStreamWaitEvent(r.s, r.slice_ev[k], 0));
        if (k == 0) FA_CUDA(cudaEventRecord(r.ev0, r.s));
        if (int rc = up.prepare(qe, qn, te, tn, r.s)) return rc;
        qe = qn;
        te = tn;
        FA_CUDA(launch_mate_plan(pl, r.jobs + j0, r.order + j0, cnt, r.q, r.t, r.out + j0, r.cells, r.status, r.rev,
                                 r.s, launches));
        if (early_out) {
            FA_CUDA(cudaEventRecord(r.done_ev[k], r.s));
            FA_CUDA(cudaStreamWaitEvent(r.ds, r.done_ev[k], 0));
            FA_CUDA(cudaMemcpyAsync(early_out + j0, r.out + j0, sizeof(fa_kswr) * cnt, cudaMemcpyDeviceToHost, r.ds));
        }
    }
    return FA_OK;
}

// The largest slice enqueue_mate_sliced cuts from n jobs.
uint32_t mate_max_slice(uint32_t n) {
    uint32_t prev = 0, mx = 0;
    for (int k = 1; k <= kMateSlices; ++k) {
        const uint32_t e = k == kMateSlices ? n : (uint32_t)((uint64_t)n * kGradedCum[kMateSlices][k - 1] / 32);
        mx = std::max(mx, e - prev);
        prev = e;
    }
    return mx;
}

// A byte-code host mate-SW batch of kPipeMinJobs jobs or more, sliced (enqueue_mate_sliced)
// on the context's main, copy and prep streams; results into a page-locked `out` come back
// slice by slice.  Results and statistics are those of one launch over the batch.
// `make_up(qseq_dev, tseq_dev)` gives the sequence functor once the byte buffers exist; the
// caller has checked that slicing applies (mate_sliceable).
bool mate_sliceable(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n, const fa_kswr *out) {
    return c && p && p->m == 5 && jobs && out && n >= kPipeMinJobs && c->slices_single != 1;
}

template <class MakeUp>
int mate_host_sliced(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n, uint64_t qseq_len,
                     uint64_t tseq_len, MakeUp make_up, fa_kswr *out, fa_ext_stats *stats,
                     std::chrono::steady_clock::time_point t0) {
    FA_CUDA(cudaSetDevice(c->device));
    FA_CUDA(c->jobs.ensure(sizeof(fa_mate_job) * (size_t)n));
    FA_CUDA(c->order.ensure(4ull * n));
    FA_CUDA(c->out.ensure(sizeof(fa_kswr) * (size_t)n));
    FA_CUDA(c->misc.ensure(kMiscBytes));
    FA_CUDA(c->qseq.ensure(((qseq_len + 15) & ~(uint64_t)15) + 16));   // unpacking writes whole 16-base words
    FA_CUDA(c->tseq.ensure(((tseq_len + 15) & ~(uint64_t)15) + 16));
    FA_CUDA(c->mate_rev.ensure(4ull * (2 + (size_t)mate_max_slice(n))));
    if (int rc = ensure_pipe_streams(c)) return rc;
    if (int rc = ensure_host_stage(c, 4ull * n)) return rc;
    const bool early = host_pinned(out);
    cudaStream_t s = c->stream, cs = c->copy_stream, ds = c->prep_stream;
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    FA_CUDA(cudaEventRecord(c->fork_ev, s));
    FA_CUDA(cudaStreamWaitEvent(cs, c->fork_ev, 0));
    FA_CUDA(cudaStreamWaitEvent(ds, c->fork_ev, 0));
    const MateSliceRes r{s, cs, ds, c->slice_ev, c->done_ev, c->ev0, c->jobs.as<fa_mate_job>(),
                         c->order.as<uint32_t>(), c->qseq.as<uint8_t>(), c->tseq.as<uint8_t>(), c->out.as<fa_kswr>(),
                         m.cells, m.status, c->mate_rev.as<uint32_t>()};
    uint32_t launches = 0;
    int rc = FA_OK;
    const auto up = make_up(c->qseq.as<uint8_t>(), c->tseq.as<uint8_t>(), &rc);
    if (rc == FA_OK) rc = up.init(cs, s, m.status);
    if (rc == FA_OK)
        rc = enqueue_mate_sliced(p, jobs, n, qseq_len, tseq_len, up, static_cast<uint32_t *>(c->h_stage),
                                 early ? out : nullptr, r, &launches);
    if (rc) {
        cudaStreamSynchronize(cs);
        cudaStreamSynchronize(s);
        cudaStreamSynchronize(ds);
        return rc;
    }
    FA_CUDA(cudaEventRecord(c->ev1, s));
    const int rs = read_status(c, s);
    FA_CUDA(cudaStreamSynchronize(ds));
    FA_CUDA(cudaStreamSynchronize(cs));
    if (rs) return rs;
    if (!early) FA_CUDA(cudaMemcpy(out, c->out.p, sizeof(fa_kswr) * (size_t)n, cudaMemcpyDeviceToHost));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        unsigned long long cells = 0;
        FA_CUDA(cudaMemcpy(&cells, m.cells, 8, cudaMemcpyDeviceToHost));
        stats->cells = stats->cells_executed = cells;
        stats->kernel_ms = ms;
        stats->kernel_launches = launches;
        stats->jobs = n;
        stats->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return FA_OK;
}

extern "C" {

const char *fa_last_error(void) { return g_err.c_str(); }
const char *fa_version(void) { return "ferrous_b200 0.1 (sm_100a)"; }

int fa_ctx_create(int device, fa_ctx **out) {
    if (!out) return fail(FA_ERR_ARG, "null out");
    *out = nullptr;
    int ndev = 0;
    FA_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(FA_ERR_ARG, "device %d not present (%d)", device, ndev);
    FA_CUDA(cudaSetDevice(device));
    fa_ctx *c = new fa_ctx();
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        delete c;
        return fail(FA_ERR_CUDA, "device %d is not sm_100-class", device);
    }
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        delete c;
        return fail(FA_ERR_CUDA, "stream/event creation failed");
    }
    *out = c;
    return FA_OK;
}

void fa_ctx_destroy(fa_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    for (DevBuf *b : {&c->jobs, &c->order, &c->qseq, &c->tseq, &c->out, &c->clamped, &c->cells_job,
                      &c->misc, &c->w_first, &c->w_cur, &c->prev, &c->kk, &c->w_final, &c->tries,
                      &c->missed, &c->list_a, &c->list_b, &c->hist, &c->feat, &c->wbf, &c->part_n,
                      &c->part_w, &c->ovf, &c->reg_in, &c->reg_out, &c->col_in, &c->col_plan, &c->col_out, &c->col_pk, &c->part_blk[0], &c->part_blk[1], &c->part_blk[2], &c->part_blk[3],
                      &c->cg_in, &c->cg_scratch, &c->cg_out, &c->mc_in, &c->mc_plan, &c->mc_out, &c->is_buf,
                      &c->qruns, &c->truns})
        b->release();
    for (auto &pr : c->span_ev)
        for (auto &e : pr)
            if (e) cudaEventDestroy(e);
    for (int l = 1; l < fa_ctx::kLanes; ++l) {
        for (int k = 0; k < 2; ++k) {
            if (c->lane_aux[l][k]) cudaStreamDestroy(c->lane_aux[l][k]);
            if (c->lane_join[l][k]) cudaEventDestroy(c->lane_join[l][k]);
        }
        if (c->lane_fork[l]) cudaEventDestroy(c->lane_fork[l]);
        if (c->lane_done[l]) cudaEventDestroy(c->lane_done[l]);
    }
    for (auto &e : c->lane_ev)
        if (e) cudaEventDestroy(e);
    for (DevBuf *b : {&c->pm_jobs, &c->pm_order, &c->pm_q, &c->pm_t, &c->pm_out, &c->pm_misc, &c->pm_rev,
                      &c->mate_rev, &c->mate_pk})
        b->release();
    if (c->pm_ev0) cudaEventDestroy(c->pm_ev0);
    if (c->pm_ev1) cudaEventDestroy(c->pm_ev1);
    if (c->pm_stream) cudaStreamDestroy(c->pm_stream);
    if (c->pm_copy) cudaStreamDestroy(c->pm_copy);
    if (c->pm_fork) cudaEventDestroy(c->pm_fork);
    for (auto &e : c->pm_slice_ev)
        if (e) cudaEventDestroy(e);
    for (int l = 1; l < fa_ctx::kLanes; ++l)
        if (c->lane_s[l]) cudaStreamDestroy(c->lane_s[l]);
    c->lane_misc.release();
    c->ref_pac.release();
    for (int k = 0; k < 2; ++k) {
        if (c->join_ev[k]) cudaEventDestroy(c->join_ev[k]);
        if (c->aux[k]) cudaStreamDestroy(c->aux[k]);
    }
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    for (int k = 0; k < fa_ctx::kSides; ++k) {
        if (c->side[k]) cudaStreamDestroy(c->side[k]);
        if (c->side_fork[k]) cudaEventDestroy(c->side_fork[k]);
        if (c->side_join[k]) cudaEventDestroy(c->side_join[k]);
    }
    c->class_ovf_n.release();
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    for (auto &e : c->slice_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->done_ev)
        if (e) cudaEventDestroy(e);
    if (c->jobs_ev) cudaEventDestroy(c->jobs_ev);
    for (int k = 0; k < kSlices; ++k) {
        if (c->job_ev[k]) cudaEventDestroy(c->job_ev[k]);
        if (c->info_ev[k]) cudaEventDestroy(c->info_ev[k]);
    }
    if (c->prep_stream) cudaStreamDestroy(c->prep_stream);
    if (c->h_slice_info) cudaFreeHost(c->h_slice_info);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    c->chunk_scratch.release();
    if (c->kev0) cudaEventDestroy(c->kev0);
    if (c->kev1) cudaEventDestroy(c->kev1);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int fa_probe_int_peak(fa_ctx *c, int kind, double *ops_per_s, float *ms) {
    if (!c || !ops_per_s) return fail(FA_ERR_ARG, "null argument");
    if (kind < 0 || kind > 9) return fail(FA_ERR_ARG, "unknown probe kind %d", kind);
    FA_CUDA(cudaSetDevice(c->device));
    const double r = probe_int_peak(kind, c->sm_count, c->stream, ms);
    if (r <= 0) return fail(FA_ERR_CUDA, "probe kernel failed");
    *ops_per_s = r;
    return FA_OK;
}

int fa_device_info(fa_ctx *c, int *sm_count, int *smem_optin_bytes) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (sm_count) *sm_count = c->sm_count;
    if (smem_optin_bytes) *smem_optin_bytes = (int)c->smem_optin;
    return FA_OK;
}

uint32_t fa_mate_xtra(int32_t mate_len, int32_t match_score, int32_t min_seed_len) {
    uint32_t x = FA_KSW_XSUBO | FA_KSW_XSTART;
    if (mate_len * match_score < 250) x |= FA_KSW_XBYTE;
    return x | (uint32_t)(min_seed_len * match_score);
}

int fa_ext_batch_policy(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_job *jobs,
                        uint32_t n, const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq,
                        uint64_t tseq_len, const int32_t *w_first, fa_ext_result *out,
                        int32_t *w_final, fa_ext_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (int rc = check_host_call(c, p, pol, jobs, n, out)) return rc;
    if (n == 0) return FA_OK;
    if (!qseq || !tseq) return fail(FA_ERR_ARG, "null buffer");
    if (pol && pol->mode == FA_POLICY_LEARNED && !w_first)
        return fail(FA_ERR_STATE, "learned policy needs w_first (or a loaded band model)");
    FA_CUDA(cudaSetDevice(c->device));
    return ext_batch_host(c, p, pol, jobs, n, host_bytes(qseq, qseq_len), host_bytes(tseq, tseq_len), w_first, out,
                          w_final, stats);
}

int fa_ext_batch_packed(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_job *jobs, uint32_t n,
                        const fa_packed_seq *qseq, const fa_packed_seq *tseq, const int32_t *w_first,
                        fa_ext_result *out, int32_t *w_final, fa_ext_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (int rc = check_host_call(c, p, pol, jobs, n, out)) return rc;
    if (n == 0) return FA_OK;
    HostSeq hq, ht;
    if (int rc = host_packed(qseq, "query", &hq)) return rc;
    if (int rc = host_packed(tseq, "target", &ht)) return rc;
    if (pol && pol->mode == FA_POLICY_LEARNED && !w_first)
        return fail(FA_ERR_STATE, "learned policy needs w_first (or a band model: fa_ext_batch_learned_packed)");
    FA_CUDA(cudaSetDevice(c->device));
    return ext_batch_host(c, p, pol, jobs, n, hq, ht, w_first, out, w_final, stats);
}

int fa_ext_batch_learned(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_band_model *model,
                         float margin, const fa_job *jobs, uint32_t n, const uint8_t *qseq, uint64_t qseq_len,
                         const uint8_t *tseq, uint64_t tseq_len, const fa_band_hint *hints, fa_ext_result *out,
                         int32_t *w_first_out, int32_t *w_final, fa_ext_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!model) return fail(FA_ERR_STATE, "no band model");
    if (!pol || pol->mode != FA_POLICY_LEARNED) return fail(FA_ERR_ARG, "fa_ext_batch_learned needs FA_POLICY_LEARNED");
    if (int rc = check_host_call(c, p, pol, jobs, n, out)) return rc;
    if (n == 0) return FA_OK;
    if (!qseq || !tseq) return fail(FA_ERR_ARG, "null buffer");
    FA_CUDA(cudaSetDevice(c->device));
    return ext_learned_host(c, p, pol, model, margin, jobs, n, host_bytes(qseq, qseq_len), host_bytes(tseq, tseq_len),
                            hints, out, w_first_out, w_final, stats);
}

int fa_ext_batch_learned_packed(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_band_model *model,
                                float margin, const fa_job *jobs, uint32_t n, const fa_packed_seq *qseq,
                                const fa_packed_seq *tseq, const fa_band_hint *hints, fa_ext_result *out,
                                int32_t *w_first_out, int32_t *w_final, fa_ext_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!model) return fail(FA_ERR_STATE, "no band model");
    if (!pol || pol->mode != FA_POLICY_LEARNED)
        return fail(FA_ERR_ARG, "fa_ext_batch_learned_packed needs FA_POLICY_LEARNED");
    if (int rc = check_host_call(c, p, pol, jobs, n, out)) return rc;
    if (n == 0) return FA_OK;
    HostSeq hq, ht;
    if (int rc = host_packed(qseq, "query", &hq)) return rc;
    if (int rc = host_packed(tseq, "target", &ht)) return rc;
    FA_CUDA(cudaSetDevice(c->device));
    return ext_learned_host(c, p, pol, model, margin, jobs, n, hq, ht, hints, out, w_first_out, w_final, stats);
}

int fa_ext_batch(fa_ctx *c, const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq,
                 uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len, fa_ext_result *out,
                 fa_ext_stats *stats) {
    return fa_ext_batch_policy(c, p, nullptr, jobs, n, qseq, qseq_len, tseq, tseq_len, nullptr, out,
                               nullptr, stats);
}

int fa_ext_batch_device(fa_ctx *c, const fa_params *p, const fa_job *d_jobs, uint32_t n,
                        const uint8_t *d_qseq, const uint8_t *d_tseq, const uint32_t *d_order,
                        fa_ext_result *d_out, void *stream) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (int rc = check_params(p)) return rc;
    if (n == 0) return FA_OK;
    if (!d_jobs || !d_qseq || !d_tseq || !d_out) return fail(FA_ERR_ARG, "null buffer");
    // byte codes: the kernels take the caller's word that every job lies inside the buffers
    return ext_batch_device(c, p, d_jobs, n, SeqBuf{d_qseq, ~0ull, nullptr, 0, 0}, SeqBuf{d_tseq, ~0ull, nullptr, 0, 0},
                            d_order, d_out, stream);
}

int fa_ext_batch_packed_device(fa_ctx *c, const fa_params *p, const fa_job *d_jobs, uint32_t n,
                               const fa_packed_seq *d_qseq, const fa_packed_seq *d_tseq, const uint32_t *d_order,
                               fa_ext_result *d_out, void *stream) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (int rc = check_params(p)) return rc;
    if (n == 0) return FA_OK;
    if (!d_jobs || !d_qseq || !d_tseq || !d_out) return fail(FA_ERR_ARG, "null buffer");
    SeqBuf q, t;
    for (auto [src, dst, what] : {std::tuple{d_qseq, &q, "query"}, std::tuple{d_tseq, &t, "target"}}) {
        if (!src->bases || (src->n_nruns && !src->n_runs)) return fail(FA_ERR_ARG, "null packed %s buffer", what);
        if ((uintptr_t)src->bases % 4) return fail(FA_ERR_ARG, "packed %s bases must be 4-byte aligned", what);
        if (src->n_nruns >= (1ull << 32)) return fail(FA_ERR_CAPACITY, "packed %s buffer: too many N runs", what);
        *dst = SeqBuf{src->bases, (src->n_bases + 3) / 4, src->n_runs, (uint32_t)src->n_nruns, 1};
    }
    return ext_batch_device(c, p, d_jobs, n, q, t, d_order, d_out, stream);
}

int fa_ctx_set_kernel(fa_ctx *c, int kernel) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (kernel < FA_KERNEL_AUTO || kernel > FA_KERNEL_ROWS2)
        return fail(FA_ERR_ARG, "unknown kernel choice %d", kernel);
    c->kernel = kernel;
    c->tuned.clear();
    return FA_OK;
}

int fa_ctx_set_threads(fa_ctx *c, int threads_per_block) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (threads_per_block != 64 && threads_per_block != 128 && threads_per_block != 256)
        return fail(FA_ERR_ARG, "threads per block must be 64, 128 or 256 (got %d)", threads_per_block);
    c->threads = threads_per_block;
    return FA_OK;
}

int fa_ctx_kernel_choice(fa_ctx *c, int *kernel, int *threads_per_block, int cap, int *cand_kernel,
                         int *cand_threads, float *cand_ms, int *n_cand) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (kernel) *kernel = c->last_choice.kernel;
    if (threads_per_block) *threads_per_block = c->last_choice.tpb;
    const int nc = (int)c->last_tuning.size();
    for (int k = 0; k < nc && k < cap; ++k) {
        if (cand_kernel) cand_kernel[k] = c->last_tuning[k].first.kernel;
        if (cand_threads) cand_threads[k] = c->last_tuning[k].first.tpb;
        if (cand_ms) cand_ms[k] = c->last_tuning[k].second;
    }
    if (n_cand) *n_cand = nc;
    return FA_OK;
}

int fa_ctx_set_slices(fa_ctx *c, int single_band, int policy_rounds) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    for (int v : {single_band, policy_rounds})
        if (v < -1 || v > kSlices) return fail(FA_ERR_ARG, "slice count %d outside 1..%d", v, kSlices);
    if (single_band) c->slices_single = single_band < 0 ? 0 : single_band;
    if (policy_rounds) c->slices_rounds = policy_rounds < 0 ? 0 : policy_rounds;
    return FA_OK;
}

int fa_ctx_set_graph(fa_ctx *c, int enable) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    FA_CUDA(cudaSetDevice(c->device));
    c->graph = enable != 0;
    if (!c->graph && c->gexec) {
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
        c->gkey.clear();
    }
    return FA_OK;
}

int fa_ctx_set_timing(fa_ctx *c, int enable) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    FA_CUDA(cudaSetDevice(c->device));
    if (enable && !c->kev0) {
        FA_CUDA(cudaEventCreate(&c->kev0));
        FA_CUDA(cudaEventCreate(&c->kev1));
    }
    c->timing = enable != 0;
    return FA_OK;
}

int fa_ctx_last_timing(fa_ctx *c, float *kernel_ms, int *launches) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (launches) *launches = (int)c->last_launches;
    if (kernel_ms) {
        *kernel_ms = 0.f;
        if (c->timing && c->kev0) {
            FA_CUDA(cudaEventSynchronize(c->kev1));
            FA_CUDA(cudaEventElapsedTime(kernel_ms, c->kev0, c->kev1));
        }
    }
    return FA_OK;
}

int fa_ctx_sync(fa_ctx *c) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->last_stream ? c->last_stream : c->stream;
    FA_CUDA(cudaStreamSynchronize(s));
    if (c->misc.p) return read_status(c, s);
    return FA_OK;
}

int fa_mate_sw_batch_device(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *d_jobs, uint32_t n,
                            const uint8_t *d_qseq, const uint8_t *d_tseq, fa_kswr *d_out, void *stream) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!p || p->m != 5) return fail(FA_ERR_ARG, "alphabet size must be 5");
    if (n == 0) return FA_OK;
    if (!d_jobs || !d_qseq || !d_tseq || !d_out) return fail(FA_ERR_ARG, "null buffer");
    int mn = 127, mx = 0;
    for (int i = 0; i < 25; ++i) { mn = std::min<int>(mn, p->mat[i]); mx = std::max<int>(mx, p->mat[i]); }
    if (mx <= 0) return fail(FA_ERR_ARG, "scoring matrix needs a positive entry");
    MateParams mp;
    memcpy(mp.mat, p->mat, 25);
    mp.m = 5;
    mp.o_del = p->o_del; mp.e_del = p->e_del; mp.o_ins = p->o_ins; mp.e_ins = p->e_ins;
    mp.shift = (uint8_t)(256 - mn);
    mp.max = mx;
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    FA_CUDA(c->misc.ensure(kMiscBytes));
    FA_CUDA(c->order.ensure(4ull * n));
    FA_CUDA(c->list_a.ensure(4ull * n));
    FA_CUDA(c->mate_rev.ensure(4ull * (2 + (size_t)n)));
    FA_CUDA(c->hist.ensure(sizeof(uint32_t) * (FA_MAX_QLEN + 1)));
    Misc m = misc_of(c);
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    uint32_t *info = c->hist.as<uint32_t>();
    FA_CUDA(launch_mate_split(d_jobs, n, c->order.as<uint32_t>(), c->list_a.as<uint32_t>(), info, s));
    uint32_t h[8];
    FA_CUDA(cudaMemcpyAsync(h, info, sizeof(h), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (h[5]) return fail(FA_ERR_ARG, "a mate job has qlen <= 0 or tlen < 0");
    if (h[2] > 16 * 32 || h[3] > 8 * 32) return fail(FA_ERR_CAPACITY, "a mate job's query exceeds the lane limit");
    if (h[4] > FA_MAX_TLEN) return fail(FA_ERR_CAPACITY, "a mate job's target is too long");
    uint32_t launches = 1;
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    if (h[0]) {
        FA_CUDA(launch_mate_sw(true, d_jobs, c->order.as<uint32_t>(), h[0], d_qseq, d_tseq, mp,
                               (int)(0xFFFFFFFFu - h[6]), (int)h[2], (int)h[4],
                               d_out, m.cells, m.status, c->mate_rev.as<uint32_t>(), s));
        launches += 2;
    }
    if (h[1]) {
        FA_CUDA(launch_mate_sw(false, d_jobs, c->list_a.as<uint32_t>(), h[1], d_qseq, d_tseq, mp, 1, (int)h[3],
                               (int)h[4], d_out, m.cells, m.status, nullptr, s));
        ++launches;
    }
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = launches;
    c->last_stream = s;
    return FA_OK;
}

int fa_merge_regions_device(fa_ctx *c, const fa_region_opts *opt, const uint32_t *d_chain_first, uint32_t n_chains,
                            const int32_t *d_query_len, const fa_seed_ext *d_seeds, uint32_t n_seeds,
                            const fa_ext_result *d_left, uint32_t n_left, const fa_ext_result *d_right,
                            uint32_t n_right, fa_region *d_out, void *stream) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!opt) return fail(FA_ERR_ARG, "null options");
    if (n_chains == 0) return FA_OK;
    if (!d_chain_first || !d_query_len || !d_out || (n_seeds && !d_seeds) || (n_left && !d_left) ||
        (n_right && !d_right))
        return fail(FA_ERR_ARG, "null buffer");
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    FA_CUDA(c->misc.ensure(kMiscBytes));
    FA_CUDA(cudaMemsetAsync(c->misc.p, 0, 64, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    FA_CUDA(launch_merge_regions(*opt, d_chain_first, n_chains, d_query_len, d_seeds, n_seeds, d_left, n_left, d_right,
                                 n_right, d_out, misc_of(c).status, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = 1;
    c->last_stream = s;
    return FA_OK;
}

int fa_merge_regions(fa_ctx *c, const fa_region_opts *opt, const uint32_t *chain_first, uint32_t n_chains,
                     const int32_t *query_len, const fa_seed_ext *seeds, uint32_t n_seeds,
                     const fa_ext_result *left, uint32_t n_left, const fa_ext_result *right, uint32_t n_right,
                     fa_region *out) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!opt) return fail(FA_ERR_ARG, "null options");
    if (n_chains == 0) return FA_OK;
    if (!chain_first || !query_len || !out || (n_seeds && !seeds) || (n_left && !left) || (n_right && !right))
        return fail(FA_ERR_ARG, "null buffer");
    for (uint32_t k = 0; k < n_chains; ++k)
        if (chain_first[k + 1] < chain_first[k]) return fail(FA_ERR_ARG, "chain_first is not ascending");
    if (chain_first[n_chains] > n_seeds) return fail(FA_ERR_ARG, "a chain's seeds run past the seed array");
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    // one input buffer: chain bounds | query lengths | seeds | left results | right results
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t b_first = up16(4ull * (n_chains + 1)), b_qlen = up16(4ull * n_chains);
    const size_t b_seeds = up16(sizeof(fa_seed_ext) * n_seeds), b_left = up16(sizeof(fa_ext_result) * n_left);
    const size_t b_right = up16(sizeof(fa_ext_result) * n_right);
    FA_CUDA(c->reg_in.ensure(b_first + b_qlen + b_seeds + b_left + b_right));
    FA_CUDA(c->reg_out.ensure(sizeof(fa_region) * n_chains));
    char *d = c->reg_in.as<char>();
    uint32_t *d_first = reinterpret_cast<uint32_t *>(d);
    int32_t *d_qlen = reinterpret_cast<int32_t *>(d + b_first);
    fa_seed_ext *d_seeds = reinterpret_cast<fa_seed_ext *>(d + b_first + b_qlen);
    fa_ext_result *d_left = reinterpret_cast<fa_ext_result *>(d + b_first + b_qlen + b_seeds);
    fa_ext_result *d_right = reinterpret_cast<fa_ext_result *>(d + b_first + b_qlen + b_seeds + b_left);
    FA_CUDA(cudaMemcpyAsync(d_first, chain_first, 4ull * (n_chains + 1), cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_qlen, query_len, 4ull * n_chains, cudaMemcpyHostToDevice, s));
    if (n_seeds) FA_CUDA(cudaMemcpyAsync(d_seeds, seeds, sizeof(fa_seed_ext) * n_seeds, cudaMemcpyHostToDevice, s));
    if (n_left) FA_CUDA(cudaMemcpyAsync(d_left, left, sizeof(fa_ext_result) * n_left, cudaMemcpyHostToDevice, s));
    if (n_right)
        FA_CUDA(cudaMemcpyAsync(d_right, right, sizeof(fa_ext_result) * n_right, cudaMemcpyHostToDevice, s));
    if (int rc = fa_merge_regions_device(c, opt, d_first, n_chains, d_qlen, n_seeds ? d_seeds : nullptr, n_seeds,
                                         n_left ? d_left : nullptr, n_left, n_right ? d_right : nullptr, n_right,
                                         c->reg_out.as<fa_region>(), s))
        return rc;
    FA_CUDA(cudaMemcpyAsync(out, c->reg_out.p, sizeof(fa_region) * n_chains, cudaMemcpyDeviceToHost, s));
    return read_status(c, s);
}

}  // extern "C"

namespace {

// Device side of one job collection: the outputs on the device and the totals (x: window
// bytes, y / z: left / right jobs, w: seed-table entries).
struct CollectDev {
    fa_job *left = nullptr, *right = nullptr;
    uint8_t *q = nullptr, *t = nullptr;
    fa_seed_ext *ext = nullptr;
    uint32_t *first = nullptr;
    uint64_t *win = nullptr;
    ulonglong4 tot{};
    uint64_t read_bytes = 0;
};

// Validates, uploads, plans and fills one job collection on the context's stream.  `check`
// sees the totals (counts already filled) before the fill and may refuse the call (output
// capacity, null buffers).  d->left == nullptr on return: no chains, nothing launched.
template <class Check>
int collect_ext_run(fa_ctx *c, const fa_collect_opts *opt, const uint8_t *pac, uint64_t l_pac, const uint8_t *reads,
                    const uint64_t *read_off, uint32_t n_reads, const fa_chain *chains, uint32_t n_chains,
                    const fa_seed *seeds, uint32_t n_seeds, uint32_t *chain_first, uint64_t *chain_win,
                    fa_collect_counts *counts, Check check, CollectDev *d) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!opt || !counts || !chain_first) return fail(FA_ERR_ARG, "null argument");
    *counts = fa_collect_counts{};
    if (n_chains && (!chains || !chain_win)) return fail(FA_ERR_ARG, "null chain buffer");
    if (n_reads && (!read_off || !reads)) return fail(FA_ERR_ARG, "null read buffer");
    if (n_seeds && !seeds) return fail(FA_ERR_ARG, "null seed buffer");
    if (l_pac == 0) return fail(FA_ERR_ARG, "empty packed reference");
    if (!pac && c->ref_l_pac != l_pac)
        return fail(FA_ERR_ARG, "no resident reference of %llu bases (fa_ctx_set_reference)", (unsigned long long)l_pac);
    if (l_pac > (1ull << 62)) return fail(FA_ERR_ARG, "packed reference too long");
    // the rules the reference's slices and windows would panic on (collect_soa.rs:150-209):
    // the read offsets here (they size the upload), the chains and seeds on the device
    // (collect_check_kernel) before anything uses the plans
    for (uint32_t r = 0; r < n_reads; ++r) {
        if (read_off[r + 1] < read_off[r]) return fail(FA_ERR_ARG, "read_off is not ascending");
        if (read_off[r + 1] - read_off[r] > (uint64_t)INT32_MAX) return fail(FA_ERR_ARG, "a read is too long");
    }
    chain_first[0] = 0;
    if (n_chains == 0) return FA_OK;
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const uint64_t read_bytes = read_off[n_reads];   // reads[0 .. read_off[n_reads]) travel
    const size_t b_pac = pac ? up16((size_t)((l_pac + 3) / 4)) : 0, b_reads = up16(read_bytes + 1);
    const size_t b_off = up16(8ull * (n_reads + 1)), b_chains = up16(sizeof(fa_chain) * n_chains);
    const size_t b_seeds = up16(sizeof(fa_seed) * n_seeds);
    FA_CUDA(c->col_in.ensure(b_pac + b_reads + b_off + b_chains + b_seeds));
    char *in = c->col_in.as<char>();
    const uint8_t *d_pac = pac ? reinterpret_cast<uint8_t *>(in) : c->ref_pac.as<uint8_t>();
    uint8_t *d_reads = reinterpret_cast<uint8_t *>(in + b_pac);
    uint64_t *d_off = reinterpret_cast<uint64_t *>(in + b_pac + b_reads);
    fa_chain *d_chains = reinterpret_cast<fa_chain *>(in + b_pac + b_reads + b_off);
    fa_seed *d_seeds = reinterpret_cast<fa_seed *>(in + b_pac + b_reads + b_off + b_chains);
    if (pac) FA_CUDA(cudaMemcpyAsync(in, pac, (size_t)((l_pac + 3) / 4), cudaMemcpyHostToDevice, s));
    if (read_bytes) FA_CUDA(cudaMemcpyAsync(d_reads, reads, read_bytes, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_off, read_off, 8ull * (n_reads + 1), cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_chains, chains, sizeof(fa_chain) * n_chains, cudaMemcpyHostToDevice, s));
    if (n_seeds) FA_CUDA(cudaMemcpyAsync(d_seeds, seeds, sizeof(fa_seed) * n_seeds, cudaMemcpyHostToDevice, s));
    const size_t nb = collect_scan_blocks(n_chains);
    const size_t b_plan = up16(sizeof(CollectPlan) * n_chains);
    FA_CUDA(c->col_plan.ensure(b_plan + sizeof(ulonglong4) * (nb + 2)));
    CollectPlan *d_plan = c->col_plan.as<CollectPlan>();
    ulonglong4 *d_sums = reinterpret_cast<ulonglong4 *>(c->col_plan.as<char>() + b_plan);
    unsigned long long *d_bad = reinterpret_cast<unsigned long long *>(d_sums + nb + 1);
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    FA_CUDA(launch_collect_plan(*opt, l_pac, d_off, n_reads, d_chains, n_chains, d_seeds, n_seeds, d_plan, d_sums,
                                d_bad, s));
    ulonglong4 tot;
    unsigned long long bad[2];
    FA_CUDA(cudaMemcpyAsync(&tot, d_sums + nb, sizeof(tot), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaMemcpyAsync(bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    for (const unsigned long long b : bad) {
        static const char *const kWhy[] = {"", "read_off is not ascending", "a read is too long",
                                           "a chain's read index is out of range",
                                           "a chain's seeds run past the seed array", "a seed lies outside its read",
                                           "a seed lies outside the reference"};
        const unsigned code = (unsigned)(b & 0xFF);
        if (b != ~0ull && code >= 1 && code <= 6) return fail(FA_ERR_ARG, "%s", kWhy[code]);
    }
    counts->n_left = (uint32_t)tot.y;
    counts->n_right = (uint32_t)tot.z;
    counts->n_seed_ext = (uint32_t)tot.w;
    counts->qbuf_len = 2 * read_bytes;
    counts->tbuf_len = tot.x;
    if (int rc = check(tot)) return rc;
    const size_t b_left = up16(sizeof(fa_job) * tot.y), b_right = up16(sizeof(fa_job) * tot.z);
    const size_t b_q = up16(2 * read_bytes + 1), b_t = up16(tot.x + 1), b_ext = up16(sizeof(fa_seed_ext) * tot.w);
    const size_t b_first = up16(4ull * (n_chains + 1)), b_win = up16(16ull * n_chains);
    FA_CUDA(c->col_out.ensure(b_left + b_right + b_q + b_t + b_ext + b_first + b_win));
    char *o = c->col_out.as<char>();
    fa_job *d_left = reinterpret_cast<fa_job *>(o);
    fa_job *d_right = reinterpret_cast<fa_job *>(o + b_left);
    uint8_t *d_q = reinterpret_cast<uint8_t *>(o + b_left + b_right);
    uint8_t *d_t = reinterpret_cast<uint8_t *>(o + b_left + b_right + b_q);
    fa_seed_ext *d_ext = reinterpret_cast<fa_seed_ext *>(o + b_left + b_right + b_q + b_t);
    uint32_t *d_first = reinterpret_cast<uint32_t *>(o + b_left + b_right + b_q + b_t + b_ext);
    uint64_t *d_win = reinterpret_cast<uint64_t *>(o + b_left + b_right + b_q + b_t + b_ext + b_first);
    FA_CUDA(launch_collect_fill(*opt, d_pac, l_pac, d_reads, d_off, n_reads, d_chains, n_chains, d_seeds, d_plan,
                                d_left, d_right, d_q, d_t, d_ext, d_first, d_win, s));
    c->last_launches = 7;
    c->last_stream = s;
    *d = CollectDev{d_left, d_right, d_q, d_t, d_ext, d_first, d_win, tot, read_bytes};
    return FA_OK;
}

// The host outputs common to both collection entries: jobs, seed table, chain bounds.
int collect_ext_copy_common(fa_ctx *c, const CollectDev &d, uint32_t n_chains, fa_job *left_jobs,
                            fa_job *right_jobs, fa_seed_ext *seed_ext, uint32_t *chain_first, uint64_t *chain_win) {
    cudaStream_t s = c->stream;
    const ulonglong4 &tot = d.tot;
    if (tot.y) FA_CUDA(cudaMemcpyAsync(left_jobs, d.left, sizeof(fa_job) * tot.y, cudaMemcpyDeviceToHost, s));
    if (tot.z) FA_CUDA(cudaMemcpyAsync(right_jobs, d.right, sizeof(fa_job) * tot.z, cudaMemcpyDeviceToHost, s));
    if (tot.w) FA_CUDA(cudaMemcpyAsync(seed_ext, d.ext, sizeof(fa_seed_ext) * tot.w, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaMemcpyAsync(chain_first, d.first, 4ull * n_chains, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaMemcpyAsync(chain_win, d.win, 16ull * n_chains, cudaMemcpyDeviceToHost, s));
    chain_first[n_chains] = (uint32_t)tot.w;
    return FA_OK;
}

}  // namespace

extern "C" {

int fa_ctx_set_reference(fa_ctx *c, const uint8_t *pac, uint64_t l_pac) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    FA_CUDA(cudaSetDevice(c->device));
    c->ref_l_pac = 0;
    if (!pac) {
        c->ref_pac.release();
        return FA_OK;
    }
    if (l_pac == 0 || l_pac > (1ull << 62)) return fail(FA_ERR_ARG, "empty or oversized packed reference");
    const size_t b = (size_t)((l_pac + 3) / 4);
    FA_CUDA(c->ref_pac.ensure(b + 16));
    FA_CUDA(cudaMemcpy(c->ref_pac.p, pac, b, cudaMemcpyHostToDevice));
    c->ref_l_pac = l_pac;
    return FA_OK;
}

int fa_collect_ext_jobs(fa_ctx *c, const fa_collect_opts *opt, const uint8_t *pac, uint64_t l_pac,
                        const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads,
                        const fa_chain *chains, uint32_t n_chains, const fa_seed *seeds, uint32_t n_seeds,
                        fa_job *left_jobs, fa_job *right_jobs, uint8_t *qbuf, uint8_t *tbuf, uint64_t tbuf_cap,
                        fa_seed_ext *seed_ext, uint32_t *chain_first, uint64_t *chain_win,
                        fa_collect_counts *counts) {
    CollectDev d;
    auto check = [&](const ulonglong4 &tot) -> int {
        if (tot.x > tbuf_cap) return fail(FA_ERR_CAPACITY, "tbuf_cap is below the windows' bytes (counts->tbuf_len)");
        if ((tot.y && !left_jobs) || (tot.z && !right_jobs) || (tot.w && !seed_ext) || (counts->qbuf_len && !qbuf) ||
            (tot.x && !tbuf))
            return fail(FA_ERR_ARG, "null output buffer");
        return FA_OK;
    };
    if (int rc = collect_ext_run(c, opt, pac, l_pac, reads, read_off, n_reads, chains, n_chains, seeds, n_seeds,
                                 chain_first, chain_win, counts, check, &d))
        return rc;
    if (!d.left) return FA_OK;
    cudaStream_t s = c->stream;
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    if (d.read_bytes) FA_CUDA(cudaMemcpyAsync(qbuf, d.q, 2 * d.read_bytes, cudaMemcpyDeviceToHost, s));
    if (d.tot.x) FA_CUDA(cudaMemcpyAsync(tbuf, d.t, d.tot.x, cudaMemcpyDeviceToHost, s));
    if (int rc = collect_ext_copy_common(c, d, n_chains, left_jobs, right_jobs, seed_ext, chain_first, chain_win))
        return rc;
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

int fa_collect_ext_jobs_packed(fa_ctx *c, const fa_collect_opts *opt, const uint8_t *pac, uint64_t l_pac,
                               const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads,
                               const fa_chain *chains, uint32_t n_chains, const fa_seed *seeds, uint32_t n_seeds,
                               fa_job *left_jobs, fa_job *right_jobs, uint8_t *qbases, fa_nrun *qruns,
                               uint64_t qruns_cap, uint8_t *tbases, uint64_t tbases_cap, fa_nrun *truns,
                               uint64_t truns_cap, fa_seed_ext *seed_ext, uint32_t *chain_first,
                               uint64_t *chain_win, fa_collect_counts *counts, uint64_t *n_runs) {
    if (!n_runs) return fail(FA_ERR_ARG, "null argument");
    n_runs[0] = n_runs[1] = 0;
    CollectDev d;
    auto check = [&](const ulonglong4 &tot) -> int {
        if ((tot.x + 3) / 4 > tbases_cap)
            return fail(FA_ERR_CAPACITY, "tbases_cap is below the packed windows' bytes ((counts->tbuf_len + 3) / 4)");
        if ((tot.y && !left_jobs) || (tot.z && !right_jobs) || (tot.w && !seed_ext) || (counts->qbuf_len && !qbases) ||
            (tot.x && !tbases) || (qruns_cap && !qruns) || (truns_cap && !truns))
            return fail(FA_ERR_ARG, "null output buffer");
        return FA_OK;
    };
    if (int rc = collect_ext_run(c, opt, pac, l_pac, reads, read_off, n_reads, chains, n_chains, seeds, n_seeds,
                                 chain_first, chain_win, counts, check, &d))
        return rc;
    if (!d.left) return FA_OK;
    cudaStream_t s = c->stream;
    // pack both buffers and list their N runs on the device (the run lists hold at most one
    // run per two bases), then bring back the packed bytes and the runs
    const uint64_t nq = 2 * d.read_bytes, nt = d.tot.x;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const uint64_t rq_cap = std::min<uint64_t>(qruns_cap, nq / 2 + 1), rt_cap = std::min<uint64_t>(truns_cap, nt / 2 + 1);
    const size_t b_pq = up16(4 * ((nq + 15) / 16) + 4), b_pt = up16(4 * ((nt + 15) / 16) + 4);
    const size_t b_rq = up16(sizeof(fa_nrun) * rq_cap), b_rt = up16(sizeof(fa_nrun) * rt_cap);
    const size_t wq = pack_runs_scratch_words(nq), wt = pack_runs_scratch_words(nt);
    FA_CUDA(c->col_pk.ensure(b_pq + b_pt + b_rq + b_rt + 4 * (wq + wt)));
    char *k = c->col_pk.as<char>();
    uint8_t *d_pq = reinterpret_cast<uint8_t *>(k), *d_pt = reinterpret_cast<uint8_t *>(k + b_pq);
    fa_nrun *d_rq = reinterpret_cast<fa_nrun *>(k + b_pq + b_pt);
    fa_nrun *d_rt = reinterpret_cast<fa_nrun *>(k + b_pq + b_pt + b_rq);
    uint32_t *d_sq = reinterpret_cast<uint32_t *>(k + b_pq + b_pt + b_rq + b_rt), *d_st = d_sq + wq;
    FA_CUDA(launch_pack2(d.q, nq, d_pq, s));
    FA_CUDA(launch_pack2(d.t, nt, d_pt, s));
    FA_CUDA(launch_nruns(d.q, nq, d_rq, rq_cap, d_sq, s));
    FA_CUDA(launch_nruns(d.t, nt, d_rt, rt_cap, d_st, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches += 8;
    uint32_t cnt[2];
    FA_CUDA(cudaMemcpyAsync(&cnt[0], d_sq + wq - 1, 4, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaMemcpyAsync(&cnt[1], d_st + wt - 1, 4, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    n_runs[0] = cnt[0];
    n_runs[1] = cnt[1];
    if (cnt[0] > qruns_cap || cnt[1] > truns_cap)
        return fail(FA_ERR_CAPACITY, "an N-run buffer is too small (n_runs holds the counts)");
    if (nq) FA_CUDA(cudaMemcpyAsync(qbases, d_pq, (nq + 3) / 4, cudaMemcpyDeviceToHost, s));
    if (nt) FA_CUDA(cudaMemcpyAsync(tbases, d_pt, (nt + 3) / 4, cudaMemcpyDeviceToHost, s));
    if (cnt[0]) FA_CUDA(cudaMemcpyAsync(qruns, d_rq, sizeof(fa_nrun) * cnt[0], cudaMemcpyDeviceToHost, s));
    if (cnt[1]) FA_CUDA(cudaMemcpyAsync(truns, d_rt, sizeof(fa_nrun) * cnt[1], cudaMemcpyDeviceToHost, s));
    if (int rc = collect_ext_copy_common(c, d, n_chains, left_jobs, right_jobs, seed_ext, chain_first, chain_win))
        return rc;
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

namespace {

// Device side of one CIGAR batch: the outputs in their capacity slots.
struct CigarRun {
    CigarPlan *plan = nullptr;
    fa_cigar_result *out = nullptr;
    uint32_t *cig = nullptr;
    uint8_t *ref = nullptr, *qry = nullptr;
    uint64_t n_cig = 0, n_ref = 0, n_qry = 0;
};

// Validates the jobs, uploads them with the sequences and launches the kernel on the
// context's stream.
int cigar_launch(fa_ctx *c, const fa_params *p, const fa_cigar_job *jobs, uint32_t n, const uint8_t *qseq,
                 uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len, CigarRun *r) {
    // output and scratch offsets per job (the reference would panic on a range past its slices),
    // and the band order after them, built in page-locked staging so they go up asynchronously
    if (int rc = ensure_host_stage(c, (sizeof(CigarPlan) + 4) * (size_t)n)) return rc;
    CigarPlan *plan = static_cast<CigarPlan *>(c->h_stage);
    uint32_t *order = reinterpret_cast<uint32_t *>(plan + n);
    uint64_t cig = 0, ref = 0, qry = 0, eh = 0, tb = 0;
    int max_mat = 0, qmax = 0;
    for (int i = 0; i < 25; ++i) max_mat = std::max<int>(max_mat, p->mat[i]);
    bool narrow = true;     // every score fits the shared-memory kernel's 16-bit row state
    bool narrow13 = true;   // ... and 13 bits, leaving room for the query codes in the words
    for (uint32_t k = 0; k < n; ++k) {
        const fa_cigar_job &j = jobs[k];
        if (j.qlen < 0 || j.tlen < 0 || j.w < 0) return fail(FA_ERR_ARG, "cigar job %u: negative length or band", k);
        if (j.qlen > FA_MAX_QLEN || j.tlen > FA_MAX_TLEN) return fail(FA_ERR_CAPACITY, "cigar job %u too long", k);
        if (j.q_off + (uint64_t)j.qlen > qseq_len || j.t_off + (uint64_t)j.tlen > tseq_len)
            return fail(FA_ERR_ARG, "cigar job %u: range outside the sequence buffers", k);
        CigarPlan &pl = plan[k];
        pl.cig = cig; pl.ref = ref; pl.qry = qry; pl.eh = eh; pl.tb = tb;
        pl.wpr = cigar_band_words(j.qlen, j.w);
        pl._pad = 0;
        cig += (uint64_t)j.qlen + j.tlen + 2;
        ref += (uint64_t)j.tlen;
        qry += (uint64_t)j.qlen;
        eh += (uint64_t)j.qlen + 1;
        tb += (uint64_t)j.tlen * (pl.wpr + 1);   // per row: a header word, then the codes
        qmax = std::max(qmax, j.qlen);
        narrow = narrow && j.h0 >= 0 && (long long)j.h0 + (long long)j.qlen * max_mat <= 32767;
        narrow13 = narrow13 && j.h0 >= 0 && (long long)j.h0 + (long long)j.qlen * max_mat <= 8191;
    }
    const bool smem = narrow && qmax <= cigar_smem_qcap();
    // shared-memory kernel: jobs ordered by band, widest first (a counting sort), so that a
    // warp's jobs run rows of similar length
    if (smem) {
        constexpr int kBins = 1024;
        std::vector<uint32_t> cnt(kBins + 1, 0);
        auto bin = [&](uint32_t k) { return kBins - 1 - std::min(jobs[k].w, kBins - 1); };
        for (uint32_t k = 0; k < n; ++k) ++cnt[bin(k) + 1];
        for (int b = 0; b < kBins; ++b) cnt[b + 1] += cnt[b];
        for (uint32_t k = 0; k < n; ++k) order[cnt[bin(k)]++] = k;
    }
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t b_jobs = up16(sizeof(fa_cigar_job) * n), b_plan = up16(sizeof(CigarPlan) * n);
    // (the kernel loads a step's eight query bases together, up to seven past a job's end)
    const size_t b_q = up16(qseq_len + 8), b_t = up16(tseq_len + 1), b_ord = smem ? up16(4ull * n) : 0;
    FA_CUDA(c->cg_in.ensure(b_jobs + b_plan + b_q + b_t + b_ord));
    char *in = c->cg_in.as<char>();
    fa_cigar_job *d_jobs = reinterpret_cast<fa_cigar_job *>(in);
    CigarPlan *d_plan = reinterpret_cast<CigarPlan *>(in + b_jobs);
    uint8_t *d_q = reinterpret_cast<uint8_t *>(in + b_jobs + b_plan);
    uint8_t *d_t = reinterpret_cast<uint8_t *>(in + b_jobs + b_plan + b_q);
    uint32_t *d_order = reinterpret_cast<uint32_t *>(in + b_jobs + b_plan + b_q + b_t);
    const size_t b_eh = smem ? 0 : up16(sizeof(int2) * eh), b_tb = up16(4 * tb);
    FA_CUDA(c->cg_scratch.ensure(b_eh + b_tb));
    int2 *d_eh = c->cg_scratch.as<int2>();
    uint32_t *d_tb = reinterpret_cast<uint32_t *>(c->cg_scratch.as<char>() + b_eh);
    const size_t b_out = up16(sizeof(fa_cigar_result) * n), b_cig = up16(4 * cig);
    const size_t b_ref = up16(ref + 1), b_qry = up16(qry + 1);
    FA_CUDA(c->cg_out.ensure(b_out + b_cig + b_ref + b_qry));
    char *o = c->cg_out.as<char>();
    r->plan = d_plan;
    r->out = reinterpret_cast<fa_cigar_result *>(o);
    r->cig = reinterpret_cast<uint32_t *>(o + b_out);
    r->ref = reinterpret_cast<uint8_t *>(o + b_out + b_cig);
    r->qry = reinterpret_cast<uint8_t *>(o + b_out + b_cig + b_ref);
    r->n_cig = cig;
    r->n_ref = ref;
    r->n_qry = qry;
    FA_CUDA(cudaMemcpyAsync(d_jobs, jobs, sizeof(fa_cigar_job) * n, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_plan, plan, sizeof(CigarPlan) * n, cudaMemcpyHostToDevice, s));
    if (smem) FA_CUDA(cudaMemcpyAsync(d_order, order, 4ull * n, cudaMemcpyHostToDevice, s));
    if (qseq_len) FA_CUDA(cudaMemcpyAsync(d_q, qseq, qseq_len, cudaMemcpyHostToDevice, s));
    if (tseq_len) FA_CUDA(cudaMemcpyAsync(d_t, tseq, tseq_len, cudaMemcpyHostToDevice, s));
    const ExtParams kp = ext_params_of(p);
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    if (smem)
        FA_CUDA(launch_cigar_smem(d_jobs, d_plan, d_order, n, qmax, narrow13, d_q, d_t, kp, p->pen_clip3, d_tb, r->out,
                                  r->cig, r->ref, r->qry, s));
    else
        FA_CUDA(launch_cigar(d_jobs, d_plan, n, d_q, d_t, kp, p->pen_clip3, d_eh, d_tb, r->out, r->cig, r->ref,
                             r->qry, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = 1;
    c->last_stream = s;
    return FA_OK;
}

}  // namespace

int fa_cigar_batch(fa_ctx *c, const fa_params *p, const fa_cigar_job *jobs, uint32_t n, const uint8_t *qseq,
                   uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len, fa_cigar_result *out, uint32_t *cigar,
                   uint8_t *ref_aligned, uint8_t *query_aligned) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (int rc = check_params(p)) return rc;
    if (n == 0) return FA_OK;
    if (!jobs || !out || !cigar || !ref_aligned || !query_aligned) return fail(FA_ERR_ARG, "null buffer");
    CigarRun r;
    if (int rc = cigar_launch(c, p, jobs, n, qseq, qseq_len, tseq, tseq_len, &r)) return rc;
    cudaStream_t s = c->stream;
    FA_CUDA(cudaMemcpyAsync(out, r.out, sizeof(fa_cigar_result) * n, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaMemcpyAsync(cigar, r.cig, 4 * r.n_cig, cudaMemcpyDeviceToHost, s));
    if (r.n_ref) FA_CUDA(cudaMemcpyAsync(ref_aligned, r.ref, r.n_ref, cudaMemcpyDeviceToHost, s));
    if (r.n_qry) FA_CUDA(cudaMemcpyAsync(query_aligned, r.qry, r.n_qry, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

int fa_cigar_batch_packed(fa_ctx *c, const fa_params *p, const fa_cigar_job *jobs, uint32_t n, const uint8_t *qseq,
                          uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len, fa_cigar_result *out,
                          uint32_t *cigar, uint64_t cigar_cap, uint64_t *cigar_first, uint8_t *ref_aligned,
                          uint8_t *query_aligned) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (int rc = check_params(p)) return rc;
    if (n == 0) return FA_OK;
    if (!jobs || !out || !cigar_first || !ref_aligned || !query_aligned) return fail(FA_ERR_ARG, "null buffer");
    CigarRun r;
    if (int rc = cigar_launch(c, p, jobs, n, qseq, qseq_len, tseq, tseq_len, &r)) return rc;
    cudaStream_t s = c->stream;
    FA_CUDA(cudaMemcpyAsync(out, r.out, sizeof(fa_cigar_result) * n, cudaMemcpyDeviceToHost, s));
    if (r.n_ref) FA_CUDA(cudaMemcpyAsync(ref_aligned, r.ref, r.n_ref, cudaMemcpyDeviceToHost, s));
    if (r.n_qry) FA_CUDA(cudaMemcpyAsync(query_aligned, r.qry, r.n_qry, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    uint64_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        cigar_first[k] = total;
        total += (uint64_t)out[k].n_cigar;
    }
    if (total > cigar_cap)
        return fail(FA_ERR_CAPACITY, "cigar buffer holds %llu words, the batch has %llu", (unsigned long long)cigar_cap,
                    (unsigned long long)total);
    if (total == 0) return FA_OK;
    if (!cigar) return fail(FA_ERR_ARG, "null buffer");
    // the packed words and their offsets go to the scratch, which the kernel no longer needs
    const size_t b_first = (sizeof(uint64_t) * n + 15) & ~(size_t)15;
    FA_CUDA(c->cg_scratch.ensure(b_first + 4 * total));
    uint64_t *d_first = c->cg_scratch.as<uint64_t>();
    uint32_t *d_packed = reinterpret_cast<uint32_t *>(c->cg_scratch.as<char>() + b_first);
    FA_CUDA(cudaMemcpyAsync(d_first, cigar_first, sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s));
    FA_CUDA(launch_cigar_pack(r.plan, r.out, d_first, n, r.cig, d_packed, s));
    c->last_launches = 2;
    FA_CUDA(cudaMemcpyAsync(cigar, d_packed, 4 * total, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

int fa_collect_mate_jobs(fa_ctx *c, const fa_rescue_opts *opt, const fa_insert_bounds *bounds4, const uint8_t *pac,
                         uint64_t l_pac, const uint64_t *chr_off, const uint64_t *chr_len, uint32_t n_chr,
                         const uint8_t *reads, const uint64_t *read_off, uint32_t n_reads, const fa_rescue_aln *alns,
                         uint32_t n_alns, const fa_rescue_cand *cands, uint32_t n_cand, fa_mate_job *jobs,
                         fa_rescue_job_info *info, uint8_t *qbuf, uint64_t qbuf_cap, uint8_t *tbuf,
                         uint64_t tbuf_cap, fa_collect_counts *counts) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!opt || !bounds4 || !counts) return fail(FA_ERR_ARG, "null argument");
    *counts = fa_collect_counts{};
    if (n_cand == 0) return FA_OK;
    if (!cands || !jobs || !info || !read_off || !reads || (n_alns && !alns)) return fail(FA_ERR_ARG, "null buffer");
    if (l_pac == 0 || l_pac > (1ull << 62)) return fail(FA_ERR_ARG, "empty or oversized packed reference");
    if (!pac && c->ref_l_pac != l_pac)
        return fail(FA_ERR_ARG, "no resident reference of %llu bases (fa_ctx_set_reference)", (unsigned long long)l_pac);
    if (n_chr == 0 || !chr_off || !chr_len) return fail(FA_ERR_ARG, "no reference sequences");
    for (uint32_t k = 0; k < n_chr; ++k) {
        if (chr_off[k] + chr_len[k] > l_pac) return fail(FA_ERR_ARG, "a reference sequence runs past l_pac");
        if (k && chr_off[k] < chr_off[k - 1]) return fail(FA_ERR_ARG, "reference offsets are not ascending");
    }
    for (uint32_t r = 0; r < n_reads; ++r)
        if (read_off[r + 1] < read_off[r] || read_off[r + 1] - read_off[r] > FA_MAX_QLEN)
            return fail(FA_ERR_ARG, "read %u: bad offsets or longer than FA_MAX_QLEN", r);
    for (uint32_t k = 0; k < n_cand; ++k) {
        const fa_rescue_cand &q = cands[k];
        if (q.read >= n_reads || (uint64_t)q.aln_first + q.aln_count > n_alns || q.primary >= n_alns)
            return fail(FA_ERR_ARG, "rescue attempt %u: index out of range", k);
        if (q.anchor.ref_id < 0 || (uint32_t)q.anchor.ref_id >= n_chr)
            return fail(FA_ERR_ARG, "rescue attempt %u: anchor reference out of range", k);
    }
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const uint64_t read_bytes = read_off[n_reads];
    const size_t b_pac = pac ? up16((size_t)((l_pac + 3) / 4)) : 0, b_chr = up16(8ull * n_chr);
    const size_t b_reads = up16(read_bytes + 1), b_off = up16(8ull * (n_reads + 1));
    const size_t b_alns = up16(sizeof(fa_rescue_aln) * n_alns), b_cands = up16(sizeof(fa_rescue_cand) * n_cand);
    FA_CUDA(c->mc_in.ensure(b_pac + 2 * b_chr + b_reads + b_off + b_alns + b_cands));
    char *in = c->mc_in.as<char>();
    size_t o = 0;
    auto take = [&](size_t b) { char *p = in + o; o += b; return p; };
    uint8_t *d_pac_in = reinterpret_cast<uint8_t *>(take(b_pac));
    const uint8_t *d_pac = pac ? d_pac_in : c->ref_pac.as<uint8_t>();
    uint64_t *d_coff = reinterpret_cast<uint64_t *>(take(b_chr));
    uint64_t *d_clen = reinterpret_cast<uint64_t *>(take(b_chr));
    uint8_t *d_reads = reinterpret_cast<uint8_t *>(take(b_reads));
    uint64_t *d_off = reinterpret_cast<uint64_t *>(take(b_off));
    fa_rescue_aln *d_alns = reinterpret_cast<fa_rescue_aln *>(take(b_alns));
    fa_rescue_cand *d_cands = reinterpret_cast<fa_rescue_cand *>(take(b_cands));
    if (pac) FA_CUDA(cudaMemcpyAsync(d_pac_in, pac, (size_t)((l_pac + 3) / 4), cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_coff, chr_off, 8ull * n_chr, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_clen, chr_len, 8ull * n_chr, cudaMemcpyHostToDevice, s));
    if (read_bytes) FA_CUDA(cudaMemcpyAsync(d_reads, reads, read_bytes, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_off, read_off, 8ull * (n_reads + 1), cudaMemcpyHostToDevice, s));
    if (n_alns) FA_CUDA(cudaMemcpyAsync(d_alns, alns, sizeof(fa_rescue_aln) * n_alns, cudaMemcpyHostToDevice, s));
    FA_CUDA(cudaMemcpyAsync(d_cands, cands, sizeof(fa_rescue_cand) * n_cand, cudaMemcpyHostToDevice, s));
    const size_t nb = collect_scan_blocks(n_cand);
    const size_t b_plan = up16(sizeof(CollectPlan) * n_cand);
    FA_CUDA(c->mc_plan.ensure(b_plan + sizeof(ulonglong4) * (nb + 1)));
    CollectPlan *d_plan = c->mc_plan.as<CollectPlan>();
    ulonglong4 *d_sums = reinterpret_cast<ulonglong4 *>(c->mc_plan.as<char>() + b_plan);
    const RescueRef ref{l_pac, d_pac, d_coff, d_clen, n_chr};
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    FA_CUDA(launch_mate_collect_plan(*opt, bounds4, ref, d_off, d_alns, d_cands, n_cand, d_plan, s));
    FA_CUDA(launch_plan_scan(d_plan, n_cand, d_sums, s));
    ulonglong4 tot;
    FA_CUDA(cudaMemcpyAsync(&tot, d_sums + nb, sizeof(tot), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    counts->n_left = (uint32_t)tot.y;
    counts->qbuf_len = tot.z;
    counts->tbuf_len = tot.x;
    if (tot.x > tbuf_cap || tot.z > qbuf_cap)
        return fail(FA_ERR_CAPACITY, "qbuf_cap or tbuf_cap below the jobs' bytes (counts->qbuf_len, tbuf_len)");
    if ((tot.z && !qbuf) || (tot.x && !tbuf)) return fail(FA_ERR_ARG, "null sequence buffer");
    const size_t b_jobs = up16(sizeof(fa_mate_job) * tot.y), b_info = up16(sizeof(fa_rescue_job_info) * tot.y);
    const size_t b_q = up16(tot.z + 1), b_t = up16(tot.x + 1);
    FA_CUDA(c->mc_out.ensure(b_jobs + b_info + b_q + b_t));
    char *out = c->mc_out.as<char>();
    fa_mate_job *d_jobs = reinterpret_cast<fa_mate_job *>(out);
    fa_rescue_job_info *d_info = reinterpret_cast<fa_rescue_job_info *>(out + b_jobs);
    uint8_t *d_q = reinterpret_cast<uint8_t *>(out + b_jobs + b_info);
    uint8_t *d_t = reinterpret_cast<uint8_t *>(out + b_jobs + b_info + b_q);
    FA_CUDA(launch_mate_collect_fill(*opt, bounds4, ref, d_reads, d_off, d_alns, d_cands, n_cand, d_plan, d_jobs,
                                     d_info, d_q, d_t, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = 5;
    c->last_stream = s;
    if (tot.y) {
        FA_CUDA(cudaMemcpyAsync(jobs, d_jobs, sizeof(fa_mate_job) * tot.y, cudaMemcpyDeviceToHost, s));
        FA_CUDA(cudaMemcpyAsync(info, d_info, sizeof(fa_rescue_job_info) * tot.y, cudaMemcpyDeviceToHost, s));
    }
    if (tot.z) FA_CUDA(cudaMemcpyAsync(qbuf, d_q, tot.z, cudaMemcpyDeviceToHost, s));
    if (tot.x) FA_CUDA(cudaMemcpyAsync(tbuf, d_t, tot.x, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

int fa_insert_size_stats(fa_ctx *c, uint64_t l_pac, const int64_t *pairs, uint32_t n, fa_insert_stats *out4) {
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (!out4 || (n && !pairs)) return fail(FA_ERR_ARG, "null buffer");
    if (l_pac == 0 || l_pac > (1ull << 62)) return fail(FA_ERR_ARG, "l_pac out of range");
    FA_CUDA(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t b_pairs = up16(16ull * n), b_hist = up16(insert_hist_bytes());
    FA_CUDA(c->is_buf.ensure(b_pairs + b_hist + sizeof(fa_insert_stats) * 4));
    char *b = c->is_buf.as<char>();
    int64_t *d_pairs = reinterpret_cast<int64_t *>(b);
    uint32_t *d_hist = reinterpret_cast<uint32_t *>(b + b_pairs);
    fa_insert_stats *d_out = reinterpret_cast<fa_insert_stats *>(b + b_pairs + b_hist);
    if (n) FA_CUDA(cudaMemcpyAsync(d_pairs, pairs, 16ull * n, cudaMemcpyHostToDevice, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev0, s));
    FA_CUDA(launch_insert_stats((int64_t)l_pac, d_pairs, n, d_hist, d_out, s));
    if (c->timing) FA_CUDA(cudaEventRecord(c->kev1, s));
    c->last_launches = n ? 2 : 1;
    c->last_stream = s;
    FA_CUDA(cudaMemcpyAsync(out4, d_out, sizeof(fa_insert_stats) * 4, cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    return FA_OK;
}

int fa_ctx_last_cells(fa_ctx *c, unsigned long long *cells) {
    if (!c || !cells) return fail(FA_ERR_ARG, "null argument");
    *cells = 0;
    if (!c->misc.p) return FA_OK;
    FA_CUDA(cudaMemcpy(cells, misc_of(c).cells, 8, cudaMemcpyDeviceToHost));
    return FA_OK;
}

int fa_pair_batch(fa_ctx *c, const fa_params *p, const fa_policy *pol, const fa_band_model *model, float margin,
                  const fa_job *jobs, uint32_t n, const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq,
                  uint64_t tseq_len, const fa_band_hint *hints, fa_ext_result *out, const fa_mate_params *mp,
                  const fa_mate_job *mjobs, uint32_t mn, const uint8_t *mqseq, uint64_t mqseq_len,
                  const uint8_t *mtseq, uint64_t mtseq_len, fa_kswr *mout, fa_ext_stats *stats,
                  fa_ext_stats *mate_stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (mate_stats) memset(mate_stats, 0, sizeof(*mate_stats));
    if (!c) return fail(FA_ERR_ARG, "null context");
    if (model && (!pol || pol->mode != FA_POLICY_LEARNED))
        return fail(FA_ERR_ARG, "a band model needs FA_POLICY_LEARNED");
    if (!model && pol && pol->mode == FA_POLICY_LEARNED)
        return fail(FA_ERR_STATE, "FA_POLICY_LEARNED needs a band model");
    if (int rc = check_host_call(c, p, pol, jobs, n, out)) return rc;
    if (n && (!qseq || !tseq)) return fail(FA_ERR_ARG, "null buffer");
    if (!mp || mp->m != 5) return fail(FA_ERR_ARG, "mate alphabet size must be 5");
    if (mn && (!mjobs || !mout || !mqseq || !mtseq)) return fail(FA_ERR_ARG, "null mate buffer");
    // a large mate half runs in job-index slices whose uploads overlap its kernels
    const bool msliced = mn >= kPipeMinJobs && c->slices_single != 1;
    MateHostPlan pl;
    if (mn && !msliced)
        if (int rc = plan_mate_host(mp, mjobs, mn, mqseq_len, mtseq_len, &pl)) return rc;
    FA_CUDA(cudaSetDevice(c->device));
    // the mate half, asynchronous on its own stream: uploads, kernels, results back
    if (!c->pm_stream) {
        FA_CUDA(cudaStreamCreateWithFlags(&c->pm_stream, cudaStreamNonBlocking));
        FA_CUDA(cudaStreamCreateWithFlags(&c->pm_copy, cudaStreamNonBlocking));
        FA_CUDA(cudaEventCreate(&c->pm_ev0));
        FA_CUDA(cudaEventCreate(&c->pm_ev1));
        FA_CUDA(cudaEventCreateWithFlags(&c->pm_fork, cudaEventDisableTiming));
        for (auto &e : c->pm_slice_ev) FA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t ms = c->pm_stream;
    uint32_t mlaunches = 0;
    if (mn && msliced) {
        FA_CUDA(c->pm_jobs.ensure(sizeof(fa_mate_job) * (size_t)mn));
        FA_CUDA(c->pm_order.ensure(4ull * mn));
        FA_CUDA(c->pm_q.ensure(mqseq_len + 1));
        FA_CUDA(c->pm_t.ensure(mtseq_len + 1));
        FA_CUDA(c->pm_out.ensure(sizeof(fa_kswr) * (size_t)mn));
        FA_CUDA(c->pm_misc.ensure(64));
        FA_CUDA(c->pm_rev.ensure(4ull * (2 + (size_t)mate_max_slice(mn))));
        if (int rc = ensure_host_stage(c, 4ull * mn)) return rc;
        FA_CUDA(cudaMemsetAsync(c->pm_misc.p, 0, 64, ms));
        FA_CUDA(cudaEventRecord(c->pm_fork, ms));
        FA_CUDA(cudaStreamWaitEvent(c->pm_copy, c->pm_fork, 0));
        const MateSliceRes r{ms, c->pm_copy, nullptr, c->pm_slice_ev, nullptr, c->pm_ev0, c->pm_jobs.as<fa_mate_job>(),
                             c->pm_order.as<uint32_t>(), c->pm_q.as<uint8_t>(), c->pm_t.as<uint8_t>(),
                             c->pm_out.as<fa_kswr>(),
                             reinterpret_cast<unsigned long long *>(c->pm_misc.as<char>() + 8),
                             c->pm_misc.as<uint32_t>(), c->pm_rev.as<uint32_t>()};
        const MateBytesUp up{mqseq, mtseq, c->pm_q.as<uint8_t>(), c->pm_t.as<uint8_t>()};
        if (int rc = enqueue_mate_sliced(mp, mjobs, mn, mqseq_len, mtseq_len, up, static_cast<uint32_t *>(c->h_stage),
                                         nullptr, r, &mlaunches)) {
            cudaStreamSynchronize(c->pm_copy);
            cudaStreamSynchronize(ms);
            return rc;
        }
        FA_CUDA(cudaEventRecord(c->pm_ev1, ms));
        FA_CUDA(cudaMemcpyAsync(mout, c->pm_out.p, sizeof(fa_kswr) * (size_t)mn, cudaMemcpyDeviceToHost, ms));
    } else if (mn) {
        FA_CUDA(c->pm_jobs.ensure(sizeof(fa_mate_job) * (size_t)mn));
        FA_CUDA(c->pm_order.ensure(4ull * mn));
        FA_CUDA(c->pm_q.ensure(mqseq_len));
        FA_CUDA(c->pm_t.ensure(mtseq_len));
        FA_CUDA(c->pm_out.ensure(sizeof(fa_kswr) * (size_t)mn));
        FA_CUDA(c->pm_misc.ensure(64));
        FA_CUDA(c->pm_rev.ensure(4ull * (2 + (size_t)pl.n_byte)));
        FA_CUDA(cudaMemsetAsync(c->pm_misc.p, 0, 64, ms));
        FA_CUDA(cudaMemcpyAsync(c->pm_jobs.p, mjobs, sizeof(fa_mate_job) * (size_t)mn, cudaMemcpyHostToDevice, ms));
        FA_CUDA(cudaMemcpyAsync(c->pm_order.p, pl.order.data(), 4ull * mn, cudaMemcpyHostToDevice, ms));
        FA_CUDA(cudaMemcpyAsync(c->pm_q.p, mqseq, mqseq_len, cudaMemcpyHostToDevice, ms));
        FA_CUDA(cudaMemcpyAsync(c->pm_t.p, mtseq, mtseq_len, cudaMemcpyHostToDevice, ms));
        FA_CUDA(cudaEventRecord(c->pm_ev0, ms));
        uint32_t *st = c->pm_misc.as<uint32_t>();
        unsigned long long *cells = reinterpret_cast<unsigned long long *>(c->pm_misc.as<char>() + 8);
        FA_CUDA(launch_mate_plan(pl, c->pm_jobs.as<fa_mate_job>(), c->pm_order.as<uint32_t>(), mn,
                                 c->pm_q.as<uint8_t>(), c->pm_t.as<uint8_t>(), c->pm_out.as<fa_kswr>(), cells, st,
                                 c->pm_rev.as<uint32_t>(), ms, &mlaunches));
        FA_CUDA(cudaEventRecord(c->pm_ev1, ms));
        FA_CUDA(cudaMemcpyAsync(mout, c->pm_out.p, sizeof(fa_kswr) * (size_t)mn, cudaMemcpyDeviceToHost, ms));
    }
    // the extension half on the main stream, meanwhile
    int rc = FA_OK;
    if (n) {
        rc = model ? ext_learned_host(c, p, pol, model, margin, jobs, n, host_bytes(qseq, qseq_len),
                                      host_bytes(tseq, tseq_len), hints, out, nullptr, nullptr, stats)
                   : ext_batch_host(c, p, pol, jobs, n, host_bytes(qseq, qseq_len), host_bytes(tseq, tseq_len),
                                    nullptr, out, nullptr, stats);
    }
    // the mate half's end (also on an extension error, so the caller's buffers are free)
    const cudaError_t es = cudaStreamSynchronize(ms);
    if (msliced) cudaStreamSynchronize(c->pm_copy);
    if (rc) return rc;
    FA_CUDA(es);
    if (mn) {
        uint32_t h[4];
        FA_CUDA(cudaMemcpy(h, c->pm_misc.p, 16, cudaMemcpyDeviceToHost));
        if (h[0] & ST_BAD_CODE) return fail(FA_ERR_ARG, "a mate sequence byte is outside the alphabet (codes 0-4)");
        if (h[0] & ST_BLIST) return fail(FA_ERR_CAPACITY, "mate-SW run list overflow");
        if (h[0]) return fail(FA_ERR_ARG, "a mate job was rejected by the kernels");
        if (mate_stats) {
            float k_ms = 0.f;
            cudaEventElapsedTime(&k_ms, c->pm_ev0, c->pm_ev1);
            unsigned long long cells = (unsigned long long)h[2] | (unsigned long long)h[3] << 32;
            mate_stats->cells = mate_stats->cells_executed = cells;
            mate_stats->kernel_ms = k_ms;
            mate_stats->kernel_launches = mlaunches;
            mate_stats->jobs = mn;
        }
    }
    const float total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) stats->total_ms = total;
    if (mate_stats) mate_stats->total_ms = total;
    return FA_OK;
}

int fa_mate_sw_batch(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                     const uint8_t *qseq, uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len,
                     fa_kswr *out, fa_ext_stats *stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n && (!qseq || !tseq)) return fail(FA_ERR_ARG, "null buffer");
    if (mate_sliceable(c, p, jobs, n, out))
        return mate_host_sliced(c, p, jobs, n, qseq_len, tseq_len,
                                [&](uint8_t *dq, uint8_t *dt, int *) { return MateBytesUp{qseq, tseq, dq, dt}; }, out,
                                stats, t0);
    auto upload = [&](cudaStream_t s) -> int {
        FA_CUDA(c->qseq.ensure(qseq_len));
        FA_CUDA(c->tseq.ensure(tseq_len));
        FA_CUDA(cudaMemcpyAsync(c->qseq.p, qseq, qseq_len, cudaMemcpyHostToDevice, s));
        FA_CUDA(cudaMemcpyAsync(c->tseq.p, tseq, tseq_len, cudaMemcpyHostToDevice, s));
        return FA_OK;
    };
    return mate_host_batch(c, p, jobs, n, qseq_len, tseq_len, upload, out, stats, t0);
}

int fa_mate_sw_batch_packed(fa_ctx *c, const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                            const fa_packed_seq *qseq, const fa_packed_seq *tseq, fa_kswr *out, fa_ext_stats *stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n == 0) return c ? FA_OK : fail(FA_ERR_ARG, "null context");
    HostSeq hq, ht;
    if (int rc = host_packed(qseq, "query", &hq)) return rc;
    if (int rc = host_packed(tseq, "target", &ht)) return rc;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    if (mate_sliceable(c, p, jobs, n, out)) {
        auto make_up = [&](uint8_t *dq, uint8_t *dt, int *rc) {
            const size_t bq = up16(hq.nbytes) + 16, bt = up16(ht.nbytes) + 16;
            const size_t brq = up16(sizeof(fa_nrun) * hq.n_runs), brt = up16(sizeof(fa_nrun) * ht.n_runs);
            MatePackedUp up{hq, ht, nullptr, nullptr, dq, dt, nullptr, nullptr, misc_of(c).status};
            const cudaError_t e = c->mate_pk.ensure(bq + bt + brq + brt);
            if (e != cudaSuccess) {
                *rc = fail(FA_ERR_CUDA, "%s", cudaGetErrorString(e));
                return up;
            }
            char *k = c->mate_pk.as<char>();
            up.pq = reinterpret_cast<uint8_t *>(k);
            up.pt = reinterpret_cast<uint8_t *>(k + bq);
            up.rq = reinterpret_cast<fa_nrun *>(k + bq + bt);
            up.rt = reinterpret_cast<fa_nrun *>(k + bq + bt + brq);
            return up;
        };
        return mate_host_sliced(c, p, jobs, n, hq.npos, ht.npos, make_up, out, stats, t0);
    }
    // the packed bases and N runs go up, and the device unpacks them to byte codes for the
    // SW kernels (which read each base many times, from cache); the runs are checked there
    auto upload = [&](cudaStream_t s) -> int {
        FA_CUDA(c->qseq.ensure(up16(hq.npos) + 16));
        FA_CUDA(c->tseq.ensure(up16(ht.npos) + 16));
        const size_t bq = up16(hq.nbytes) + 16, bt = up16(ht.nbytes) + 16;
        const size_t brq = up16(sizeof(fa_nrun) * hq.n_runs), brt = up16(sizeof(fa_nrun) * ht.n_runs);
        FA_CUDA(c->mate_pk.ensure(bq + bt + brq + brt));
        char *k = c->mate_pk.as<char>();
        uint8_t *pq = reinterpret_cast<uint8_t *>(k), *pt = reinterpret_cast<uint8_t *>(k + bq);
        fa_nrun *rq = reinterpret_cast<fa_nrun *>(k + bq + bt), *rt = reinterpret_cast<fa_nrun *>(k + bq + bt + brq);
        FA_CUDA(cudaMemcpyAsync(pq, hq.p, hq.nbytes, cudaMemcpyHostToDevice, s));
        FA_CUDA(cudaMemcpyAsync(pt, ht.p, ht.nbytes, cudaMemcpyHostToDevice, s));
        if (hq.n_runs) FA_CUDA(cudaMemcpyAsync(rq, hq.runs, sizeof(fa_nrun) * hq.n_runs, cudaMemcpyHostToDevice, s));
        if (ht.n_runs) FA_CUDA(cudaMemcpyAsync(rt, ht.runs, sizeof(fa_nrun) * ht.n_runs, cudaMemcpyHostToDevice, s));
        Misc m = misc_of(c);
        FA_CUDA(launch_runs_check(rq, (uint32_t)hq.n_runs, hq.npos, m.status, s));
        FA_CUDA(launch_runs_check(rt, (uint32_t)ht.n_runs, ht.npos, m.status, s));
        FA_CUDA(launch_unpack2(pq, hq.npos, rq, (uint32_t)hq.n_runs, c->qseq.as<uint8_t>(), s));
        FA_CUDA(launch_unpack2(pt, ht.npos, rt, (uint32_t)ht.n_runs, c->tseq.as<uint8_t>(), s));
        return FA_OK;
    };
    return mate_host_batch(c, p, jobs, n, hq.npos, ht.npos, upload, out, stats, t0);
}

}  // extern "C"
