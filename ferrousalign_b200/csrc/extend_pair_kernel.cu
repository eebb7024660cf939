// extend_pair_kernel.cu -- ksw_extend2 with int16x2 cells: two extensions per thread.
//
// Same recurrence as ext_packed_kernel (ksw_affine_gap.rs:952-1169), but every thread
// runs two length-adjacent jobs in the two 16-bit halves of its registers (job A low,
// job B high), so each Blackwell DPX instruction updates two cells:
//   score pair   one PRMT on an 8-byte table indexed by (query code XOR target code),
//                valid for bwa-form matrices (a on the diagonal, -b off it, N = -1 or 0)
//   M' pair      __viaddmin_s16x2(M, s, k*M): equals M ? M + s : 0 up to values <= 0,
//                which the following max/relu steps treat exactly like 0
//   H pair       __vimax3_s16x2(M', E, F)
//   E, F pairs   __viaddmax_s16x2_relu
//   row max      max.s16x2 with per-half predicated argmax updates (first column of
//                the row maximum)
// Column state: one 8-byte shared-memory word per column (H pair, E pair) and one
// 16-bit PRMT selector pair of the query codes, interleaved with stride blockDim.x.
//
// The two jobs have different adaptive bands.  Each row is swept over the union of the
// two column ranges in at most three segments; in a segment each half is either in its
// job's range, to the left of it (its results there are never read again and are
// discarded: its F/H/max chains restart where its range begins), or to the right of it
// (frozen: a store mask keeps that half's previous contents, which later rows read as
// the reference's stale band-edge cells).  All segments share one loop body.  Exact while h0 + a*qlen < 8192 and a <= 3.

#include <vector>

#include "fa_device.cuh"
#include "fa_kernels.h"
#include "fa_packed.cuh"

namespace fa {

// PRMT in its generic mode; the host branch restates the documented byte-select
// semantics so the kernel body can also run on the CPU (tests).
__host__ __device__ __forceinline__ uint32_t prmt32(uint32_t lo, uint32_t hi, uint32_t sel) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return r;
#else
    const uint64_t src = (uint64_t)hi << 32 | lo;
    uint32_t r = 0;
    for (int k = 0; k < 4; ++k) {
        const uint32_t nib = (sel >> (4 * k)) & 0xFu;
        uint32_t byte = (uint32_t)(src >> (8 * (nib & 7u))) & 0xFFu;
        if (nib & 8u) byte = (byte & 0x80u) ? 0xFFu : 0x00u;
        r |= byte << (8 * k);
    }
    return r;
#endif
}

// Per-half signed running maximum m = max(m, h); a half whose maximum strictly grows
// takes column j as its argmax, so ties keep the first column (ksw_affine_gap.rs:1060-1063).
// Written out instead of __vibmax_s16x2: that intrinsic's inline assembly reads its
// input after writing its output without an early-clobber constraint, and when both
// are given one register its "kept" predicates come out always true.
__host__ __device__ __forceinline__ void max_argmax_s16x2(uint32_t &m, uint32_t h, int j, int &mjA, int &mjB) {
#ifdef __CUDA_ARCH__
    uint32_t mn;
    asm("{\n\t.reg .pred plo, phi;\n\t.reg .s16 n0, n1, o0, o1;\n\t"
        "max.s16x2 %0, %3, %4;\n\t"
        "mov.b32 {n0, n1}, %0;\n\t"
        "mov.b32 {o0, o1}, %3;\n\t"
        "setp.ne.s16 plo, n0, o0;\n\t"
        "setp.ne.s16 phi, n1, o1;\n\t"
        "@plo mov.b32 %1, %5;\n\t"
        "@phi mov.b32 %2, %5;\n\t}"
        : "=&r"(mn), "+r"(mjA), "+r"(mjB)
        : "r"(m), "r"(h), "r"(j));
    m = mn;
#else
    const int16_t m0 = (int16_t)(m & 0xffffu), m1 = (int16_t)(m >> 16);
    const int16_t h0 = (int16_t)(h & 0xffffu), h1 = (int16_t)(h >> 16);
    if (h0 > m0) mjA = j;
    if (h1 > m1) mjB = j;
    m = (uint32_t)(uint16_t)(h0 > m0 ? h0 : m0) | (uint32_t)(uint16_t)(h1 > m1 ? h1 : m1) << 16;
#endif
}

__host__ __device__ __forceinline__ void status_or(uint32_t *st, uint32_t v) {
#ifdef __CUDA_ARCH__
    atomicOr(st, v);
#else
    *st |= v;
#endif
}

struct PairConsts {
    uint32_t tab_lo, tab_hi;          // score table [a, -b, -b, -b, n, n, n, n]
    uint32_t neg_oedel2, neg_edel2;   // -(o_del+e_del), -e_del in both halves
    uint32_t neg_oeins2, neg_eins2;
    uint32_t kmul;                    // 2 or 4: k*M >= M + a for every M >= 1
};

// One segment [j0, j1) of a row.  `live` selects the halves whose stores take the new
// values; the other half (a job whose range ended left of j0) keeps its previous
// contents.  Every segment runs this same loop body, so threads of a warp that sit in
// different kinds of segment do not diverge.
template <bool SYM, int T>
__host__ __device__ __forceinline__ void pair_segment(uint2 *__restrict__ col, const uint16_t *__restrict__ qs,
                                                      int j0, int j1, uint32_t tsel, const PairConsts &k,
                                                      uint32_t live, uint32_t &f, uint32_t &h1, uint32_t &m,
                                                      int &mjA, int &mjB)
{
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
        const uint2 w = col[j * T];
        const uint32_t sel = (uint32_t)qs[j * T] ^ tsel;
        const uint32_t s = prmt32(k.tab_lo, k.tab_hi, sel);
        const uint32_t M = w.x;
        const uint32_t Mp = __viaddmin_s16x2(M, s, M * k.kmul);
        const uint32_t e = w.y;
        const uint32_t h = __vimax3_s16x2(Mp, e, f);
        const uint32_t tdel = __viaddmax_s16x2(Mp, k.neg_oedel2, 0x80008000u);
        const uint32_t enew = __viaddmax_s16x2_relu(e, k.neg_edel2, tdel);
        if (SYM) {
            f = __viaddmax_s16x2_relu(f, k.neg_eins2, tdel);
        } else {
            const uint32_t tins = __viaddmax_s16x2(Mp, k.neg_oeins2, 0x80008000u);
            f = __viaddmax_s16x2_relu(f, k.neg_eins2, tins);
        }
        max_argmax_s16x2(m, h, j, mjA, mjB);
        uint2 o;
        o.x = (h1 & live) | (w.x & ~live);
        o.y = (enew & live) | (w.y & ~live);
        col[j * T] = o;
        h1 = h;
    }
}

__host__ __device__ __forceinline__ uint32_t set_lo(uint32_t x, uint32_t v) { return (x & 0xffff0000u) | (v & 0xffffu); }
__host__ __device__ __forceinline__ uint32_t set_hi(uint32_t x, uint32_t v) { return (x & 0xffffu) | (v << 16); }
__host__ __device__ __forceinline__ int get_half(uint32_t x, int hi) { return hi ? (int)(x >> 16) : (int)(x & 0xffffu); }

struct JobState {
    const uint8_t *T;
    int qlen, tlen, h0, w;
    int beg, end;                  // adaptive range of the next row
    int best, max_i, max_j, max_ie, gscore, max_off;
    int live;                      // still extending
    int clamped;
    uint32_t cells;
    uint32_t jid;
};

// The work of one thread: jobs order[2*pair] and order[2*pair+1].  col/qs point at the
// thread's first column word; consecutive columns are T words apart (a compile-time
// stride, so the compiler can overlap a column's loads with the previous column's
// stores).  Returns the cells
// of both jobs.  Host-callable so the CPU tests can run this exact code.
template <bool SYM, int T>
__host__ __device__ __forceinline__ unsigned long long ext_pair_thread(
    uint32_t pair, uint2 *__restrict__ col, uint16_t *__restrict__ qs, const fa_job *__restrict__ jobs,
    const uint32_t *__restrict__ order, uint32_t n, const uint8_t *__restrict__ qseq,
    const uint8_t *__restrict__ tseq, const ExtParams &p, const PairConsts &kc, int n_code_t, int qcap,
    const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out, uint8_t *__restrict__ clamped_out,
    uint32_t *__restrict__ cells_job, uint32_t *__restrict__ status)
{
    const uint32_t ia = 2 * pair, ib = 2 * pair + 1;
    unsigned long long cells_total = 0;

    if (ia < n) {
        JobState J[2];
        uint32_t bad = 0;
#pragma unroll
        for (int x = 0; x < 2; ++x) {
            JobState &s = J[x];
            const uint32_t gi = x ? ib : ia;
            s.live = gi < n;
            s.jid = s.live ? (order ? order[gi] : gi) : 0;
            fa_job jb;
            if (s.live) jb = jobs[s.jid];
            else { jb.qlen = 1; jb.tlen = 0; jb.h0 = 1; jb.w = 0; jb.q_off = jb.t_off = 0; }
            s.qlen = jb.qlen; s.tlen = jb.tlen; s.h0 = jb.h0;
            s.T = tseq + jb.t_off;
            s.cells = 0; s.clamped = 0;
            s.best = jb.h0; s.max_i = s.max_j = s.max_ie = -1; s.gscore = -1; s.max_off = 0;
            s.beg = 0; s.end = jb.qlen;
            if (s.live && (jb.h0 < 0 || (jb.h0 == 0 && !(p.flags & FA_PARAM_H0_ZERO)) || jb.qlen <= 0 || jb.tlen < 0)) {
                status_or(status, ST_ARG);
                s.live = 0;
            } else if (s.live && jb.h0 == 0) {
                // FA_PARAM_H0_ZERO: the recurrence as written is all zero after row 0; the job's
                // final state is set here and written out with the others at the end
                const int w0 = ext_band_clamp(jb.qlen, w_try ? w_try[s.jid] : jb.w, p);
                fa_ext_result r;
                s.cells = ext_h0_zero_result(jb.qlen, jb.tlen, w0, &r);
                s.best = r.score; s.max_j = r.qle - 1; s.max_i = r.tle - 1; s.max_ie = r.gtle - 1;
                s.gscore = r.gscore; s.max_off = r.max_off;
                s.clamped = jb.tlen > 0 && jb.qlen > w0 + 1 ? 1 : 0;
                s.live = 0;
            }
            else if (s.live && (jb.qlen > qcap || jb.h0 + p.max_score * jb.qlen > kPackedHMax)) {
                status_or(status, ST_CAPACITY); s.live = 0;
            }
            s.w = s.live ? ext_band_clamp(s.qlen, w_try ? w_try[s.jid] : jb.w, p) : 0;
        }
        const int e_ins = p.e_ins, oe_ins = p.o_ins + p.e_ins;
        // query selectors and the first row of both jobs
        const uint8_t *QA = qseq + (J[0].live ? jobs[J[0].jid].q_off : 0);
        const uint8_t *QB = qseq + (J[1].live ? jobs[J[1].jid].q_off : 0);
        const int qmax = max(J[0].live ? J[0].qlen : 0, J[1].live ? J[1].qlen : 0);
        int hpA = J[0].h0, hpB = J[1].h0;
        bool fillA = true, fillB = true;
        for (int j = 0; j <= qmax; ++j) {
            uint32_t sel = 0;
            int hA = 0, hB = 0;
            if (J[0].live && j <= J[0].qlen) {
                if (j < J[0].qlen) {
                    const uint32_t c = QA[j];
                    bad |= c > 4u;
                    sel |= c >= 4u ? 0x4Cu : c * 0x11u;
                }
                if (j == 0) hA = J[0].h0;
                else if (j == 1) hA = J[0].h0 > oe_ins ? J[0].h0 - oe_ins : 0;
                else if (fillA && hpA > e_ins) hA = hpA - e_ins;
                else { fillA = false; hA = 0; }
                hpA = hA;
            }
            if (J[1].live && j <= J[1].qlen) {
                if (j < J[1].qlen) {
                    const uint32_t c = QB[j];
                    bad |= c > 4u;
                    sel |= (c >= 4u ? 0x4Cu : c * 0x11u) << 8;
                }
                if (j == 0) hB = J[1].h0;
                else if (j == 1) hB = J[1].h0 > oe_ins ? J[1].h0 - oe_ins : 0;
                else if (fillB && hpB > e_ins) hB = hpB - e_ins;
                else { fillB = false; hB = 0; }
                hpB = hB;
            }
            qs[j * T] = (uint16_t)sel;
            col[j * T] = make_uint2((uint32_t)hA | (uint32_t)hB << 16, 0u);
        }

        const int tmax = max(J[0].live ? J[0].tlen : 0, J[1].live ? J[1].tlen : 0);
        for (int i = 0; i < tmax && (J[0].live | J[1].live); ++i) {
            // per-job row setup: band clamp, first column, target selector nibbles
            int b[2], e[2], h1i[2];
            uint32_t tsel = 0;
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                JobState &s = J[x];
                if (s.live && i >= s.tlen) s.live = 0;
                if (!s.live) { b[x] = e[x] = 0; h1i[x] = 0; continue; }
                uint32_t tb = s.T[i];
                if (tb > 4u) { bad = 1; tb = 4; }
                const uint32_t tc = tb >= 4u ? (uint32_t)n_code_t : tb;
                tsel |= (tc | (tc | 8u) << 4) << (8 * x);
                const int beg_a = s.beg, end_a = s.end < s.qlen ? s.end : s.qlen;
                if (s.beg < i - s.w) s.beg = i - s.w;
                if (s.end > i + s.w + 1) s.end = i + s.w + 1;
                if (s.end > s.qlen) s.end = s.qlen;
                s.clamped |= (s.beg != beg_a) | (s.end != end_a);
                b[x] = s.beg;
                e[x] = s.end;
                int h1 = 0;
                if (s.beg == 0) {
                    h1 = s.h0 - (p.o_del + p.e_del * (i + 1));
                    if (h1 < 0) h1 = 0;
                }
                h1i[x] = h1;
            }
            // an empty or finished range never constrains the sweep
            const bool actA = J[0].live && e[0] > b[0], actB = J[1].live && e[1] > b[1];
            uint32_t f = 0, h1 = (uint32_t)h1i[0] | (uint32_t)h1i[1] << 16, m = 0;
            int mjA = -1, mjB = -1;
            int hEndA = h1i[0], hEndB = h1i[1];     // h1 at each job's end column
            uint32_t mSave = 0;
            int mjSaveA = -1, mjSaveB = -1;
            if (actA || actB) {
                // boundaries: ranges [b0,e0) and [b1,e1); left of a range = discard, right = frozen
                const int lo = actA && actB ? min(b[0], b[1]) : (actA ? b[0] : b[1]);
                const int hi = actA && actB ? max(e[0], e[1]) : (actA ? e[0] : e[1]);
                // sorted unique cut points: lo, interior range boundaries, then hi
                int cut[6];
                int nc = 0;
                cut[nc++] = lo;
                const int pts[4] = {actA ? b[0] : lo, actB ? b[1] : lo, actA ? e[0] : hi, actB ? e[1] : hi};
                for (int t = 0; t < 4; ++t) {
                    const int v = pts[t];
                    if (v <= lo || v >= hi) continue;
                    bool dup = false;
                    for (int r = 0; r < nc; ++r) dup |= cut[r] == v;
                    if (dup) continue;
                    int u = nc;
                    while (u > 0 && cut[u - 1] > v) { cut[u] = cut[u - 1]; --u; }
                    cut[u] = v;
                    ++nc;
                }
                cut[nc] = hi;
                for (int sg = 0; sg < nc; ++sg) {
                    const int j0 = cut[sg], j1 = cut[sg + 1];
                    if (j1 <= j0) continue;
                    // a half whose range begins here restarts its F, H and max chains
                    if (actA && j0 == b[0]) { f &= 0xffff0000u; h1 = set_lo(h1, h1i[0]); m &= 0xffff0000u; mjA = -1; }
                    if (actB && j0 == b[1]) { f &= 0xffffu; h1 = set_hi(h1, h1i[1]); m &= 0xffffu; mjB = -1; }
                    // a half whose range ended keeps its h1 / max for the end-of-row bookkeeping
                    const bool frzA = actA ? j0 >= e[0] : false;
                    const bool frzB = actB ? j0 >= e[1] : false;
                    if (actA && j0 == e[0]) { hEndA = (int)(h1 & 0xffffu); mSave = set_lo(mSave, m); mjSaveA = mjA; }
                    if (actB && j0 == e[1]) { hEndB = (int)(h1 >> 16); mSave = set_hi(mSave, m >> 16); mjSaveB = mjB; }
                    const uint32_t live = (frzA ? 0u : 0x0000ffffu) | (frzB ? 0u : 0xffff0000u);
                    pair_segment<SYM, T>(col, qs, j0, j1, tsel, kc, live, f, h1, m, mjA, mjB);
                }
                if (actA && e[0] == hi) { hEndA = (int)(h1 & 0xffffu); mSave = set_lo(mSave, m); mjSaveA = mjA; }
                if (actB && e[1] == hi) { hEndB = (int)(h1 >> 16); mSave = set_hi(mSave, m >> 16); mjSaveB = mjB; }
            }
            // eh[end] = {h1, 0} for each job (after every segment wrote its words)
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                JobState &s = J[x];
                if (!s.live) continue;
                const int hEnd = x ? hEndB : hEndA;
                uint2 wd = col[s.end * T];
                if (x) { wd.x = set_hi(wd.x, (uint32_t)hEnd); wd.y &= 0xffffu; }
                else { wd.x = set_lo(wd.x, (uint32_t)hEnd); wd.y &= 0xffff0000u; }
                col[s.end * T] = wd;
            }
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                JobState &s = J[x];
                if (!s.live) continue;
                const bool act = x ? actB : actA;
                const int hEnd = x ? hEndB : hEndA;
                int m_row = act ? get_half(mSave, x) : 0;
                const int mj = x ? mjSaveB : mjSaveA;
                if (s.end > s.beg) s.cells += s.end - s.beg;
                if (s.end == s.qlen && s.gscore < hEnd) { s.gscore = hEnd; s.max_ie = i; }
                if (m_row == 0) { s.live = 0; continue; }
                if (m_row > s.best) {
                    s.best = m_row; s.max_i = i; s.max_j = mj;
                    const int off = mj > i ? mj - i : i - mj;
                    if (s.max_off < off) s.max_off = off;
                } else if (p.zdrop > 0) {
                    const int di = i - s.max_i, dj = mj - s.max_j;
                    if (di > dj) {
                        if (s.best - m_row - (di - dj) * p.e_del > p.zdrop) { s.live = 0; continue; }
                    } else if (s.best - m_row - (dj - di) * p.e_ins > p.zdrop) {
                        s.live = 0; continue;
                    }
                }
                // adaptive band for the next row: zero test on this job's half
                int nb = s.beg;
                while (nb < s.end) {
                    const uint2 wd = col[nb * T];
                    if (get_half(wd.x, x) | get_half(wd.y, x)) break;
                    ++nb;
                }
                s.beg = nb;
                int ne = s.end;
                while (ne > s.beg) {
                    const uint2 wd = col[ne * T];
                    if (get_half(wd.x, x) | get_half(wd.y, x)) break;
                    --ne;
                }
                s.end = ne + 2 < s.qlen ? ne + 2 : s.qlen;
            }
        }
        if (bad) status_or(status, ST_BAD_CODE);
#pragma unroll
        for (int x = 0; x < 2; ++x) {
            JobState &s = J[x];
            const uint32_t gi = x ? ib : ia;
            if (gi >= n) continue;
            fa_ext_result r;
            r.score = s.best; r.qle = s.max_j + 1; r.tle = s.max_i + 1; r.gtle = s.max_ie + 1;
            r.gscore = s.gscore; r.max_off = s.max_off;
            out[s.jid] = r;
            if (clamped_out) clamped_out[s.jid] = (uint8_t)s.clamped;
            if (cells_job) cells_job[s.jid] = s.cells;
            cells_total += s.cells;
        }
    }
    return cells_total;
}

template <bool SYM>
__global__ void __launch_bounds__(kPairThreads)
ext_pair_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ order, uint32_t n,
                const uint32_t *__restrict__ n_dev, const uint8_t *__restrict__ qseq,
                const uint8_t *__restrict__ tseq, const ExtParams p, PairConsts kc, int n_code_t, int qcap,
                const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out,
                uint8_t *__restrict__ clamped_out, uint32_t *__restrict__ cells_job,
                unsigned long long *__restrict__ cells_out, uint32_t *__restrict__ status)
{
    extern __shared__ __align__(16) unsigned char psmem[];
    constexpr int T = kPairThreads;
    uint2 *col = reinterpret_cast<uint2 *>(psmem) + threadIdx.x;
    uint16_t *qs = reinterpret_cast<uint16_t *>(reinterpret_cast<uint2 *>(psmem) + (size_t)(qcap + 1) * T) +
                   threadIdx.x;
    if (n_dev) n = min(n, *n_dev);   // device-side job count (retry rounds)
    unsigned long long cells_total =
        ext_pair_thread<SYM, T>(blockIdx.x * T + threadIdx.x, col, qs, jobs, order, n, qseq, tseq, p, kc, n_code_t,
                             qcap, w_try, out, clamped_out, cells_job, status);
    if (cells_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cells_total += __shfl_down_sync(0xffffffffu, cells_total, o);
        if ((threadIdx.x & 31) == 0 && cells_total) atomicAdd(cells_out, cells_total);
    }
}

PairConsts pair_consts(const ExtParams &p, int *n_code_t, bool *sym) {
    const int a = p.mat[0], b = -p.mat[1], nn = p.mat[4];
    PairConsts kc;
    const uint32_t nb = (uint32_t)(uint8_t)(int8_t)(-b), na = (uint32_t)(uint8_t)(int8_t)nn;
    kc.tab_lo = (uint32_t)(uint8_t)a | nb << 8 | nb << 16 | nb << 24;
    kc.tab_hi = na * 0x01010101u;
    auto rep = [](int v) { return ((uint32_t)(uint16_t)(int16_t)v) * 0x00010001u; };
    kc.neg_oedel2 = rep(-(p.o_del + p.e_del));
    kc.neg_edel2 = rep(-p.e_del);
    kc.neg_oeins2 = rep(-(p.o_ins + p.e_ins));
    kc.neg_eins2 = rep(-p.e_ins);
    kc.kmul = a <= 1 ? 2u : 4u;
    *n_code_t = nn == -1 ? 5 : 4;
    *sym = p.o_del == p.o_ins && p.e_del == p.e_ins;
    return kc;
}

#ifdef FA_HOST_KERNEL_TESTS
// Runs the int16x2 thread body on the CPU for every pair of `order`.  Compiled only into
// the test harness (tests/kernel_host), never into the shipped library.
int ext_pair_host(const fa_job *jobs, const uint32_t *order, uint32_t n, const uint8_t *qseq, const uint8_t *tseq,
                  const ExtParams &p, int qcap, fa_ext_result *out, uint32_t *status) {
    int n_code_t = 0;
    bool sym = false;
    const PairConsts kc = pair_consts(p, &n_code_t, &sym);
    std::vector<uint2> col((size_t)(qcap + 1));
    std::vector<uint16_t> qs((size_t)(qcap + 1));
    for (uint32_t pr = 0; pr < (n + 1) / 2; ++pr) {
        if (sym)
            ext_pair_thread<true, 1>(pr, col.data(), qs.data(), jobs, order, n, qseq, tseq, p, kc, n_code_t, qcap,
                                  nullptr, out, nullptr, nullptr, status);
        else
            ext_pair_thread<false, 1>(pr, col.data(), qs.data(), jobs, order, n, qseq, tseq, p, kc, n_code_t, qcap,
                                   nullptr, out, nullptr, nullptr, status);
    }
    return 0;
}
#endif  // FA_HOST_KERNEL_TESTS

size_t ext_pair_smem_bytes(int qcap) {
    return (size_t)(qcap + 1) * kPairThreads * (sizeof(uint2) + sizeof(uint16_t));
}

// bwa-form scoring: mat[t][q] = a (t == q < 4), -b (t != q, both < 4), n (either is N),
// with 1 <= a <= 3, n in {-1, 0}, and b >= 1 when n = -1.
bool ext_pair_eligible(const ExtParams &p) {
    const int a = p.mat[0], b = -p.mat[1], n = p.mat[4];
    if (a < 1 || a > 3 || (n != -1 && n != 0) || (n == -1 && b < 1) || b > 127) return false;
    for (int t = 0; t < 5; ++t)
        for (int q = 0; q < 5; ++q) {
            const int v = p.mat[t * 5 + q];
            const int want = (t == 4 || q == 4) ? n : (t == q ? a : -b);
            if (v != want) return false;
        }
    if (p.o_del + p.e_del > 16000 || p.o_ins + p.e_ins > 16000) return false;
    return true;
}

cudaError_t launch_ext_pair(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n, const uint32_t *d_n,
                            const SeqBuf &q, const SeqBuf &t, const ExtParams &p, int qcap, const int32_t *d_w_try,
                            fa_ext_result *d_out, uint8_t *d_clamped, uint32_t *d_cells_job,
                            unsigned long long *d_cells, uint32_t *d_status, cudaStream_t stream)
{
    if (q.packed || t.packed) return cudaErrorNotSupported;   // byte codes only
    const uint8_t *d_qseq = q.p, *d_tseq = t.p;
    if (n == 0) return cudaSuccess;
    int n_code_t = 0;
    bool sym = false;
    const PairConsts kc = pair_consts(p, &n_code_t, &sym);
    const size_t smem = ext_pair_smem_bytes(qcap);
    const uint32_t pairs = (n + 1) / 2;
    const uint32_t blocks = (pairs + kPairThreads - 1) / kPairThreads;
    cudaError_t err;
    if (sym) {
        err = cudaFuncSetAttribute(ext_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        ext_pair_kernel<true><<<blocks, kPairThreads, smem, stream>>>(d_jobs, d_order, n, d_n, d_qseq, d_tseq, p, kc,
                                                                      n_code_t, qcap, d_w_try, d_out, d_clamped,
                                                                      d_cells_job, d_cells, d_status);
    } else {
        err = cudaFuncSetAttribute(ext_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        ext_pair_kernel<false><<<blocks, kPairThreads, smem, stream>>>(d_jobs, d_order, n, d_n, d_qseq, d_tseq, p, kc,
                                                                       n_code_t, qcap, d_w_try, d_out, d_clamped,
                                                                       d_cells_job, d_cells, d_status);
    }
    return cudaGetLastError();
}

}  // namespace fa
