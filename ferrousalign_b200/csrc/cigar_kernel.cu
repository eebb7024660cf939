// cigar_kernel.cu -- banded Smith-Waterman with traceback for CIGAR regeneration (sm_100a).
//
// scalar_banded_swa (src/core/alignment/banded_swa/scalar/implementation.rs:5-440), the
// alignment the region step runs to turn a region's bounds back into a CIGAR
// (src/pipelines/linear/region.rs:1029-1070): the banded row recurrence of ksw_extend2
// with three differences -- the match term is clamped at zero (H(i-1,j-1) + s, then 0
// if negative) rather than gated on H(i-1,j-1) > 0, the band is used as given, and every
// cell records which of M, E (deletion) and F (insertion) it took (ties to M, then E) --
// followed by a traceback from the best cell to the matrix edge that emits run-length
// M / D / I operations and the aligned reference and query bases, a 5' soft clip for the
// query left over, and at the 3' end either a soft clip or an M run to the query end by
// bwa-mem2's clip rule (gscore <= 0 or gscore <= score - pen_clip3: clip).
//
// One thread per alignment, jobs ordered by band so that a warp's rows have similar
// lengths.  The row state (H, E per query column) sits in shared memory as 16-bit pairs
// when every score of the batch fits (otherwise in a per-job int32 global scratch); each
// row's cells run eight at a time in straight-line code.  The traceback codes take two
// bits per cell of the row's band [cb, ce) behind a header word naming it (at most
// min(2w + 1, qlen) columns), kept per job in global memory; cells outside a row's band
// were never written and read as M, as the reference's zero-initialised matrix does.

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

namespace {

constexpr int kCigarThreads = 64;
constexpr size_t kCigarSmemMax = 96 * 1024;   // shared row state per block, at most
constexpr uint8_t TB_M = 0, TB_D = 1, TB_I = 2;   // types.rs:101-103
constexpr int kMaxTraceSteps = 10000;             // implementation.rs:253

// Traceback codes: row i holds a header word (its first coded column cb, and the count
// ce - cb) and then two bits per column from cb on; a cell outside [cb, ce) was never
// written and reads as M, as the reference's zero-initialised matrix does.
struct CigarCtx {
    const uint32_t *tb;
    int wpr;
    __device__ __forceinline__ uint32_t at(int ii, int jj) const {   // tb[ii][jj] of the reference
        if (ii == 0) return jj == 0 ? TB_M : TB_I;
        if (jj == 0) return TB_D;
        const uint32_t *row = tb + (size_t)(ii - 1) * (wpr + 1);
        const uint32_t hdr = row[0];
        const int k = jj - 1 - (int)(hdr & 0xFFFFu);
        if (k < 0 || k >= (int)(hdr >> 16)) return TB_M;
        return (row[1 + (k >> 4)] >> ((k & 15) * 2)) & 3u;
    }
};

__device__ __forceinline__ uint32_t cigar_op(uint32_t op, uint32_t len) { return len << 4 | op; }

// Row state of one job (H of the previous row's cell and E, per query column 0..qlen): int32
// pairs in a per-job global scratch, or 16-bit pairs in shared memory (one word per column,
// the block's jobs interleaved so that each thread's accesses hit its own bank).
// ldq(j, Q, q): the column's (H, E) and its query code (raw, as the sequence holds it);
// st(j, h, e, q) stores a column the row computed, st_end(j, h) the row's end word (E = 0).
struct EhGlobal {
    static constexpr bool kNarrow = false;   // scores may pass 16 bits
    int2 *eh;
    __device__ __forceinline__ int2 ld(int j) const { return eh[j]; }
    __device__ __forceinline__ int2 ldq(int j, const uint8_t *Q, uint32_t &q) const { q = Q[j]; return eh[j]; }
    __device__ __forceinline__ void init(int j, int h, const uint8_t *) const { eh[j] = make_int2(h, 0); }
    __device__ __forceinline__ void st(int j, int h, int e, uint32_t) const { eh[j] = make_int2(h, e); }
    __device__ __forceinline__ void st_end(int j, int h) const { eh[j] = make_int2(h, 0); }
};
struct EhShared {
    static constexpr bool kNarrow = true;    // every score < 32768
    uint32_t *w;   // w[j * stride]
    int stride;
    __device__ __forceinline__ int2 ld(int j) const {
        const uint32_t v = w[j * stride];
        return make_int2((int)(v & 0xFFFFu), (int)(v >> 16));
    }
    __device__ __forceinline__ int2 ldq(int j, const uint8_t *Q, uint32_t &q) const { q = Q[j]; return ld(j); }
    __device__ __forceinline__ void init(int j, int h, const uint8_t *) const { w[j * stride] = (uint32_t)h; }
    __device__ __forceinline__ void st(int j, int h, int e, uint32_t) const {
        w[j * stride] = (uint32_t)h | (uint32_t)e << 16;
    }
    __device__ __forceinline__ void st_end(int j, int h) const { w[j * stride] = (uint32_t)h; }
};
// The same with the column's query code in the word (H in bits 0-12, E in 13-25, the code
// clamped to 4 in 26-28): every score < 8192, and a step reads no query byte from global
// memory (the traceback reads the raw bases).
struct EhSharedQ {
    static constexpr bool kNarrow = true;
    uint32_t *w;
    int stride;
    __device__ __forceinline__ int2 ld(int j) const {
        const uint32_t v = w[j * stride];
        return make_int2((int)(v & 0x1FFFu), (int)((v >> 13) & 0x1FFFu));
    }
    __device__ __forceinline__ int2 ldq(int j, const uint8_t *, uint32_t &q) const {
        const uint32_t v = w[j * stride];
        q = v >> 26;
        return make_int2((int)(v & 0x1FFFu), (int)((v >> 13) & 0x1FFFu));
    }
    __device__ __forceinline__ void init(int j, int h, const uint8_t *Q) const {
        const uint32_t q = Q ? min((uint32_t)Q[j], 4u) : 0u;
        w[j * stride] = (uint32_t)h | q << 26;
    }
    __device__ __forceinline__ void st(int j, int h, int e, uint32_t q) const {
        w[j * stride] = (uint32_t)h | (uint32_t)e << 13 | q << 26;
    }
    __device__ __forceinline__ void st_end(int j, int h) const {
        uint32_t *x = &w[j * stride];
        *x = (*x & 0xFC000000u) | (uint32_t)h;
    }
};

// One alignment: the banded rows into the row state and the traceback words, then the
// traceback, clips and result of job k.
// The scoring matrix rows as PRMT tables: rt[t] holds mat[t][0..3], rt[5 + t] mat[t][4]
// (one signed byte per query code), for target code t.  Threads 0-4 write them; the caller
// synchronises before use.
__device__ __forceinline__ void cigar_row_tables(uint32_t *rt, const ExtParams &p) {
    if (threadIdx.x < 5) {
        const int t = threadIdx.x;
        rt[t] = (uint32_t)(uint8_t)p.mat[t * 5] | (uint32_t)(uint8_t)p.mat[t * 5 + 1] << 8 |
                (uint32_t)(uint8_t)p.mat[t * 5 + 2] << 16 | (uint32_t)(uint8_t)p.mat[t * 5 + 3] << 24;
        rt[5 + t] = (uint32_t)(uint8_t)p.mat[t * 5 + 4];
    }
}

// rt: the scoring matrix as PRMT tables in shared memory (cigar_row_tables).
template <class EH>
__device__ __forceinline__ void cigar_job(uint32_t k, const fa_cigar_job &J, const CigarPlan &P,
                                          const uint8_t *__restrict__ qseq, const uint8_t *__restrict__ tseq,
                                          const ExtParams &p, int pen_clip3, const EH eh, const uint32_t *rt,
                                          uint32_t *__restrict__ tb_all, fa_cigar_result *__restrict__ out,
                                          uint32_t *__restrict__ cigar, uint8_t *__restrict__ ref_al,
                                          uint8_t *__restrict__ qry_al)
{
    fa_cigar_result r;
    r.score = r.qle = r.tle = r.gtle = r.gscore = r.max_off = 0;
    r.n_cigar = r.n_ref = r.n_query = 0;
    r.cells = 0;
    const int qlen = J.qlen, tlen = J.tlen, w = J.w, h0 = J.h0;
    if (qlen <= 0 || tlen <= 0) {   // implementation.rs:17-30
        out[k] = r;
        return;
    }
    const uint8_t *Q = qseq + J.q_off;
    const uint8_t *T = tseq + J.t_off;
    uint32_t *tb = tb_all + P.tb;
    const int oe_del = p.o_del + p.e_del, oe_ins = p.o_ins + p.e_ins;
    // first row (implementation.rs:67-75)
    // (a row state that carries the query codes gets them here, column qlen none)
    eh.init(0, h0, Q);   // qlen >= 1 here
    int hp = h0 > oe_ins ? h0 - oe_ins : 0;
    eh.init(1, hp, qlen > 1 ? Q : nullptr);
    for (int j = 2; j <= qlen; ++j) {
        hp = hp > p.e_ins ? hp - p.e_ins : 0;
        eh.init(j, hp, j < qlen ? Q : nullptr);
    }
    int max_score = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, max_off = 0;
    int beg = 0, end = qlen, cells = 0;
    int t_next = T[0];   // the next row's target base, loaded a row ahead
    for (int i = 0; i < tlen; ++i) {
        const int t_cur = t_next;
        if (i + 1 < tlen) t_next = T[i + 1];
        const int tbase = t_cur < 4 ? t_cur : 4;
        const uint32_t rlo = rt[tbase], rhi = rt[5 + tbase];   // this row's scores, one byte per query code
        int cb = beg, ce = end;
        if (cb < i - w) cb = i - w;
        if (ce > i + w + 1) ce = i + w + 1;
        if (ce > qlen) ce = qlen;
        int h1 = 0;
        if (cb == 0) {
            h1 = h0 - (p.o_del + p.e_del * (i + 1));
            if (h1 < 0) h1 = 0;
        }
        int f = 0;
        // row maximum and its first column: packed h << 16 | (0xFFFF - j) for 16-bit scores,
        // else as a pair
        int best = 0, m_val = 0, mj = -1;
        uint32_t *rowtb = tb + (size_t)i * (P.wpr + 1);
        rowtb[0] = (uint32_t)cb | (uint32_t)(ce > cb ? ce - cb : 0) << 16;   // the columns this row codes
        uint32_t acc = 0;
        // eight columns a step: their row-state words and query bases are loaded together
        // (each is overwritten only at its own column, so the loads may run ahead)
        for (int j0 = cb, st = 0; j0 < ce; j0 += 8, ++st) {
            int2 ev[8];
            uint32_t qv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                ev[u] = make_int2(0, 0);
                qv[u] = 0;
                if (j0 + u < ce) ev[u] = eh.ldq(j0 + u, Q, qv[u]);
            }
            uint32_t chunk = 0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int j = j0 + u;
                if (j >= ce) break;
                const uint32_t q = min(qv[u], 4u);
                uint32_t sv;
                asm("prmt.b32 %0, %1, %2, %3;" : "=r"(sv) : "r"(rlo), "r"(rhi), "r"(q | (q | 8u) << 4));
                const int m = __viaddmax_s32_relu(ev[u].x, (int)(int16_t)(sv & 0xFFFFu), 0);   // clamped at zero
                const int e = ev[u].y;
                const int ef = max(e, f);
                const int h = max(m, ef);
                const uint32_t code = m >= ef ? TB_M : (e >= f ? TB_D : TB_I);
                chunk |= code << (2 * u);
                if (EH::kNarrow) {
                    best = max(best, h << 16 | (0xFFFF - j));
                } else if (m_val < h) {
                    m_val = h;
                    mj = j;
                }
                const int en = __viaddmax_s32_relu(e, -p.e_del, m - oe_del);
                eh.st(j, h1, en, q);   // H of the previous row's cell, E for the next row
                f = __viaddmax_s32_relu(f, -p.e_ins, m - oe_ins);
                h1 = h;
            }
            if (st & 1) {
                rowtb[1 + (st >> 1)] = acc | chunk << 16;
            } else {
                acc = chunk;
                if (j0 + 8 >= ce) rowtb[1 + (st >> 1)] = acc;
            }
        }
        if (EH::kNarrow) {
            m_val = best >> 16;
            mj = 0xFFFF - (best & 0xFFFF);
        }
        if (ce > cb) cells += ce - cb;
        eh.st_end(ce, h1);
        if (ce == qlen && gscore < h1) { gscore = h1; max_ie = i; }
        if (m_val == 0) break;
        if (m_val > max_score) {
            max_score = m_val;
            max_i = i;
            max_j = mj;
            const int off = mj > i ? mj - i : i - mj;
            max_off = max_off > off ? max_off : off;
        } else if (p.zdrop > 0) {
            const int di = i - max_i, dj = mj - max_j;
            if (di > dj) {
                if (max_score - m_val - (di - dj) * p.e_del > p.zdrop) break;
            } else if (max_score - m_val - (dj - di) * p.e_ins > p.zdrop) {
                break;
            }
        }
        int nb = cb;
        while (nb < ce) {
            const int2 v = eh.ld(nb);
            if (v.x != 0 || v.y != 0) break;
            ++nb;
        }
        beg = nb;
        int ne = ce;
        while (ne >= beg) {
            const int2 v = eh.ld(ne);
            if (v.x != 0 || v.y != 0) break;
            --ne;
        }
        end = ne + 2 < qlen ? ne + 2 : qlen;
    }

    // traceback from the best cell (implementation.rs:239-321); operations and bases come
    // out last to first and are reversed afterwards.  Slot 0 is kept for a 5' clip.
    const CigarCtx tbx{tb, P.wpr};
    uint32_t *ops = cigar + P.cig;
    uint8_t *ra = ref_al + P.ref, *qa = qry_al + P.qry;
    int ci = max_i + 1, cj = max_j + 1, nops = 0, nr = 0, nq = 0;
    for (int it = 0; (ci > 0 || cj > 0) && it < kMaxTraceSteps; ++it) {
        const int pi = ci, pj = cj;
        const uint32_t code = tbx.at(ci, cj);
        int cnt = 0;
        if (code == TB_M) {
            while (ci > 0 && cj > 0 && tbx.at(ci, cj) == TB_M) {
                ra[nr++] = T[ci - 1];
                qa[nq++] = Q[cj - 1];
                --ci;
                --cj;
                ++cnt;
            }
            if (cnt) ops[1 + nops++] = cigar_op(0, cnt);
        } else if (code == TB_D) {
            while (ci > 0 && tbx.at(ci, cj) == TB_D) {
                ra[nr++] = T[ci - 1];
                --ci;
                ++cnt;
            }
            if (cnt) ops[1 + nops++] = cigar_op(2, cnt);
        } else if (code == TB_I) {
            while (cj > 0 && tbx.at(ci, cj) == TB_I) {
                qa[nq++] = Q[cj - 1];
                --cj;
                ++cnt;
            }
            if (cnt) ops[1 + nops++] = cigar_op(1, cnt);
        } else {
            break;
        }
        if (ci == pi && cj == pj) break;
    }
    for (int a = 0, b = nops - 1; a < b; ++a, --b) {
        const uint32_t t = ops[1 + a];
        ops[1 + a] = ops[1 + b];
        ops[1 + b] = t;
    }
    for (int a = 0, b = nr - 1; a < b; ++a, --b) {
        const uint8_t t = ra[a];
        ra[a] = ra[b];
        ra[b] = t;
    }
    for (int a = 0, b = nq - 1; a < b; ++a, --b) {
        const uint8_t t = qa[a];
        qa[a] = qa[b];
        qa[b] = t;
    }
    // clips (implementation.rs:340-412)
    const int qs = cj, qe = max_j + 1;
    int total = nops;
    if (qs > 0) {
        ops[0] = cigar_op(4, qs);
        ++total;
    } else {
        for (int a = 0; a < nops; ++a) ops[a] = ops[a + 1];
    }
    if (qe < qlen) {
        const bool clip = gscore <= 0 || gscore <= max_score - pen_clip3;
        ops[total++] = cigar_op(clip ? 4 : 0, qlen - qe);
    }
    r.score = max_score;
    r.qle = max_j + 1;
    r.tle = max_i + 1;
    r.gtle = max_ie + 1;
    r.gscore = gscore;
    r.max_off = max_off;
    r.n_cigar = total;
    r.n_ref = nr;
    r.n_query = nq;
    r.cells = cells;
    out[k] = r;
}

__global__ void __launch_bounds__(kCigarThreads)
cigar_kernel(const fa_cigar_job *__restrict__ jobs, const CigarPlan *__restrict__ plan, uint32_t n,
             const uint8_t *__restrict__ qseq, const uint8_t *__restrict__ tseq, const ExtParams p, int pen_clip3,
             int2 *__restrict__ eh_all, uint32_t *__restrict__ tb_all, fa_cigar_result *__restrict__ out,
             uint32_t *__restrict__ cigar, uint8_t *__restrict__ ref_al, uint8_t *__restrict__ qry_al)
{
    __shared__ uint32_t rt[10];
    cigar_row_tables(rt, p);
    __syncthreads();
    const uint32_t k = blockIdx.x * kCigarThreads + threadIdx.x;
    if (k >= n) return;
    const CigarPlan P = plan[k];
    cigar_job(k, jobs[k], P, qseq, tseq, p, pen_clip3, EhGlobal{eh_all + P.eh}, rt, tb_all, out, cigar, ref_al,
              qry_al);
}

// The row state in shared memory as 16-bit pairs (every score of the batch fits: the host
// checks h0 + qlen * max <= 32767), jobs taken in `order` (similar bands side by side in a
// warp), (qcap + 1) words per thread.
// QW: the row-state words also carry the query codes (EhSharedQ).
template <bool QW>
__global__ void __launch_bounds__(kCigarThreads)
cigar_smem_kernel(const fa_cigar_job *__restrict__ jobs, const CigarPlan *__restrict__ plan,
                  const uint32_t *__restrict__ order, uint32_t n, const uint8_t *__restrict__ qseq,
                  const uint8_t *__restrict__ tseq, const ExtParams p, int pen_clip3, uint32_t *__restrict__ tb_all,
                  fa_cigar_result *__restrict__ out, uint32_t *__restrict__ cigar, uint8_t *__restrict__ ref_al,
                  uint8_t *__restrict__ qry_al)
{
    extern __shared__ uint32_t ehs[];   // 16 words of tables, then the row state
    cigar_row_tables(ehs, p);
    __syncthreads();
    const uint32_t t = blockIdx.x * kCigarThreads + threadIdx.x;
    if (t >= n) return;
    const uint32_t k = order[t];
    if (QW)
        cigar_job(k, jobs[k], plan[k], qseq, tseq, p, pen_clip3, EhSharedQ{ehs + 16 + threadIdx.x, kCigarThreads},
                  ehs, tb_all, out, cigar, ref_al, qry_al);
    else
        cigar_job(k, jobs[k], plan[k], qseq, tseq, p, pen_clip3, EhShared{ehs + 16 + threadIdx.x, kCigarThreads},
                  ehs, tb_all, out, cigar, ref_al, qry_al);
}

// Packs the jobs' CIGAR words back to back: job k's n_cigar words from its capacity slot
// to first[k] (one warp per job; a job has a handful of operations).
__global__ void __launch_bounds__(256)
cigar_pack_kernel(const CigarPlan *__restrict__ plan, const fa_cigar_result *__restrict__ res,
                  const uint64_t *__restrict__ first, uint32_t n, const uint32_t *__restrict__ cigar,
                  uint32_t *__restrict__ packed)
{
    const uint32_t k = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (k >= n) return;
    const uint32_t *src = cigar + plan[k].cig;
    uint32_t *dst = packed + first[k];
    const int m = res[k].n_cigar;
    for (int i = threadIdx.x & 31; i < m; i += 32) dst[i] = src[i];
}

}  // namespace

int cigar_band_words(int qlen, int w) {
    const long long cols = 2ll * w + 1 < qlen ? 2ll * w + 1 : qlen;
    return cols <= 0 ? 0 : (int)((cols + 15) / 16);
}

cudaError_t launch_cigar(const fa_cigar_job *d_jobs, const CigarPlan *d_plan, uint32_t n, const uint8_t *d_qseq,
                         const uint8_t *d_tseq, const ExtParams &p, int pen_clip3, int2 *d_eh, uint32_t *d_tb,
                         fa_cigar_result *d_out, uint32_t *d_cigar, uint8_t *d_ref_al, uint8_t *d_qry_al,
                         cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    cigar_kernel<<<(n + kCigarThreads - 1) / kCigarThreads, kCigarThreads, 0, s>>>(
        d_jobs, d_plan, n, d_qseq, d_tseq, p, pen_clip3, d_eh, d_tb, d_out, d_cigar, d_ref_al, d_qry_al);
    return cudaGetLastError();
}

cudaError_t launch_cigar_smem(const fa_cigar_job *d_jobs, const CigarPlan *d_plan, const uint32_t *d_order,
                              uint32_t n, int qcap, bool qwords, const uint8_t *d_qseq, const uint8_t *d_tseq,
                              const ExtParams &p, int pen_clip3, uint32_t *d_tb, fa_cigar_result *d_out,
                              uint32_t *d_cigar, uint8_t *d_ref_al, uint8_t *d_qry_al, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const size_t smem = sizeof(uint32_t) * (16 + kCigarThreads * (size_t)(qcap + 1));
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        kernel<<<(n + kCigarThreads - 1) / kCigarThreads, kCigarThreads, smem, s>>>(
            d_jobs, d_plan, d_order, n, d_qseq, d_tseq, p, pen_clip3, d_tb, d_out, d_cigar, d_ref_al, d_qry_al);
        return cudaGetLastError();
    };
    return qwords ? go(cigar_smem_kernel<true>) : go(cigar_smem_kernel<false>);
}

int cigar_smem_qcap() { return (int)((kCigarSmemMax - 64) / (sizeof(uint32_t) * kCigarThreads)) - 1; }

cudaError_t launch_cigar_pack(const CigarPlan *d_plan, const fa_cigar_result *d_res, const uint64_t *d_first,
                              uint32_t n, const uint32_t *d_cigar, uint32_t *d_packed, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    cigar_pack_kernel<<<(n + 7) / 8, 256, 0, s>>>(d_plan, d_res, d_first, n, d_cigar, d_packed);
    return cudaGetLastError();
}

}  // namespace fa
