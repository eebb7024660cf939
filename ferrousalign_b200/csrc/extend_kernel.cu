// extend_kernel.cu -- banded seed extension (ksw_extend2 semantics) on sm_100a.
//
// One thread owns one extension job (inter-sequence parallelism, as the reference's
// SIMD lanes do) and runs the exact row recurrence of ksw_extend2
// (src/core/alignment/ksw_affine_gap.rs:952-1169), including its adaptive beg/end
// rescans, stale band-edge cells, first-column max rule, z-drop with diagonal
// correction and the earliest-row gscore rule.  Jobs are processed in
// length-sorted order so the 32 jobs of a warp have similar row counts.
//
// Per-thread column state lives in shared memory, one 32-bit word per query
// column, interleaved with stride blockDim.x so every access is bank-conflict
// free whatever column each lane is on:
//     word = H(16 bits) << 16 | E(13 bits) << 3 | query code (3 bits)
// The packed form is exact while h0 + max(mat) * qlen < 8192, which bounds every
// H and E the recurrence can produce; the host routes other jobs elsewhere.
// Cell updates use the Blackwell DPX integer instructions (3-way max, fused
// add-max with ReLU).

#include "fa_cert.cuh"
#include "fa_device.cuh"
#include "fa_kernels.h"
#include "fa_packed.cuh"

namespace fa {

// PRMT in the generic mode: selector nibble bit 3 replicates the sign of the
// selected byte, so (q, q|8, q|8, q|8) sign-extends table byte q to 32 bits.
__device__ __forceinline__ int32_t prmt_s8(uint32_t lo, uint32_t hi, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return static_cast<int32_t>(r);
}

// RING = 0: one shared-memory word per query column (any band).  RING = R > 0: only R
// column words, column j in slot j mod R, plus the query packed 8 codes per word -- for
// bands w <= R/2 - 1, whose rows span at most 2w+2 columns, so a slot is never reused
// while the recurrence can still read it; far less shared memory per job, so several
// times the resident warps.  Columns entering the ring get their query code explicitly,
// and a column the rows grow into after a trim gets the value the full array would
// hold there: 0 once written (trimmed cells are zero), its first-row value if never.
// PK: the sequences are 2-bit packed (SeqBuf.packed), read 16 bases per word load.
template <bool CERT, int RING, int TPB, bool PK>
__global__ void __launch_bounds__(TPB)
ext_packed_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ order,
                  uint32_t n, const uint32_t *__restrict__ first_dev, const uint32_t *__restrict__ n_dev,
                  const SeqBuf qs, const SeqBuf ts, const ExtParams p, int qcap,
                  const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out,
                  uint8_t *__restrict__ clamped_out, uint32_t *__restrict__ cells_job,
                  unsigned long long *__restrict__ cells_out, uint32_t *__restrict__ status)
{
    extern __shared__ uint32_t smem[];
    constexpr int T = TPB;   // threads (= jobs) per block; also the stride of the column words
    const uint32_t first = first_dev ? *first_dev : 0u;   // device-side sub-range of the order
    const uint32_t gi = first + blockIdx.x * T + threadIdx.x;
    uint32_t cells = 0;
    if (n_dev) n = min(n, *n_dev);   // device-side job count (retry rounds)

    if (gi < n) {
        const uint32_t jid = order ? order[gi] : gi;
        const fa_job jb = jobs[jid];
        uint32_t *col = smem + threadIdx.x;
        uint32_t *qw = smem + RING * T + threadIdx.x;     // RING: packed query codes
        const int qlen = jb.qlen, tlen = jb.tlen, h0 = jb.h0;
        const int w = ext_band_clamp(qlen, w_try ? w_try[jid] : jb.w, p);
        if (h0 < 0 || (h0 == 0 && !(p.flags & FA_PARAM_H0_ZERO)) || qlen <= 0 || tlen < 0) {
            atomicOr(status, ST_ARG);
        } else if (h0 == 0) {
            // FA_PARAM_H0_ZERO: the recurrence as written is all zero after row 0
            fa_ext_result r;
            cells = ext_h0_zero_result(qlen, tlen, w, &r);
            out[jid] = r;
            if (clamped_out)
                clamped_out[jid] = (uint8_t)((tlen > 0 && qlen > w + 1 ? 1 : 0) | (CERT ? kBandHintNone << 2 : 0));
            if (cells_job) cells_job[jid] = cells;
        } else if (qlen > qcap || h0 + p.max_score * qlen > kPackedHMax || (RING > 0 && 2 * w + 2 > RING)) {
            atomicOr(status, ST_CAPACITY);
        } else {
            const int oe_del = p.o_del + p.e_del, oe_ins = p.o_ins + p.e_ins;
            const int e_del = p.e_del, e_ins = p.e_ins;
            const uint8_t *Q = qs.p + jb.q_off;    // byte codes (PK false)
            const uint8_t *Tg = ts.p + jb.t_off;
            PackedReader qr, tr;                    // packed bases (PK true)
            if (PK) {
                qr.init(qs, jb.q_off, qlen);
                tr.init(ts, jb.t_off, tlen);
            }
            // eight query codes from column j0 on (0 past the query)
            auto load8 = [&](int j0, uint32_t *qb) {
                if (PK) {
                    uint32_t v[2];
                    qr.getw<2>(j0, v);
#pragma unroll
                    for (int u = 0; u < 8; ++u) qb[u] = (v[u / 4] >> (8 * (u & 3))) & 0xFFu;
                } else {
#pragma unroll
                    for (int u = 0; u < 8; ++u) qb[u] = j0 + u < qlen ? (uint32_t)Q[j0 + u] : 0u;
                }
            };
            // scoring rows as PRMT tables, indexed only with constants
            uint32_t rlo[5], rhi[5];
#pragma unroll
            for (int t = 0; t < 5; ++t) {
                rlo[t] = (uint8_t)p.mat[t * 5] | (uint32_t)(uint8_t)p.mat[t * 5 + 1] << 8 |
                         (uint32_t)(uint8_t)p.mat[t * 5 + 2] << 16 | (uint32_t)(uint8_t)p.mat[t * 5 + 3] << 24;
                rhi[t] = (uint8_t)p.mat[t * 5 + 4];
            }

            // Query codes and the first row: eh[0]=h0, eh[1]=h0-oe_ins, then -e_ins
            // while the previous value exceeds e_ins (ksw_affine_gap.rs:1017-1025).
            uint32_t bad = 0;
            int hp = h0, init_reach = 0;
            bool filling = true;
            // first-row value of column j >= 1 (positive exactly up to init_reach)
            auto init_h = [&](int j) { return j == 0 ? h0 : (j <= init_reach ? h0 - oe_ins - (j - 1) * e_ins : 0); };
            if (RING > 0) {
                init_reach = h0 <= oe_ins ? 0 : (e_ins == 0 ? qlen : min(qlen, 1 + (h0 - oe_ins - 1) / e_ins));
                for (int j0 = 0; j0 < qlen; j0 += 8) {
                    uint32_t qb[8];
                    load8(j0, qb);
                    uint32_t word = 0;
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        bad |= qb[u] >= (uint32_t)p.m;
                        word |= (qb[u] & 7u) << (4 * u);
                        const int j = j0 + u;
                        if (j < RING && j < qlen) col[j * T] = (uint32_t)init_h(j) << 16 | (qb[u] & 7u);
                    }
                    qw[(j0 >> 3) * T] = word;
                }
                if (qlen < RING) col[qlen * T] = (uint32_t)init_h(qlen) << 16;
            }
            // eight independent byte loads in flight per thread before their first use
            for (int j0 = 0; RING == 0 && j0 <= qlen; j0 += 8) {
                uint32_t qb[8];
                load8(j0, qb);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int j = j0 + u;
                    if (j <= qlen) {
                        uint32_t q = qb[u];
                        if (j < qlen) {
                            bad |= q >= (uint32_t)p.m;
                            q &= 7u;
                        }
                        int h;
                        if (j == 0) h = h0;
                        else if (j == 1) h = h0 > oe_ins ? h0 - oe_ins : 0;
                        else if (filling && hp > e_ins) h = hp - e_ins;
                        else { filling = false; h = 0; }
                        hp = h;
                        if (CERT && j > 0 && h > 0) init_reach = j;
                        col[j * T] = (uint32_t)h << 16 | q;
                    }
                }
            }

            int best = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, max_off = 0;
            int beg = 0, end = qlen, clamped = 0;
            const int a = p.max_score;
            ExitBound xb;
            int bmax = ExitBound::NEG, first_fail = INT32_MAX, max_written = -1, rows = 0, prev_end = 0;
            int srun = 0, sev = 0, slast = 0;   // bound shortfall: running max, at the last event, last row
            bool row_ok = true, stale = false, broke = false, zbreak = false;
            auto slot = [](int j) { return RING > 0 ? (j & (RING - 1)) : j; };
            auto qcode = [&](int j) { return (qw[(j >> 3) * T] >> (4 * (j & 7))) & 7u; };
            if (CERT) xb.init();
            // target bases arrive 5 to 8 rows ahead of their row: tq0 holds the current
            // group of four, tq1 the next, loaded when tq0 is used up
            uint32_t tq0 = 0, tq1 = 0;
            PackedStream4 tstream;   // PK: target positions 0, 4, 8, ...
            if (PK) {
                tstream.start(0);
                tq0 = tstream.next4(tr);
                tq1 = tstream.next4(tr);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k < tlen) tq0 |= (uint32_t)Tg[k] << (8 * k);
                    if (4 + k < tlen) tq1 |= (uint32_t)Tg[4 + k] << (8 * k);
                }
            }
            for (int i = 0; i < tlen; ++i) {
                const uint32_t tb = tq0 & 0xFFu;
                tq0 >>= 8;
                if ((i & 3) == 3) {
                    tq0 = tq1;
                    tq1 = 0;
                    if (PK) {
                        tq1 = tstream.next4(tr);   // positions i + 5 .. i + 8
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (i + 5 + k < tlen) tq1 |= (uint32_t)Tg[i + 5 + k] << (8 * k);
                    }
                }
                if (tb >= (uint32_t)p.m) { bad = 1; break; }
                uint32_t row_lo = rlo[0], row_hi = rhi[0];
#pragma unroll
                for (int t = 1; t < 5; ++t)
                    if (tb == (uint32_t)t) { row_lo = rlo[t]; row_hi = rhi[t]; }

                const int beg_a = beg, end_a = end < qlen ? end : qlen;
                if (beg < i - w) beg = i - w;
                if (end > i + w + 1) end = i + w + 1;
                if (end > qlen) end = qlen;
                clamped |= (beg != beg_a) | (end != end_a);
                if (CERT) {
                    ++rows;
                    if (i == 0) {
                        if (end < qlen) xb.add(0, (int)(col[slot(end) * T] >> 16), -1, end - 1, qlen, a, e_del);
                    } else {
                        for (int j = beg_a; j < beg && j < qlen; ++j)          // columns the band drops
                            xb.add(1, (int)((col[slot(j) * T] >> 3) & 0x1FFFu), i, j, qlen, a, e_del);
                        if (beg_a == 0 && beg > 0)                            // the first column leaves
                            xb.add(1, h0 - (p.o_del + e_del * i), i - 1, -1, qlen, a, e_del);
                        const int lo = max(beg, max_written + 1), hi = min(end - 1, init_reach);
                        stale |= lo <= hi;                                    // a never-written column
                    }
                }

                int h1 = 0;
                if (beg == 0) {
                    h1 = h0 - (p.o_del + e_del * (i + 1));
                    if (h1 < 0) h1 = 0;
                }
                if (RING > 0) {
                    // a column grown into after a trim: the full array's value there
                    if (i > 0 && end > prev_end + 1) {
                        const int j = prev_end + 1;
                        const int hv = j > max_written ? init_h(j) : 0;
                        col[slot(j) * T] = (uint32_t)hv << 16 | qcode(j);
                    }
                }
                int f = 0, key = 0;
#pragma unroll 4
                for (int j = beg; j < end; ++j) {
                    const uint32_t wd = col[slot(j) * T];
                    int h;
                    if constexpr (!CERT) {
                        // Unpacking, the key and the repacking as multiplies and high
                        // multiplies, which can issue on the FMA pipe beside the DPX max/add
                        // work on the integer pipe (measured faster for this variant; the
                        // certificate variants keep the shift form, which needs fewer
                        // registers there).
                        const int M = (int)__umulhi(wd, 1u << 16);                  // bits 16..31
                        const int e = (int)__umulhi(wd * (1u << 16), 1u << 13);     // bits 3..15
                        const uint32_t q = wd & 7u;
                        const int s = prmt_s8(row_lo, row_hi, q * 0x1111u + 0x8880u);
                        // M == 0 leaves no diagonal term (ksw_extend2's `M ? M + s : 0`); any
                        // value <= 0 acts exactly like 0 in every max below, and for M > 0
                        // M * 8192 exceeds M + s
                        const int Mp = __viaddmin_s32(M, s, M * 8192);
                        h = __vimax3_s32(Mp, e, f);
                        const int e_new = __viaddmax_s32_relu(e, -e_del, Mp - oe_del);
                        f = __viaddmax_s32_relu(f, -e_ins, Mp - oe_ins);
                        key = max(key, h * 4096 + (4095 - j));   // first column of the row max
                        col[slot(j) * T] = (uint32_t)h1 * 65536u + (uint32_t)e_new * 8u + q;
                    } else {
                        const int M = (int)(wd >> 16);
                        const int e = (int)((wd >> 3) & 0x1FFFu);
                        const uint32_t q = wd & 7u;
                        const int s = prmt_s8(row_lo, row_hi, q * 0x1111u + 0x8880u);
                        const int Mp = M ? M + s : 0;
                        h = __vimax3_s32(Mp, e, f);
                        const int e_new = __viaddmax_s32_relu(e, -e_del, Mp - oe_del);
                        f = __viaddmax_s32_relu(f, -e_ins, Mp - oe_ins);
                        key = max(key, (h << 12) | (4095 - j));   // first column of the row max
                        col[slot(j) * T] = (uint32_t)h1 << 16 | (uint32_t)e_new << 3 | q;
                    }
                    h1 = h;
                }
                if (RING > 0) {
                    col[slot(end) * T] = (uint32_t)h1 << 16 | (end < qlen ? qcode(end) : 0u);
                    max_written = max(max_written, end);
                    prev_end = end;
                } else {
                    const uint32_t wd = col[end * T];
                    col[end * T] = (uint32_t)h1 << 16 | (wd & 7u);
                }
                if (end > beg) cells += end - beg;
                if (end == qlen && gscore < h1) { gscore = h1; max_ie = i; }
                const int m_row = key >> 12;
                const int mj = 4095 - (key & 4095);
                if (CERT) {
                    if (RING == 0) max_written = max(max_written, end);
                    if (end < qlen) xb.add(0, f, i, end, qlen, a, e_del);   // F past the row's end
                    const int b = xb.at(i, a, e_del);
                    row_ok = m_row > 0 ? b < m_row : b <= 0;
                    if (!row_ok && first_fail == INT32_MAX) first_fail = i;
                    slast = row_ok ? 0 : b - m_row + 1;
                    srun = max(srun, slast);
                    if (max_ie == i) sev = srun;
                    bmax = max(bmax, b);
                }
                if (m_row == 0) { broke = true; break; }
                if (m_row > best) {
                    best = m_row; max_i = i; max_j = mj;
                    if (CERT) sev = srun;
                    const int off = mj > i ? mj - i : i - mj;
                    if (max_off < off) max_off = off;
                } else if (p.zdrop > 0) {
                    const int di = i - max_i, dj = mj - max_j;
                    if (di > dj) {
                        if (best - m_row - (di - dj) * e_del > p.zdrop) { broke = zbreak = true; break; }
                    } else if (best - m_row - (dj - di) * e_ins > p.zdrop) {
                        broke = zbreak = true;
                        break;
                    }
                }
                int nb = beg;
                while (nb < end && (col[slot(nb) * T] >> 3) == 0) ++nb;
                beg = nb;
                int ne = end;
                while (ne > beg && (col[slot(ne) * T] >> 3) == 0) --ne;
                end = ne + 2 < qlen ? ne + 2 : qlen;
            }
            if (bad) atomicOr(status, ST_BAD_CODE);
            fa_ext_result r;
            r.score = best;
            r.qle = max_j + 1;
            r.tle = max_i + 1;
            r.gtle = max_ie + 1;
            r.gscore = gscore;
            r.max_off = max_off;
            out[jid] = r;
            uint8_t flags = (uint8_t)clamped;
            if (CERT) {
                const int i_ev = max(max_i, max_ie), lim = min(best, gscore);
                // after a zero row every live path has left the region: a wider run's
                // remaining rows are bounded by the tents over [last row, tlen-1]
                const int fut = (broke && !zbreak) ? xb.max_over(rows - 1, tlen - 1, a, e_del) : ExitBound::NEG;
                const bool tail_ok = !broke || (zbreak ? row_ok : fut < lim);
                const int W = ext_band_clamp(qlen, jb.w, p);
                const bool wide_clean = init_reach <= min(W + 1, qlen);
                const bool cert = !stale && gscore > 0 && first_fail > i_ev && tail_ok && bmax < lim && wide_clean;
                flags |= (uint8_t)cert << 1;
                // bits 2-7: extra band columns the certificate's shortfall asks for (63: none);
                // widening the band moves every exit at least one gap extension further away
                int slack = sev;                            // rows up to the last event count
                if (broke && zbreak) slack = max(slack, slast);
                if (bmax >= lim) slack = max(slack, bmax - lim + 1);
                if (broke && !zbreak && fut >= lim) slack = max(slack, fut - lim + 1);
                const int e_min = min(e_del, e_ins);
                int hint = kBandHintNone;
                if (!stale && gscore > 0 && e_min > 0 && wide_clean)
                    hint = min(kBandHintNone, (max(slack, 1) + e_min - 1) / e_min);
                flags |= (uint8_t)(hint << 2);
            }
            if (clamped_out) clamped_out[jid] = flags;
            if (cells_job) cells_job[jid] = cells;
        }
    }
    if (cells_out) {
        unsigned long long c = cells;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(cells_out, c);
    }
}

size_t ext_packed_smem_bytes(int qcap, int ring, int tpb) {
    const size_t words = ring > 0 ? (size_t)ring + (size_t)(qcap + 7) / 8 : (size_t)qcap + 1;
    return words * (size_t)tpb * sizeof(uint32_t);
}

namespace {
template <bool CERT, int RING, int TPB>
cudaError_t launch_variant(size_t smem, cudaStream_t stream, const fa_job *d_jobs, const uint32_t *d_order,
                           uint32_t n, const uint32_t *d_first, const uint32_t *d_n, const SeqBuf &d_qseq,
                           const SeqBuf &d_tseq, const ExtParams &p, int qcap, const int32_t *d_w_try,
                           fa_ext_result *d_out, uint8_t *d_clamped, uint32_t *d_cells_job,
                           unsigned long long *d_cells, uint32_t *d_status)
{
    if (d_qseq.packed) {
        cudaError_t err = cudaFuncSetAttribute(ext_packed_kernel<CERT, RING, TPB, true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        ext_packed_kernel<CERT, RING, TPB, true><<<(n + TPB - 1) / TPB, TPB, smem, stream>>>(
            d_jobs, d_order, n, d_first, d_n, d_qseq, d_tseq, p, qcap, d_w_try, d_out, d_clamped, d_cells_job,
            d_cells, d_status);
        return cudaGetLastError();
    }
    cudaError_t err = cudaFuncSetAttribute(ext_packed_kernel<CERT, RING, TPB, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const uint32_t blocks = (n + TPB - 1) / TPB;
    ext_packed_kernel<CERT, RING, TPB, false><<<blocks, TPB, smem, stream>>>(
        d_jobs, d_order, n, d_first, d_n, d_qseq, d_tseq, p, qcap, d_w_try, d_out, d_clamped, d_cells_job,
        d_cells, d_status);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_ext_packed(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n,
                              const uint32_t *d_first, const uint32_t *d_n, const SeqBuf &d_qseq,
                              const SeqBuf &d_tseq, const ExtParams &p, int qcap, int ring,
                              const int32_t *d_w_try, fa_ext_result *d_out, uint8_t *d_clamped, bool cert,
                              uint32_t *d_cells_job, unsigned long long *d_cells, uint32_t *d_status,
                              cudaStream_t stream, int tpb)
{
    if (n == 0) return cudaSuccess;
    if (ring != 0 && ring != 32 && ring != 64) return cudaErrorInvalidValue;
    // the certificate variant only where a judge reads it (it adds work to every row);
    // block sizes other than the default only for the plain full-row kernel
    const bool c = cert && d_clamped;
    if (c || ring != 0 || (tpb != 64 && tpb != 256)) tpb = kExtThreads;
    if (tpb == 256) {   // a block of 256 jobs holds twice the shared memory: fall back when it does not fit
        int dev = 0, optin = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
            ext_packed_smem_bytes(qcap, ring, 256) > (size_t)optin)
            tpb = kExtThreads;
    }
    const size_t smem = ext_packed_smem_bytes(qcap, ring, tpb);
#define FA_EXT_LAUNCH(CV, RV, TV) launch_variant<CV, RV, TV>(smem, stream, d_jobs, d_order, n, d_first, d_n, d_qseq, \
                                                             d_tseq, p, qcap, d_w_try, d_out, d_clamped, d_cells_job, \
                                                             d_cells, d_status)
    if (ring == 32) return c ? FA_EXT_LAUNCH(true, 32, kExtThreads) : FA_EXT_LAUNCH(false, 32, kExtThreads);
    if (ring == 64) return c ? FA_EXT_LAUNCH(true, 64, kExtThreads) : FA_EXT_LAUNCH(false, 64, kExtThreads);
    if (c) return FA_EXT_LAUNCH(true, 0, kExtThreads);
    if (tpb == 64) return FA_EXT_LAUNCH(false, 0, 64);
    if (tpb == 256) return FA_EXT_LAUNCH(false, 0, 256);
    return FA_EXT_LAUNCH(false, 0, kExtThreads);
#undef FA_EXT_LAUNCH
}

}  // namespace fa
