// extend_rows2_kernel.cu -- banded seed extension, two target rows per thread (sm_100a).
//
// Same recurrence, band rescans, stale-cell semantics and outputs as ext_packed_kernel
// (ksw_extend2, src/core/alignment/ksw_affine_gap.rs:952-1169).  One thread owns one job
// and computes rows i and i+1 together in int16x2 registers: the low half holds row i at
// column j, the high half row i+1 at column j-1.  Row i+1's inputs at column j-1 (row i's
// H at column j-2 and its E for column j-1) are the low half's results of the two previous
// steps, so they never pass through shared memory, and every DPX instruction updates two
// cells.  Shared memory is read once (row i-1's column word) and written once (row i+1's)
// per two cells.
//
// Column words are 16 bits, H in the low byte and E in the high byte: exact while
// h0 + max(mat) * qlen <= 255, which bounds every H and E the recurrence produces.  Other
// jobs go to an overflow list that the int32 kernel runs next.  Query codes are stored as
// PRMT selector bytes; the score is byte (t XOR q) of the table [a, -b, -b, -b, n, n, n, n]
// with the sign replicated into the high byte, so the kernel serves bwa-form matrices
// (ext_pair_eligible): a on the diagonal, -b off it, n (0 or -1) for N.
//
// Row i+1's band follows from row i's final words: its first column is row i's first
// non-zero word (found while the first steps run), its end from row i's last positive H
// (tracked every step).  Until row i has ended the high half runs on; cells past row i+1's
// true end see only zero inputs, so their H is row i+1's decaying F (below its row max,
// never a first argmax) and their E is zero, and their words are cleared after the pair,
// which leaves shared memory as the one-row recurrence leaves it on every column a later
// row can read.

#include "fa_cert.cuh"
#include "fa_device.cuh"
#include "fa_kernels.h"
#include "fa_packed.cuh"

namespace fa {

namespace {

// PRMT, generic mode (byte select, nibble bit 3 replicates the selected byte's sign); the
// host branch states those semantics so the thread body also runs on the CPU (tests).
__host__ __device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
#else
    const uint64_t src = (uint64_t)b << 32 | a;
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

__host__ __device__ __forceinline__ void or_status(uint32_t *st, uint32_t v) {
#ifdef __CUDA_ARCH__
    atomicOr(st, v);
#else
    *st |= v;
#endif
}

__host__ __device__ __forceinline__ uint32_t take_slot(uint32_t *cnt) {
#ifdef __CUDA_ARCH__
    return atomicAdd(cnt, 1u);
#else
    return (*cnt)++;
#endif
}

__host__ __device__ __forceinline__ uint32_t mulhi(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ inline uint32_t dup16(int v) { return (uint32_t)(v & 0xFFFF) * 0x10001u; }

}  // namespace


// One job.  eh[slot(c) * T]: the column word of column c (H | E << 8); with RING = R > 0 only
// R slots, column c in slot c mod R, for bands with 2w + 3 <= R (a row pair touches at most
// 2w + 3 consecutive columns, so a slot is never reused while a later step can read it).
// sb[c * T]: the selector byte of query column c.  SYM: o_del + e_del == o_ins + e_ins and
// e_del == e_ins, so E and F open from one shared term.  CERT: also evaluates the exit-bound
// certificate (flags bit 1) and its band hint (bits 2-7) exactly as the int32 kernel does.
// Returns the cells the recurrence evaluated.
// PK: the sequences are 2-bit packed (SeqBuf.packed), read 16 bases per word load.
template <int T, bool SYM, bool CERT, int RING, bool PK = false>
__host__ __device__ __forceinline__ uint32_t rows2_thread(
    uint32_t jid, uint16_t *__restrict__ eh, uint8_t *__restrict__ sb, const fa_job *__restrict__ jobs,
    const SeqBuf &qs, const SeqBuf &ts, const ExtParams &p, int qcap,
    const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out, uint8_t *__restrict__ clamped_out,
    uint32_t *__restrict__ cells_job, uint32_t *__restrict__ status, uint32_t *__restrict__ ovf,
    uint32_t *__restrict__ ovf_n)
{
    const fa_job jb = jobs[jid];
    const int qlen = jb.qlen, tlen = jb.tlen, h0 = jb.h0;
    const int a = p.max_score;
    if (h0 < 0 || (h0 == 0 && !(p.flags & FA_PARAM_H0_ZERO)) || qlen <= 0 || tlen < 0) {
        or_status(status, ST_ARG);
        return 0;
    }
    if (qlen > qcap) {
        or_status(status, ST_CAPACITY);
        return 0;
    }
    if (h0 == 0) {   // FA_PARAM_H0_ZERO: the recurrence as written is all zero after row 0
        const int w0 = ext_band_clamp(qlen, w_try ? w_try[jid] : jb.w, p);
        fa_ext_result r;
        const uint32_t c = ext_h0_zero_result(qlen, tlen, w0, &r);
        out[jid] = r;
        if (clamped_out)
            clamped_out[jid] = (uint8_t)((tlen > 0 && qlen > w0 + 1 ? 1 : 0) | (CERT ? kBandHintNone << 2 : 0));
        if (cells_job) cells_job[jid] = c;
        return c;
    }
    if (h0 > 255 || a * qlen > 255 - h0) {
        // needs wider cells: the int32 kernel (ovf null: the job was listed before the launch)
        if (ovf) ovf[take_slot(ovf_n)] = jid;
        return 0;
    }
    const int w = ext_band_clamp(qlen, w_try ? w_try[jid] : jb.w, p);
    if (RING > 0 && 2 * w + 3 > RING) {
        or_status(status, ST_CAPACITY);
        return 0;
    }
    uint32_t cells = 0;
    const int oe_del = p.o_del + p.e_del, oe_ins = p.o_ins + p.e_ins;
    const int e_del = p.e_del, e_ins = p.e_ins;
    const uint32_t NOED = dup16(-oe_del), NED = dup16(-e_del), NOEI = dup16(-oe_ins), NEI = dup16(-e_ins);
    const uint32_t TAB = (uint32_t)(uint8_t)p.mat[0] | (uint32_t)(uint8_t)p.mat[1] * 0x01010100u;
    const uint32_t TABN = (uint32_t)(uint8_t)p.mat[4] * 0x01010101u;
    const uint32_t kmul = a <= 1 ? 2u : 4u;   // kmul * M >= M + a for every M >= 1
    // selector nibble of a query N: lands on bytes 4-7 (n) for t < 4 and, for a target N, on
    // a byte whose sign is n's (n = -1: -b; n = 0: a)
    const uint32_t qn = p.mat[4] < 0 ? 13u : 12u;
    const uint8_t *Q = qs.p + jb.q_off;    // byte codes (PK false)
    const uint8_t *Tg = ts.p + jb.t_off;
    PackedReader qr, tr;                    // packed bases (PK true)
    if (PK) {
        qr.init(qs, jb.q_off, qlen);
        tr.init(ts, jb.t_off, tlen);
    }
    auto slot = [](int c) { return RING > 0 ? (c & (RING - 1)) : c; };
    // first row (ksw_affine_gap.rs:1017-1025): h0, h0-oe_ins, then -e_ins while the previous
    // value exceeds e_ins, so positive exactly up to init_reach; E = 0
    const int init_reach = h0 <= oe_ins ? 0 : (e_ins == 0 ? qlen : min(qlen, 1 + (h0 - oe_ins - 1) / e_ins));
    auto init_h = [&](int c) { return c == 0 ? h0 : (c <= init_reach ? h0 - oe_ins - (c - 1) * e_ins : 0); };

    uint32_t bad = 0;
    for (int j0 = 0; j0 < qlen; j0 += 16) {
        uint32_t qb[16];
        if (PK) {
            uint32_t v[4];
            qr.getw<4>(j0, v);
#pragma unroll
            for (int u = 0; u < 16; ++u) qb[u] = (v[u / 4] >> (8 * (u & 3))) & 0xFFu;
        } else {
#pragma unroll
            for (int u = 0; u < 16; ++u) qb[u] = j0 + u < qlen ? (uint32_t)Q[j0 + u] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            if (j0 + u < qlen) {
                bad |= qb[u] >= (uint32_t)p.m;
                sb[(j0 + u) * T] = (uint8_t)(qb[u] < 4u ? qb[u] * 0x11u + 0x80u : qn * 0x11u);
            }
        }
    }
    for (int c = 0; c <= qlen && (RING == 0 || c < RING); ++c) eh[slot(c) * T] = (uint16_t)init_h(c);
    auto score1 = [&](uint32_t t, int c) -> int {   // one cell of row t at column c
        return (int)(int16_t)(prmt(TAB, TABN, (uint32_t)sb[c * T] ^ (t * 0x11u)) & 0xFFFFu);
    };

    // pair state, int16x2: low half row i, high half row i+1 (one column behind); sprev:
    // the previous step's selector byte (the high half's query column)
    uint32_t hpp = 0, hp = 0, ep = 0, f2 = 0, km = 0, lpk = 0, tsel = 0, sprev = 0;
    // One step: low half column j, high half column j-1, from wd = eh[j] and sbj = sb[j].  ow =
    // row i+1's word for column j-1.  key = H << 8 | ck: the row max with its first column (ck
    // counts down with the column); lpv = min(H << 8 + kk, 256 + kk): 256 + kk where the low
    // row's H > 0 (its last such column).  Unpacking and the selector pair are multiply-adds,
    // so they issue beside the DPX work.
    auto core = [&](uint32_t wd, uint32_t sbj, uint32_t ck, uint32_t kk, uint32_t kk256, uint32_t &key,
                    uint32_t &lpv, uint32_t &ow) {
        const uint32_t E = mulhi(wd, 1u << 24);                   // row i-1's E byte
        const uint32_t M2 = (hpp * 65536u + wd) - E * 256u;       // (H at j-1, row i's H at j-2)
        const uint32_t e2 = ep * 65536u + E;                      // (E at j, row i's E for j-1)
        const uint32_t qsel = sprev * 256u + sbj;
        sprev = sbj;
        const uint32_t s2 = prmt(TAB, TABN, qsel ^ tsel);
        // ksw_extend2's `M ? M + s : 0`: for M > 0, kmul * M >= M + s; for M == 0 the result
        // is <= 0, which acts as 0 in every max below (halves stay apart: 4 * 255 < 2^15)
        const uint32_t Mp = __viaddmin_s16x2(M2, s2, M2 * kmul);
        const uint32_t h2 = __vimax3_s16x2(Mp, e2, f2);
        uint32_t en2;
        if (SYM) {
            const uint32_t t = __viaddmax_s16x2_relu(Mp, NOED, 0u);
            en2 = __viaddmax_s16x2(e2, NED, t);
            f2 = __viaddmax_s16x2(f2, NED, t);
        } else {
            en2 = __viaddmax_s16x2(e2, NED, __viaddmax_s16x2_relu(Mp, NOED, 0u));
            f2 = __viaddmax_s16x2(f2, NEI, __viaddmax_s16x2_relu(Mp, NOEI, 0u));
        }
        key = h2 * 256u + ck;
        lpv = __viaddmin_u16x2(h2 * 256u, kk, kk256);
        ow = prmt(hp, en2, 0x62u);                                // (H of row i+1 at j-2, its E for j-1)
        hpp = hp;
        hp = h2;
        ep = en2;
    };
    // a single step at column j, folded into km / lpk at once
    auto step1 = [&](int j, uint32_t &ow) {
        uint32_t key, lpv;
        core((uint32_t)eh[slot(j) * T], (uint32_t)sb[j * T], 0u, 0u, 256u, key, lpv, ow);
        km = __viaddmax_u16x2(key, (uint32_t)(255 - j) | (uint32_t)((256 - j) & 0xFFFF) << 16, km);
        lpk = __viaddmax_u16x2(lpv, (uint32_t)j, lpk);
    };

    int best = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, max_off = 0;
    int beg = 0, end = qlen, clamped = 0;
    // last row's end and the largest end so far: stale columns of the ring and the certificate
    int prev_end = 0, max_written = -1;
    // a column past every row end written so far: 0 once written (trimmed cells are zero), its
    // first-row value if never (the full array holds exactly that)
    auto stale_word = [&](int c) -> uint32_t {
        if (RING == 0 || c <= prev_end) return (uint32_t)eh[slot(c) * T];
        return c > max_written ? (uint32_t)init_h(c) : 0u;
    };
    // certificate state (CERT): exits of rows up to the current one in xb, row i+1's left
    // exits met while row i runs in xh until row i has been judged
    ExitBound xb, xh;
    int bmax = ExitBound::NEG, first_fail = INT32_MAX, rows = 0, srun = 0, sev = 0, slast = 0;
    bool row_ok = true, stale = false, broke = false, zbreak = false;
    if (CERT) xb.init();
    auto cert_row = [&](int r, int m, int e, int fexit) {   // row r judged, after its gscore update
        if (e < qlen) xb.add(0, fexit, r, e, qlen, a, e_del);             // F past the row's end
        const int b = xb.at(r, a, e_del);
        row_ok = m > 0 ? b < m : b <= 0;
        if (!row_ok && first_fail == INT32_MAX) first_fail = r;
        slast = row_ok ? 0 : b - m + 1;
        srun = max(srun, slast);
        if (max_ie == r) sev = srun;
        bmax = max(bmax, b);
    };
    // row-end rules of ksw_extend2 for row r with max m at column mj: 0 go on, 1 zero row,
    // 2 z-drop
    auto row_end = [&](int r, int m, int mj) -> int {
        if (m == 0) return 1;
        if (m > best) {
            best = m; max_i = r; max_j = mj;
            if (CERT) sev = srun;
            const int off = mj > r ? mj - r : r - mj;
            if (max_off < off) max_off = off;
        } else if (p.zdrop > 0) {
            const int di = r - max_i, dj = mj - max_j;
            if (di > dj) {
                if (best - m - (di - dj) * e_del > p.zdrop) return 2;
            } else if (best - m - (dj - di) * e_ins > p.zdrop) {
                return 2;
            }
        }
        return 0;
    };
    // target bases: tq0 holds the current four rows, tq1 the next four
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
    for (int i = 0; i < tlen; i += 2) {
        const bool two = i + 1 < tlen;
        const uint32_t t0 = tq0 & 0xFFu, t1 = two ? (tq0 >> 8) & 0xFFu : 0u;
        tq0 >>= 16;
        if ((i & 3) == 2) {
            tq0 = tq1;
            tq1 = 0;
            if (PK) {
                tq1 = tstream.next4(tr);   // positions i + 6 .. i + 9
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (i + 6 + k < tlen) tq1 |= (uint32_t)Tg[i + 6 + k] << (8 * k);
            }
        }
        if (t0 >= (uint32_t)p.m || t1 >= (uint32_t)p.m) { bad = 1; break; }
        tsel = t0 * 0x11u | t1 * 0x1100u;

        // ---- row i: band
        const int beg_a = beg;
        {
            const int end_a = end < qlen ? end : qlen;
            if (beg < i - w) beg = i - w;
            if (end > i + w + 1) end = i + w + 1;
            if (end > qlen) end = qlen;
            clamped |= (beg != beg_a) | (end != end_a);
        }
        const int b0 = beg, e0 = end;
        if (RING > 0 && i > 0 && e0 > prev_end + 1) {
            // the column the row grows into past the last row's end
            const int c = prev_end + 1;
            eh[slot(c) * T] = (uint16_t)(c > max_written ? init_h(c) : 0);
        }
        if (CERT) {
            ++rows;
            if (i == 0) {
                if (e0 < qlen) xb.add(0, init_h(e0), -1, e0 - 1, qlen, a, e_del);   // first row past the band
            } else {
                for (int j = beg_a; j < b0 && j < qlen; ++j)                       // columns the band drops
                    xb.add(1, (int)(stale_word(j) >> 8), i, j, qlen, a, e_del);
                if (beg_a == 0 && b0 > 0) xb.add(1, h0 - (p.o_del + e_del * i), i - 1, -1, qlen, a, e_del);
                stale |= max(b0, max_written + 1) <= min(e0 - 1, init_reach);     // a never-written column
            }
            xh.init();
        }
        const int h1lo = b0 == 0 ? max(h0 - (p.o_del + e_del * (i + 1)), 0) : 0;
        hpp = 0; hp = (uint32_t)h1lo; ep = 0; f2 = 0; km = 0; lpk = 0;
        sprev = b0 > 0 ? (uint32_t)sb[(b0 - 1) * T] : 0u;

        // ---- phase A: row i alone until row i+1's first column is known (for the last row of
        // an odd count the high half just runs along, unread).  A loop condition rather than a
        // break, so the warp's threads reconverge after it (the break form ran 1.8x slower:
        // threads in different phases interleaved).
        int j = b0, hs_trim = -1, c0 = -1;
        uint32_t ow;
        bool go = j < e0;
        while (go) {
            const uint32_t hprev = hp;
            step1(j, ow);
            // row i's word for column j: (its H at j-1, its E for j)
            if (hs_trim < 0 && ((hprev | ep) & 0xFFFFu)) hs_trim = j;
            // columns row i+1's band drops on the left: their E is row i's E for them
            if (CERT && j < i + 1 - w) xh.add(1, (int)(ep & 0xFFFFu), i + 1, j, qlen, a, e_del);
            const bool start = !two || (hs_trim >= 0 && j >= i + 1 - w);
            c0 = start ? j : c0;
            ++j;
            go = !start && j < e0;
        }
        if (c0 >= 0) {
            const int h1hi = c0 == 0 ? max(h0 - (p.o_del + e_del * (i + 2)), 0) : 0;
            hp = (hp & 0xFFFFu) | (uint32_t)h1hi << 16;
            f2 &= 0xFFFFu;
            km &= 0xFFFFu;
            // ---- phase B: both rows, eight steps a group (then one of four); row i+1's word
            // for column j-1 stored each step.  Group keys carry (size-1-k) and k and are
            // folded with the group's first column.
            for (; j + 7 < e0; j += 8) {
                uint32_t wv[8], sv[8], kv[8], lv[8], ov[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    wv[k] = eh[slot(j + k) * T];
                    sv[k] = sb[(j + k) * T];
                }
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    core(wv[k], sv[k], (uint32_t)(7 - k) * 0x10001u, (uint32_t)k, 256u + k, kv[k], lv[k], ov[k]);
#pragma unroll
                for (int k = 0; k < 8; ++k) eh[slot(j - 1 + k) * T] = (uint16_t)ov[k];
                const uint32_t kb8 = (uint32_t)(248 - j) | (uint32_t)((249 - j) & 0xFFFF) << 16;
                const uint32_t kg = __vimax3_u16x2(__vimax3_u16x2(kv[0], kv[1], kv[2]),
                                                   __vimax3_u16x2(kv[3], kv[4], kv[5]),
                                                   __vimax3_u16x2(kv[6], kv[7], kv[7]));
                const uint32_t lg = __vimax3_u16x2(__vimax3_u16x2(lv[0], lv[1], lv[2]),
                                                   __vimax3_u16x2(lv[3], lv[4], lv[5]),
                                                   __vimax3_u16x2(lv[6], lv[7], lv[7]));
                km = __viaddmax_u16x2(kg, kb8, km);
                lpk = __viaddmax_u16x2(lg, (uint32_t)j, lpk);
            }
            if (j + 3 < e0) {
                const uint32_t kb = (uint32_t)(252 - j) | (uint32_t)((253 - j) & 0xFFFF) << 16;
                uint32_t wv[4], sv[4], kv[4], lv[4], ov[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    wv[k] = eh[slot(j + k) * T];
                    sv[k] = sb[(j + k) * T];
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    core(wv[k], sv[k], (uint32_t)(3 - k) * 0x10001u, (uint32_t)k, 256u + k, kv[k], lv[k], ov[k]);
#pragma unroll
                for (int k = 0; k < 4; ++k) eh[slot(j - 1 + k) * T] = (uint16_t)ov[k];
                km = __viaddmax_u16x2(__viaddmax_u16x2(kv[3], 0u, __vimax3_u16x2(kv[0], kv[1], kv[2])), kb, km);
                lpk = __viaddmax_u16x2(__viaddmax_u16x2(lv[3], 0u, __vimax3_u16x2(lv[0], lv[1], lv[2])),
                                       (uint32_t)j, lpk);
                j += 4;
            }
            while (j < e0) {
                step1(j, ow);
                eh[slot(j - 1) * T] = (uint16_t)ow;
                ++j;
            }
        }

        // ---- row i ends (hp's low half: H at e0-1, or the row's h1 when empty; f2's low
        // half: F past the row's last column)
        const int hlast = (int)(hp & 0xFFFFu);
        if (e0 > b0) cells += e0 - b0;
        if (e0 == qlen && gscore < hlast) { gscore = hlast; max_ie = i; }
        const int m_lo = (int)((km & 0xFFFFu) >> 8);
        if (CERT) cert_row(i, m_lo, e0, (int)(f2 & 0xFFFFu));
        const int st_lo = row_end(i, m_lo, 255 - (int)(km & 0xFFu));
        if (st_lo) {
            broke = true;
            zbreak = st_lo == 2;
            break;
        }
        // the stale word past row i's end, before anything of this pair can change it
        const uint32_t past = two && e0 + 1 <= qlen ? stale_word(e0 + 1) : 0u;
        max_written = max(max_written, e0);
        if (!two) break;

        // ---- row i+1: band from row i's words
        const int lp = (int)(lpk & 0xFFFFu) - 256;   // row i's last column with H > 0
        const int b1a = hs_trim >= 0 ? hs_trim : e0;
        const int e1a = lp + 3 < qlen ? lp + 3 : qlen;
        int b1 = b1a, e1 = e1a;
        if (b1 < i + 1 - w) b1 = i + 1 - w;
        if (e1 > i + w + 2) e1 = i + w + 2;
        clamped |= (b1 != b1a) | (e1 != e1a);
        if (CERT) {
            ++rows;
            for (int c = max(e0 + 1, b1a); c < b1 && c < qlen; ++c)   // dropped columns past row i's end
                xh.add(1, (int)((c == e0 + 1 ? past : stale_word(c)) >> 8), i + 1, c, qlen, a, e_del);
            if (b1a == 0 && b1 > 0) xh.add(1, h0 - (p.o_del + e_del * (i + 1)), i, -1, qlen, a, e_del);
            xb.merge(xh);
            stale |= max(b1, max_written + 1) <= min(e1 - 1, init_reach);
        }
        int h1h, fh, kh;
        if (c0 >= 0) {
            h1h = (int)(hp >> 16); fh = (int)(f2 >> 16); kh = (int)(km >> 16);
        } else {
            h1h = b1 == 0 ? max(h0 - (p.o_del + e_del * (i + 2)), 0) : 0; fh = 0; kh = 0;
        }
        if (c0 >= 0 && e1 <= e0 - 1) {
            // row i+1 already ran past its end: its word at e1 holds (H at e1-1, 0) unless e1
            // is the column the last step did not reach.  Column e1-1 had zero inputs (row i
            // has no positive H past e1-3), so its H is its F, and F past the end is that less
            // one gap extension.
            if (e1 == e0 - 1) eh[slot(e1) * T] = (uint16_t)h1h;
            fh = max((int)(eh[slot(e1) * T] & 0xFFu) - e_ins, 0);
        } else {
            // ---- phase C: row i+1's columns from max(c0, e0-1) on, one at a time
            for (int c = c0 >= 0 ? e0 - 1 : b1; c < e1; ++c) {
                int M, e;
                if (c < e0) { M = (int)(hpp & 0xFFFFu); e = (int)(ep & 0xFFFFu); }   // c == e0-1
                else if (c == e0) { M = (int)(hp & 0xFFFFu); e = 0; }               // row i's end word
                else { M = (int)(past & 0xFFu); e = (int)(past >> 8); }             // c == e0+1
                const int s = score1(t1, c);
                const int Mp = M ? M + s : 0;
                const int h = max(max(Mp, e), fh);
                const int en = max(max(e - e_del, Mp - oe_del), 0);
                fh = max(max(fh - e_ins, Mp - oe_ins), 0);
                kh = max(kh, h << 8 | (255 - c));
                eh[slot(c) * T] = (uint16_t)(h1h | en << 8);
                h1h = h;
            }
            eh[slot(e1) * T] = (uint16_t)h1h;
        }
        for (int c = e1 + 1; c <= e0; ++c) eh[slot(c) * T] = 0;   // row i's zero words
        if (e1 > b1) cells += e1 - b1;
        if (e1 == qlen && gscore < h1h) { gscore = h1h; max_ie = i + 1; }
        if (CERT) cert_row(i + 1, kh >> 8, e1, fh);
        max_written = max(max_written, e1);
        prev_end = e1;
        const int st_hi = row_end(i + 1, kh >> 8, 255 - (kh & 0xFF));
        if (st_hi) {
            broke = true;
            zbreak = st_hi == 2;
            break;
        }
        // rescans for the next pair (ksw_affine_gap.rs:1155-1166) on row i+1's words
        int nb = b1;
        while (nb < e1 && eh[slot(nb) * T] == 0) ++nb;
        beg = nb;
        int ne = e1;
        while (ne > beg && eh[slot(ne) * T] == 0) --ne;
        end = ne + 2 < qlen ? ne + 2 : qlen;
    }
    if (bad) or_status(status, ST_BAD_CODE);
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
        // after a zero row every live path has left the region: a wider run's remaining rows
        // are bounded by the tents over [last row, tlen-1]
        const int fut = (broke && !zbreak) ? xb.max_over(rows - 1, tlen - 1, a, e_del) : ExitBound::NEG;
        const bool tail_ok = !broke || (zbreak ? row_ok : fut < lim);
        const int W = ext_band_clamp(qlen, jb.w, p);
        const bool wide_clean = init_reach <= min(W + 1, qlen);
        const bool cert = !stale && gscore > 0 && first_fail > i_ev && tail_ok && bmax < lim && wide_clean;
        flags |= (uint8_t)cert << 1;
        // bits 2-7: extra band columns the certificate's shortfall asks for (63: none)
        int slack = sev;
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
    return cells;
}

template <int TPB, bool SYM, bool CERT, int RING, bool PK>
__global__ void __launch_bounds__(TPB)
ext_rows2_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ order, uint32_t n,
                 const uint32_t *__restrict__ first_dev, const uint32_t *__restrict__ n_dev,
                 const SeqBuf qs, const SeqBuf ts, const ExtParams p, int qcap,
                 const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out,
                 uint8_t *__restrict__ clamped_out, uint32_t *__restrict__ cells_job,
                 unsigned long long *__restrict__ cells_out, uint32_t *__restrict__ status,
                 uint32_t *__restrict__ ovf, uint32_t *__restrict__ ovf_n)
{
    extern __shared__ uint32_t smem[];
    const uint32_t first = first_dev ? *first_dev : 0u;   // device-side sub-range of the order
    const uint32_t gi = first + blockIdx.x * TPB + threadIdx.x;
    uint32_t cells = 0;
    if (n_dev) n = min(n, *n_dev);
    if (gi < n) {
        constexpr int slots = RING > 0 ? RING : 0;
        const int words = slots > 0 ? slots : qcap + 1;
        // Per-thread slots within a column: the 32 lanes of a warp get 32 different 32-bit
        // words of every column (two warps share a word of 16-bit column words, four a word
        // of selector bytes at 128 threads per block), so lanes at different columns never
        // meet in one bank; the column stride stays TPB entries.
        static_assert(TPB == 64 || TPB == 128, "the slot maps cover 64 or 128 threads per block");
        const int t = threadIdx.x;
        const int e_off = 2 * (((t >> 6) << 5) + (t & 31)) + ((t >> 5) & 1);
        const int s_off = TPB >= 128 ? 4 * (((t >> 7) << 5) + (t & 31)) + ((t >> 5) & 3)
                                     : 4 * ((t & 31) >> 1) + 2 * (t & 1) + ((t >> 5) & 1);
        uint16_t *eh = reinterpret_cast<uint16_t *>(smem) + e_off;
        uint8_t *sb = reinterpret_cast<uint8_t *>(smem) + (size_t)words * TPB * 2 + s_off;
        cells = rows2_thread<TPB, SYM, CERT, RING, PK>(order ? order[gi] : gi, eh, sb, jobs, qs, ts, p, qcap, w_try,
                                                       out, clamped_out, cells_job, status, ovf, ovf_n);
    }
    if (cells_out) {
        unsigned long long c = cells;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(cells_out, c);
    }
}

// Persistent form of the plain kernel: as many blocks as stay resident, each warp taking
// the next 32 jobs of the (longest-first) order from a device counter until none are left,
// so the batch runs as one launch without a tail of partly filled last waves and SMs that
// finish their share early take over the rest.  The claim is warp-uniform (lane 0 takes it,
// a shuffle hands it round), so the warp's lanes stay together between jobs.
template <int TPB, bool SYM, bool CERT, int RING, bool PK>
__global__ void __launch_bounds__(TPB, 1)
ext_rows2_persist_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ order, uint32_t n,
                         const uint32_t *__restrict__ first_dev, const uint32_t *__restrict__ n_dev,
                         uint32_t *__restrict__ work, const SeqBuf qs, const SeqBuf ts, const ExtParams p,
                         int qcap,
                         const int32_t *__restrict__ w_try, fa_ext_result *__restrict__ out,
                         uint8_t *__restrict__ clamped_out, uint32_t *__restrict__ cells_job,
                         unsigned long long *__restrict__ cells_out, uint32_t *__restrict__ status,
                         uint32_t *__restrict__ ovf, uint32_t *__restrict__ ovf_n)
{
    extern __shared__ uint32_t smem[];
    const uint32_t first = first_dev ? *first_dev : 0u;   // device-side sub-range of the order
    if (n_dev) n = min(n, *n_dev);
    const uint32_t count = n > first ? n - first : 0u;
    const int t = threadIdx.x, lane = t & 31;
    const int words = RING > 0 ? RING : qcap + 1;
    static_assert(TPB == 64 || TPB == 128, "the slot maps cover 64 or 128 threads per block");
    const int e_off = 2 * (((t >> 6) << 5) + (t & 31)) + ((t >> 5) & 1);
    const int s_off = TPB >= 128 ? 4 * (((t >> 7) << 5) + (t & 31)) + ((t >> 5) & 3)
                                 : 4 * ((t & 31) >> 1) + 2 * (t & 1) + ((t >> 5) & 1);
    uint16_t *eh = reinterpret_cast<uint16_t *>(smem) + e_off;
    uint8_t *sb = reinterpret_cast<uint8_t *>(smem) + (size_t)words * TPB * 2 + s_off;
    uint32_t cells = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(work, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t k = base + lane;
        if (k < count) {
            const uint32_t gi = first + k;
            cells += rows2_thread<TPB, SYM, CERT, RING, PK>(order ? order[gi] : gi, eh, sb, jobs, qs, ts, p, qcap,
                                                        w_try, out, clamped_out, cells_job, status, ovf, ovf_n);
        }
    }
    if (cells_out) {
        unsigned long long c = cells;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0 && c) atomicAdd(cells_out, c);
    }
}

// True for the jobs rows2_thread hands on to the int32 kernel: the ones that pass its argument
// and capacity checks with h0 >= 1 (h0 == 0 has its closed form) and whose h0 + a * qlen can
// pass 255 (a = the largest matrix score).
__host__ __device__ __forceinline__ bool rows2_int32_job(const fa_job &jb, int qcap, int a) {
    if (jb.h0 < 1 || jb.qlen <= 0 || jb.tlen < 0 || jb.qlen > qcap) return false;
    return jb.h0 > 255 || a * jb.qlen > 255 - jb.h0;
}

// The jobs of order[first .. n) that rows2_thread hands on to the int32 kernel, listed before
// the two-row launch so their int32 pass can start at once; the two-row launch then runs with
// a null list and skips them.  Same sub-range rules as the two-row kernels (first_dev, n_dev).
__global__ void rows2_ovf_list_kernel(const fa_job *__restrict__ jobs, const uint32_t *__restrict__ order,
                                      uint32_t n, const uint32_t *__restrict__ first_dev,
                                      const uint32_t *__restrict__ n_dev, int qcap, int a,
                                      uint32_t *__restrict__ ovf, uint32_t *__restrict__ ovf_n)
{
    const uint32_t first = first_dev ? *first_dev : 0u;
    if (n_dev) n = min(n, *n_dev);
    for (uint32_t gi = first + blockIdx.x * blockDim.x + threadIdx.x; gi < n; gi += gridDim.x * blockDim.x) {
        const uint32_t jid = order ? order[gi] : gi;
        if (rows2_int32_job(jobs[jid], qcap, a)) ovf[atomicAdd(ovf_n, 1u)] = jid;
    }
}

bool ext_rows2_sym(const ExtParams &p) {
    return p.o_del + p.e_del == p.o_ins + p.e_ins && p.e_del == p.e_ins;
}

size_t ext_rows2_smem_bytes(int qcap, int tpb, int ring) {
    const size_t words = ring > 0 ? (size_t)ring : (size_t)qcap + 1;
    return words * tpb * sizeof(uint16_t) + (size_t)(qcap + 3) / 4 * 4 * tpb;
}

// Any capacity whose shared memory fits: jobs past kRows2MaxQ columns always exceed the 8-bit
// bound and go to the int32 kernel through the overflow list.
bool ext_rows2_eligible(const ExtParams &p, int qcap) {
    return qcap >= 1 && qcap <= FA_MAX_QLEN && ext_pair_eligible(p);
}

namespace {
template <int TPB, bool SYM, bool CERT, int RING, bool PK>
cudaError_t launch_rows2_variant(size_t smem, cudaStream_t stream, const fa_job *d_jobs, const uint32_t *d_order,
                                 uint32_t n, const uint32_t *d_first, const uint32_t *d_n, const SeqBuf &d_qseq,
                                 const SeqBuf &d_tseq, const ExtParams &p, int qcap, const int32_t *d_w_try,
                                 fa_ext_result *d_out, uint8_t *d_clamped, uint32_t *d_cells_job,
                                 unsigned long long *d_cells, uint32_t *d_status, uint32_t *d_ovf, uint32_t *d_ovf_n)
{
    cudaError_t err = cudaFuncSetAttribute(ext_rows2_kernel<TPB, SYM, CERT, RING, PK>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const uint32_t blocks = (n + TPB - 1) / TPB;
    ext_rows2_kernel<TPB, SYM, CERT, RING, PK><<<blocks, TPB, smem, stream>>>(
        d_jobs, d_order, n, d_first, d_n, d_qseq, d_tseq, p, qcap, d_w_try, d_out, d_clamped, d_cells_job, d_cells,
        d_status, d_ovf, d_ovf_n);
    return cudaGetLastError();
}
}  // namespace

namespace {
template <bool PK>
cudaError_t launch_rows2_seq(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n, const uint32_t *d_first,
                             const uint32_t *d_n, const SeqBuf &d_qseq, const SeqBuf &d_tseq, const ExtParams &p,
                             int qcap, int ring, bool cert, const int32_t *d_w_try, fa_ext_result *d_out,
                             uint8_t *d_clamped, uint32_t *d_cells_job, unsigned long long *d_cells,
                             uint32_t *d_status, uint32_t *d_ovf, uint32_t *d_ovf_n, cudaStream_t stream, int tpb,
                             uint32_t *d_work, cudaStream_t ovf_stream, cudaEvent_t ovf_ev, bool ovf_early)
{
    if (n == 0) return cudaSuccess;
    if (!ext_rows2_eligible(p, qcap) || !d_ovf || !d_ovf_n) return cudaErrorInvalidValue;
    if (ring != 0 && ring != 32 && ring != 64) return cudaErrorInvalidValue;
    const bool c = cert && d_clamped;
    cudaError_t err = cudaMemsetAsync(d_ovf_n, 0, sizeof(uint32_t), stream);
    if (err != cudaSuccess) return err;
    // the certificate and ring variants run 64 threads per block; the plain one 64 or 128
    const int t = (c || ring != 0) ? 64 : (tpb == 128 ? 128 : 64);
    const size_t smem = ext_rows2_smem_bytes(qcap, t, ring);
    const bool sym = ext_rows2_sym(p);
    // early: the overflow jobs are listed first and their int32 pass starts on the side
    // stream before the two-row launch, which then skips them (a null list)
    uint32_t *const d_ovf_all = d_ovf;
    if (ovf_stream && ovf_early) {
        int dev = 0, sms = 0;
        if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
        if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
        const uint32_t blocks = std::min<uint32_t>((n + 255) / 256, (uint32_t)sms * 8);
        rows2_ovf_list_kernel<<<blocks, 256, 0, stream>>>(d_jobs, d_order, n, d_first, d_n, qcap, p.max_score, d_ovf,
                                                          d_ovf_n);
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
        if ((err = cudaEventRecord(ovf_ev, stream)) != cudaSuccess) return err;
        if ((err = cudaStreamWaitEvent(ovf_stream, ovf_ev, 0)) != cudaSuccess) return err;
        if ((err = launch_ext_packed(d_jobs, d_ovf, n, nullptr, d_ovf_n, d_qseq, d_tseq, p, qcap, ring, d_w_try, d_out,
                                     d_clamped, c, d_cells_job, d_cells, d_status, ovf_stream)) != cudaSuccess)
            return err;
        d_ovf = nullptr;
    }
#define FA_ROWS2(TV, SV, CV, RV) launch_rows2_variant<TV, SV, CV, RV, PK>(smem, stream, d_jobs, d_order, n, d_first, d_n, \
                                                                      d_qseq, d_tseq, p, qcap, d_w_try, d_out,    \
                                                                      d_clamped, d_cells_job, d_cells, d_status,  \
                                                                      d_ovf, d_ovf_n)
    // persistent: one block per resident slot, warps claiming jobs from d_work
    auto go = [&](auto kernel, int tv) -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(d_work, 0, sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
            return e;
        int per_sm = 0, dev = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, tv, smem)) != cudaSuccess) return e;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        const uint32_t want = (n + tv - 1) / tv, cap = (uint32_t)(per_sm > 0 ? per_sm : 1) * (uint32_t)sms;
        kernel<<<want < cap ? want : cap, tv, smem, stream>>>(d_jobs, d_order, n, d_first, d_n, d_work, d_qseq,
                                                            d_tseq, p, qcap, d_w_try, d_out, d_clamped, d_cells_job,
                                                            d_cells, d_status, d_ovf, d_ovf_n);
        return cudaGetLastError();
    };
#define FA_PERSIST(TV, SV, CV, RV) go(ext_rows2_persist_kernel<TV, SV, CV, RV, PK>, TV)
    if (d_work) {
        if (c) {
            if (ring == 32) err = sym ? FA_PERSIST(64, true, true, 32) : FA_PERSIST(64, false, true, 32);
            else if (ring == 64) err = sym ? FA_PERSIST(64, true, true, 64) : FA_PERSIST(64, false, true, 64);
            else err = sym ? FA_PERSIST(64, true, true, 0) : FA_PERSIST(64, false, true, 0);
        } else if (ring == 32) {
            err = sym ? FA_PERSIST(64, true, false, 32) : FA_PERSIST(64, false, false, 32);
        } else if (ring == 64) {
            err = sym ? FA_PERSIST(64, true, false, 64) : FA_PERSIST(64, false, false, 64);
        } else if (t == 128) {
            err = sym ? FA_PERSIST(128, true, false, 0) : FA_PERSIST(128, false, false, 0);
        } else {
            err = sym ? FA_PERSIST(64, true, false, 0) : FA_PERSIST(64, false, false, 0);
        }
    } else if (c) {
        if (ring == 32) err = sym ? FA_ROWS2(64, true, true, 32) : FA_ROWS2(64, false, true, 32);
        else if (ring == 64) err = sym ? FA_ROWS2(64, true, true, 64) : FA_ROWS2(64, false, true, 64);
        else err = sym ? FA_ROWS2(64, true, true, 0) : FA_ROWS2(64, false, true, 0);
    } else if (ring == 32) {
        err = sym ? FA_ROWS2(64, true, false, 32) : FA_ROWS2(64, false, false, 32);
    } else if (ring == 64) {
        err = sym ? FA_ROWS2(64, true, false, 64) : FA_ROWS2(64, false, false, 64);
    } else if (t == 128) {
        err = sym ? FA_ROWS2(128, true, false, 0) : FA_ROWS2(128, false, false, 0);
    } else {
        err = sym ? FA_ROWS2(64, true, false, 0) : FA_ROWS2(64, false, false, 0);
    }
#undef FA_ROWS2
#undef FA_PERSIST
    if (err != cudaSuccess || (ovf_stream && ovf_early)) return err;
    if (ovf_stream) {
        if ((err = cudaEventRecord(ovf_ev, stream)) != cudaSuccess) return err;
        if ((err = cudaStreamWaitEvent(ovf_stream, ovf_ev, 0)) != cudaSuccess) return err;
        stream = ovf_stream;
    }
    // jobs whose scores can pass 255: the int32 kernel over the overflow list, same settings
    return launch_ext_packed(d_jobs, d_ovf_all, n, nullptr, d_ovf_n, d_qseq, d_tseq, p, qcap, ring, d_w_try, d_out,
                             d_clamped, c, d_cells_job, d_cells, d_status, stream);
}
}  // namespace

cudaError_t launch_ext_rows2(const fa_job *d_jobs, const uint32_t *d_order, uint32_t n, const uint32_t *d_first,
                             const uint32_t *d_n, const SeqBuf &d_qseq, const SeqBuf &d_tseq, const ExtParams &p,
                             int qcap, int ring, bool cert, const int32_t *d_w_try, fa_ext_result *d_out,
                             uint8_t *d_clamped, uint32_t *d_cells_job, unsigned long long *d_cells,
                             uint32_t *d_status, uint32_t *d_ovf, uint32_t *d_ovf_n, cudaStream_t stream, int tpb,
                             uint32_t *d_work, cudaStream_t ovf_stream, cudaEvent_t ovf_ev, bool ovf_early)
{
    if (ovf_stream && !ovf_ev) return cudaErrorInvalidValue;
    return d_qseq.packed
               ? launch_rows2_seq<true>(d_jobs, d_order, n, d_first, d_n, d_qseq, d_tseq, p, qcap, ring, cert, d_w_try,
                                        d_out, d_clamped, d_cells_job, d_cells, d_status, d_ovf, d_ovf_n, stream, tpb,
                                        d_work, ovf_stream, ovf_ev, ovf_early)
               : launch_rows2_seq<false>(d_jobs, d_order, n, d_first, d_n, d_qseq, d_tseq, p, qcap, ring, cert,
                                         d_w_try, d_out, d_clamped, d_cells_job, d_cells, d_status, d_ovf, d_ovf_n,
                                         stream, tpb, d_work, ovf_stream, ovf_ev, ovf_early);
}

}  // namespace fa
