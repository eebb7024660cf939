// mate_kernel.cu -- mate-rescue local Smith-Waterman (ksw_align2 semantics) on sm_100a.
//
// The reference runs ksw_align2 with its 128-bit striped engine
// (src/core/alignment/ksw_affine_gap.rs:773-861): 16 u8 lanes when KSW_XBYTE is set,
// otherwise 8 i16 lanes.  Its results depend on that striping -- E is built from the
// H values before the lazy-F correction, F is restarted at every stripe boundary and
// the lazy-F loop stops after the first pass that changes nothing, padding columns
// score 0 and take part in the row maxima, and the query end is searched over
// sign-interpreted lanes.  These kernels reproduce the striped machine exactly: a
// group of 8 GPU lanes owns one job; for i16 jobs each GPU lane holds one SIMD lane of
// the reference (stripe l: query positions j + l*slen) in registers, for u8 jobs each
// holds two (sw_pass_u8x2, 16-bit halves, DPX 16x2 instructions).  The diagonal crosses
// stripes with one shuffle per row, lazy-F passes move the F carry one SIMD lane per
// pass, and row maxima, the query-end search and the second-best scan are group
// reductions.  The forward pass and the KSW_XSTART reverse pass share the same code.

#include <algorithm>
#include <climits>

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

constexpr int kMateThreads = 128;

__device__ __forceinline__ uint32_t prmt(uint32_t lo, uint32_t hi, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return r;
}

__device__ __forceinline__ int sat16(int x) { return min(max(x, -32768), 32767); }

struct SeqView {
    const uint8_t *s;
    int rev_last;   // >= 0: positions 0..rev_last are read reversed (ksw_align2 XSTART pass)
    __device__ __forceinline__ uint32_t at(int k) const {
        return rev_last >= 0 && k <= rev_last ? s[rev_last - k] : s[k];
    }
};

// One ksw_u8_impl / ksw_i16_impl run (ksw_affine_gap.rs:267-494 / 503-735) for the job
// owned by this lane group.  All lanes of the group return the same result.
template <int P, int SMAX>
__device__ fa_kswr sw_pass(SeqView Q, int qlen, SeqView Tg, int tlen, uint32_t xtra,
                           const MateParams &p, uint32_t gmask, int l, uint32_t *blist,
                           int bcap, unsigned long long &cells, uint32_t &status)
{
    constexpr bool U8 = (P == 16);
    constexpr int NQW = (SMAX + 7) / 8;
    const int slen = (qlen + P - 1) / P;
    const int off = SMAX - slen;   // segment j lives at register index j + off
    const uint32_t minsc = (xtra & FA_KSW_XSUBO) ? (xtra & 0xffffu) : 0x10000u;
    const uint32_t endsc = (xtra & FA_KSW_XSTOP) ? (xtra & 0xffffu) : 0x10000u;
    const int oe_del = p.o_del + p.e_del, oe_ins = p.o_ins + p.e_ins;
    const int e_del = p.e_del, e_ins = p.e_ins, shift = p.shift;

    // Query codes of this stripe as nibbles; 5 marks padding (profile score 0).
    uint32_t qw[NQW];
#pragma unroll
    for (int w = 0; w < NQW; ++w) qw[w] = 0x55555555u;
    uint32_t bad = 0;
#pragma unroll
    for (int a = 0; a < SMAX; ++a) {
        if (a >= off) {
            const int k = (a - off) + l * slen;
            if (k < qlen) {
                uint32_t c = Q.at(k);
                bad |= c > 4u;
                c = c > 4u ? 4u : c;
                qw[a / 8] = (qw[a / 8] & ~(0xFu << (4 * (a % 8)))) | (c << (4 * (a % 8)));
            }
        }
    }

    int H0[SMAX], H1[SMAX], E[SMAX], Hm[SMAX];
#pragma unroll
    for (int a = 0; a < SMAX; ++a) { H0[a] = 0; H1[a] = 0; E[a] = 0; Hm[a] = 0; }

    // profile rows as PRMT tables (u8: mat + shift mod 256, padding = shift; i16: mat, padding = 0),
    // indexed only with constants
    uint32_t rlo[5], rhi[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const int sh = U8 ? shift : 0;
        rlo[t] = (uint8_t)(p.mat[t * 5] + sh) | (uint32_t)(uint8_t)(p.mat[t * 5 + 1] + sh) << 8 |
                 (uint32_t)(uint8_t)(p.mat[t * 5 + 2] + sh) << 16 |
                 (uint32_t)(uint8_t)(p.mat[t * 5 + 3] + sh) << 24;
        rhi[t] = (uint8_t)(p.mat[t * 5 + 4] + sh) | (uint32_t)(uint8_t)sh << 8;
    }

    int gmax = 0, te = -1;
    int nb = 0, last_row = -2, last_sc = 0;

    for (int i = 0; i < tlen; ++i) {
        const uint32_t tb = Tg.at(i);
        if (tb > 4u) { bad = 1; break; }
        uint32_t lo = rlo[0], hi = rhi[0];
#pragma unroll
        for (int t = 1; t < 5; ++t)
            if (tb == (uint32_t)t) { lo = rlo[t]; hi = rhi[t]; }
        cells += (unsigned long long)qlen;

        int hd = __shfl_up_sync(gmask, H0[SMAX - 1], 1, P);
        if (l == 0) hd = 0;
        int f = 0, mx = 0;
#pragma unroll
        for (int a = 0; a < SMAX; ++a) {
            if (a >= off) {
                const uint32_t c = (qw[a / 8] >> (4 * (a % 8))) & 0xFu;
                int h;
                if (U8) {
                    const int s = (int)prmt(lo, hi, c | 0x7770u);
                    h = min(hd + s, 255);
                    h = max(h - shift, 0);
                } else {
                    const int s = (int)prmt(lo, hi, c * 0x1111u + 0x8880u);
                    h = sat16(hd + s);
                }
                const int e = E[a];
                h = max(h, e);
                h = max(h, f);
                mx = max(mx, h);
                H1[a] = h;
                if (U8) {
                    E[a] = __viaddmax_s32_relu(e, -e_del, h - oe_del);
                    f = __viaddmax_s32_relu(f, -e_ins, h - oe_ins);
                } else {
                    E[a] = max(sat16(e - e_del), sat16(h - oe_del));
                    f = max(sat16(f - e_ins), sat16(h - oe_ins));
                }
                hd = H0[a];
            }
        }
        // lazy-F: one lane further per pass, stop after a pass that changed nothing
        for (int pass = 0; pass < P; ++pass) {
            f = __shfl_up_sync(gmask, f, 1, P);
            if (l == 0) f = 0;
            int changed = 0;
#pragma unroll
            for (int a = 0; a < SMAX; ++a) {
                if (a >= off) {
                    const int hb = H1[a];
                    const int hn = max(hb, f);
                    changed |= hn != hb;
                    H1[a] = hn;
                    f = U8 ? max(f - e_ins, 0) : sat16(f - e_ins);
                }
            }
            if (!__any_sync(gmask, changed)) break;
        }
        const int imax = (int)__reduce_max_sync(gmask, (unsigned)mx);
        if ((uint32_t)imax >= minsc) {
            if (nb == 0 || last_row + 1 != i) {
                if (nb < bcap) {
                    if (l == 0) blist[nb] = (uint32_t)imax << 16 | (uint32_t)i;
                } else {
                    status |= ST_BLIST;
                }
                ++nb;
                last_row = i;
                last_sc = imax;
            } else if (last_sc < imax) {
                if (l == 0 && nb - 1 < bcap) blist[nb - 1] = (uint32_t)imax << 16 | (uint32_t)i;
                last_row = i;
                last_sc = imax;
            }
        }
        if (imax > gmax) {
            gmax = imax;
            te = i;
#pragma unroll
            for (int a = 0; a < SMAX; ++a) Hm[a] = H1[a];
            const bool sat = U8 ? (gmax + shift >= 255) : (gmax >= 0x7FFF);
            if (sat || (uint32_t)gmax >= endsc) break;
        }
#pragma unroll
        for (int a = 0; a < SMAX; ++a) H0[a] = H1[a];
    }
    if (bad) status |= ST_BAD_CODE;

    fa_kswr r;
    r.score = U8 ? (gmax + shift < 255 ? gmax : 255) : gmax;
    r.te = te;
    r.qe = -1; r.score2 = -1; r.te2 = -1; r.tb = -1; r.qb = -1;
    if (r.score != (U8 ? 255 : 0x7FFF)) {
        // query end: smallest position holding the largest sign-interpreted lane value
        int bv = -1, bk = -1;
#pragma unroll
        for (int a = 0; a < SMAX; ++a) {
            if (a >= off) {
                const int k = (a - off) + l * slen;
                if (k < qlen) {
                    const int v = U8 ? (int)(int8_t)(uint8_t)Hm[a] : (int)(int16_t)Hm[a];
                    if (v > bv) { bv = v; bk = k; }
                }
            }
        }
        const int gv = __reduce_max_sync(gmask, bv);
        r.qe = __reduce_min_sync(gmask, bv == gv ? bk : INT_MAX);
        if (r.qe == INT_MAX) r.qe = -1;
        if (nb > 0) {
            __syncwarp(gmask);
            const int iv = (r.score + p.max - 1) / p.max;
            const int low = te - iv, high = te + iv;
            const int cnt = nb < bcap ? nb : bcap;
            int s2 = -1, e2 = INT_MAX;
            for (int e = l; e < cnt; e += P) {
                const uint32_t b = blist[e];
                const int row = (int)(b & 0xffffu), sc = (int)(b >> 16);
                if ((row < low || row > high) && sc > s2) { s2 = sc; e2 = e; }
            }
            const int gs2 = __reduce_max_sync(gmask, s2);
            const int ge2 = __reduce_min_sync(gmask, s2 == gs2 ? e2 : INT_MAX);
            if (gs2 >= 0 && ge2 != INT_MAX) {
                r.score2 = gs2;
                r.te2 = (int)(blist[ge2] & 0xffffu);
            }
            __syncwarp(gmask);
        }
    }
    return r;
}

// The u8 engine with two SIMD lanes per GPU lane: thread l of an 8-thread group holds
// the reference's lanes 2l (low 16 bits) and 2l+1 (high 16 bits) of every segment, so
// each DPX instruction updates two cells.  Values stay within 0..255, so the 16-bit
// halves never carry; the u8 saturations are explicit: min(hd + s, 255) as
// __viaddmin_u16x2, the -shift with a zero floor and the gap updates as
// __viaddmax_s16x2_relu.  Moving a register one lane up (the diagonal between segments,
// F between lazy-F passes) is one shuffle of the group plus one PRMT.  Same results as
// sw_pass<16, SMAX>.
__device__ __forceinline__ uint32_t lane_up_u16x2(uint32_t v, uint32_t gmask, int l) {
    uint32_t prev = __shfl_up_sync(gmask, v, 1, 8);
    if (l == 0) prev = 0;
    return prmt(v, prev, 0x1076u);   // low <- previous thread's high, high <- own low
}

// hm: this group's SMAX x 8 words of shared memory for the row snapshot at the best score
// (slot a * 8 + l), kept out of registers so more groups fit on an SM.
// rt: the block's profile rows in shared memory, rt[t] / rt[5 + t] the low / high table of
// target base t (mate_row_tables).
// REV: the KSW_XSTART reverse pass (KSW_XSTOP, no KSW_XSUBO), which keeps no run list.
// FAST: the batch's jobs satisfy (qlen + 1) * max + shift <= 255 and the two gap penalties are
// equal.  Every value is the score of an alignment of at most qlen query bases, so
// hd + (mat + shift) stays below 256 and adds_epu8 never saturates: the profile byte is the
// signed matrix entry (PRMT sign-extends it to 16 bits), one __viaddmax_s16x2_relu gives
// max(hd + mat, E, 0), and the insertion and deletion terms share one subtraction.  Same
// results as the general form.
// FULL: every job of the launch has exactly SMAX segments (no per-segment range checks).
template <int SMAX, bool REV, bool FAST, bool FULL = false>
__device__ fa_kswr sw_pass_u8x2(SeqView Q, int qlen, SeqView Tg, int tlen, uint32_t xtra, const MateParams &p,
                                uint32_t gmask, int l, uint32_t *blist, int bcap, uint32_t *hm, const uint32_t *rt,
                                unsigned long long &cells, uint32_t &status)
{
    constexpr int P = 16;                      // lanes of the reference's u8 vector
    const int slen = (qlen + P - 1) / P;
    const int off = FULL ? 0 : SMAX - slen;               // segment j lives at register index j + off
    const uint32_t minsc = (xtra & FA_KSW_XSUBO) ? (xtra & 0xffffu) : 0x10000u;
    const uint32_t endsc = (xtra & FA_KSW_XSTOP) ? (xtra & 0xffffu) : 0x10000u;
    const uint32_t shift = (uint32_t)p.shift;
    const uint32_t neg_shift2 = (uint32_t)(uint16_t)(-(int)shift) * 0x10001u;
    const uint32_t neg_oedel2 = (uint32_t)(uint16_t)(-(p.o_del + p.e_del)) * 0x10001u;
    const uint32_t neg_edel2 = (uint32_t)(uint16_t)(-p.e_del) * 0x10001u;
    const uint32_t neg_oeins2 = (uint32_t)(uint16_t)(-(p.o_ins + p.e_ins)) * 0x10001u;
    const uint32_t neg_eins2 = (uint32_t)(uint16_t)(-p.e_ins) * 0x10001u;
    const uint32_t eins2 = (uint32_t)(uint16_t)p.e_ins * 0x10001u;
    const uint32_t neg_pass2 = (uint32_t)(uint16_t)(-(slen * p.e_ins)) * 0x10001u;   // F decay over a pass
    const uint32_t cap255 = 0x00FF00FFu, neg2 = 0x80008000u;

    // PRMT selectors of both lanes' query codes per segment (byte 5 of the table pair is
    // zero: code 5 marks padding, whose profile score is `shift`, held in byte 5's place
    // by the row table below)
    uint32_t sel[SMAX];
    uint32_t bad = 0;
#pragma unroll
    for (int a = 0; a < SMAX; ++a) {
        uint32_t c2[2] = {5u, 5u};
        if (a >= off) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = (a - off) + (2 * l + h) * slen;
                if (k < qlen) {
                    uint32_t c = Q.at(k);
                    bad |= c > 4u;
                    c2[h] = c > 4u ? 4u : c;
                }
            }
        }
        // result bytes: [c_lo, zero, c_hi, zero] with the zero from byte 7 of the table, or
        // (FAST) [c_lo, sign of c_lo, c_hi, sign of c_hi]
        sel[a] = FAST ? (c2[0] | (c2[0] | 8u) << 4 | c2[1] << 8 | (c2[1] | 8u) << 12)
                      : (c2[0] | 0x70u | c2[1] << 8 | 0x7000u);
    }

    // H: the previous row until a segment is updated, then the current one (in place)
    uint32_t H[SMAX], E[SMAX];
#pragma unroll
    for (int a = 0; a < SMAX; ++a) { H[a] = 0; E[a] = 0; hm[a * 8 + l] = 0; }

    int gmax = 0, te = -1;
    int nb = 0, last_row = -2, last_sc = 0;

    int rows = tlen;   // rows computed (cell count)
    uint32_t tb_next = tlen > 0 ? Tg.at(0) : 0u;
    for (int i = 0; i < tlen; ++i) {
        const uint32_t tb = tb_next;
        if (i + 1 < tlen) tb_next = Tg.at(i + 1);   // the next row's base, in flight during this row
        if (tb > 4u) { bad = 1; rows = i; break; }
        const uint32_t lo = rt[tb], hi = rt[5 + tb];

        uint32_t hd = lane_up_u16x2(H[SMAX - 1], gmask, l);
        uint32_t f = 0;
#pragma unroll
        for (int a = 0; a < SMAX; ++a) {
            if (a >= off) {
                const uint32_t s = prmt(lo, hi, sel[a]);
                const uint32_t e = E[a];
                uint32_t h;
                if (FAST) {
                    h = __viaddmax_s16x2_relu(hd, s, e);               // max(hd + mat, E, 0)
                    h = __vimax_s16x2_relu(h, f);
                } else {
                    h = __viaddmin_u16x2(hd, s, cap255);               // adds_epu8
                    h = __viaddmax_s16x2_relu(h, neg_shift2, 0u);      // subs_epu8(., shift)
                    h = __vimax3_s16x2(h, e, f);
                }
                hd = H[a];                                             // the next segment's diagonal
                H[a] = h;
                const uint32_t tdel = __viaddmax_s16x2(h, neg_oedel2, neg2);
                E[a] = __viaddmax_s16x2_relu(e, neg_edel2, tdel);
                const uint32_t tins = FAST ? tdel : __viaddmax_s16x2(h, neg_oeins2, neg2);
                f = __viaddmax_s16x2_relu(f, neg_eins2, tins);
            }
        }
        // the row maximum before the lazy-F correction (the reference's max_epu8 in the
        // segment loop): slots below `off` still hold their initial zero
        uint32_t mx = 0;
#pragma unroll
        for (int a = 0; a < SMAX; a += 2)
            mx = a + 1 < SMAX ? __vimax3_s16x2(mx, H[a], H[a + 1]) : __vimax_s16x2_relu(mx, H[a]);
        // lazy-F (the reference's loop: F moves one lane further per pass, H = max(H, F) along
        // the segments while F decays by e_ins, and the loop stops after the first pass that
        // changes nothing), in closed form.  Within the loop F never reads H, so the value a
        // lane receives at the start of pass p, g_p, follows from the main loop's final F
        // alone: g_1 = F of the lane below, g_p = that lane's relu(g_(p-1) - slen * e_ins).
        // Segment j then sees relu(g_p - j * e_ins).  Pass p changes a lane exactly when g_p
        // exceeds both every earlier g of that lane and T - 1 = min_j(H_j + j * e_ins), so the
        // loop runs on one carried value per lane (U = max(T - 1, g_1 .. g_p), G = max of the
        // g), and H takes max(H_j, relu(G - j * e_ins)) once at the end: the same H.
        {
            // T - 1 by the backward recurrence m = min(H_j, m + e_ins)
            uint32_t u = H[SMAX - 1];
#pragma unroll
            for (int a = SMAX - 2; a >= 0; --a)
                if (a >= off) u = __viaddmin_s16x2(u, eins2, H[a]);
            uint32_t g = 0, gs = lane_up_u16x2(f, gmask, l);
            for (int pass = 0; pass < P; ++pass) {
                const uint32_t un = __vimax_s16x2_relu(u, gs);
                const uint32_t changed = un ^ u;
                u = un;
                g = __vimax_s16x2_relu(g, gs);
                if (!__any_sync(gmask, changed != 0)) break;
                gs = lane_up_u16x2(__viaddmax_s16x2_relu(gs, neg_pass2, 0u), gmask, l);
            }
            if (g != 0u) {
#pragma unroll
                for (int a = 0; a < SMAX; ++a) {
                    if (a >= off) {
                        H[a] = __vimax_s16x2_relu(H[a], g);
                        g = __viaddmax_s16x2_relu(g, neg_eins2, 0u);
                    }
                }
            }
        }
        const uint32_t mx1 = max(mx & 0xffffu, mx >> 16);
        const int imax = (int)__reduce_max_sync(gmask, mx1);
        if (!REV && (uint32_t)imax >= minsc) {
            if (nb == 0 || last_row + 1 != i) {
                if (nb < bcap) {
                    if (l == 0) blist[nb] = (uint32_t)imax << 16 | (uint32_t)i;
                } else {
                    status |= ST_BLIST;
                }
                ++nb;
                last_row = i;
                last_sc = imax;
            } else if (last_sc < imax) {
                if (l == 0 && nb - 1 < bcap) blist[nb - 1] = (uint32_t)imax << 16 | (uint32_t)i;
                last_row = i;
                last_sc = imax;
            }
        }
        if (imax > gmax) {
            gmax = imax;
            te = i;
#pragma unroll
            for (int a = 0; a < SMAX; ++a) hm[a * 8 + l] = H[a];
            if (gmax + (int)shift >= 255 || (uint32_t)gmax >= endsc) { rows = i + 1; break; }
        }
    }
    cells += (unsigned long long)rows * (unsigned)qlen;
    if (bad) status |= ST_BAD_CODE;

    fa_kswr r;
    r.score = gmax + (int)shift < 255 ? gmax : 255;
    r.te = te;
    r.qe = -1; r.score2 = -1; r.te2 = -1; r.tb = -1; r.qb = -1;
    if (r.score != 255) {
        // query end: smallest position holding the largest sign-interpreted lane value
        int bv = -1, bk = -1;
#pragma unroll
        for (int a = 0; a < SMAX; ++a) {
            if (a >= off) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = (a - off) + (2 * l + h) * slen;
                    if (k < qlen) {
                        const uint32_t w = hm[a * 8 + l];
                        const int v = (int)(int8_t)(uint8_t)(h ? (w >> 16) : (w & 0xffffu));
                        if (v > bv || (v == bv && k < bk)) { bv = v; bk = k; }
                    }
                }
            }
        }
        const int gv = __reduce_max_sync(gmask, bv);
        r.qe = __reduce_min_sync(gmask, bv == gv ? bk : INT_MAX);
        if (r.qe == INT_MAX) r.qe = -1;
        if (!REV && nb > 0) {
            __syncwarp(gmask);
            const int iv = (r.score + p.max - 1) / p.max;
            const int low = te - iv, high = te + iv;
            const int cnt = nb < bcap ? nb : bcap;
            int s2 = -1, e2 = INT_MAX;
            for (int e = l; e < cnt; e += 8) {
                const uint32_t b = blist[e];
                const int row = (int)(b & 0xffffu), sc = (int)(b >> 16);
                if ((row < low || row > high) && sc > s2) { s2 = sc; e2 = e; }
            }
            const int gs2 = __reduce_max_sync(gmask, s2);
            const int ge2 = __reduce_min_sync(gmask, s2 == gs2 ? e2 : INT_MAX);
            if (gs2 >= 0 && ge2 != INT_MAX) {
                r.score2 = gs2;
                r.te2 = (int)(blist[ge2] & 0xffffu);
            }
            __syncwarp(gmask);
        }
    }
    return r;
}

// Whether ksw_align2's KSW_XSTART reverse pass (ksw_affine_gap.rs, ksw_align2) runs for a
// forward result, and whether it can change the result.  Every value of the reverse pass is
// the score of an alignment of the reversed query prefix 0..qe, so it is at most
// (qe + 1) * max: below the forward score the pass can neither stop early (KSW_XSTOP at the
// forward score, u8 saturation above it) nor set tb / qb -- it runs all tlen rows for
// nothing, and only its cell count is kept.
__device__ __forceinline__ bool mate_needs_start(const fa_kswr &r, uint32_t xtra) {
    return (xtra & FA_KSW_XSTART) && !((xtra & FA_KSW_XSUBO) && r.score < (int)(xtra & 0xffffu)) && r.qe >= 0 &&
           r.te >= 0;
}
__device__ __forceinline__ bool mate_start_reachable(const fa_kswr &r, const MateParams &p) {
    return (r.qe + 1) * p.max >= r.score;
}

template <int P, int SMAX>
__global__ void __launch_bounds__(kMateThreads)
mate_sw_kernel(const fa_mate_job *__restrict__ jobs, const uint32_t *__restrict__ order, uint32_t n,
               const uint8_t *__restrict__ qseq, const uint8_t *__restrict__ tseq, const MateParams p,
               int bcap, fa_kswr *__restrict__ out, unsigned long long *__restrict__ cells_out,
               uint32_t *__restrict__ status)
{
    extern __shared__ uint32_t bsm[];
    const uint32_t gtid = blockIdx.x * kMateThreads + threadIdx.x;
    const uint32_t gidx = gtid / P;
    const int lane = threadIdx.x & 31;
    const int l = lane % P;
    const uint32_t gmask = (P == 32 ? 0xffffffffu : ((1u << P) - 1u)) << (lane - l);
    unsigned long long cells = 0;
    uint32_t st = 0;
    if (gidx < n) {
        const uint32_t jid = order ? order[gidx] : gidx;
        const fa_mate_job jb = jobs[jid];
        uint32_t *blist = bsm + (threadIdx.x / P) * bcap;
        SeqView Q{qseq + jb.q_off, -1}, Tg{tseq + jb.t_off, -1};
        fa_kswr r = sw_pass<P, SMAX>(Q, jb.qlen, Tg, jb.tlen, jb.xtra, p, gmask, l, blist, bcap,
                                     cells, st);
        if (mate_needs_start(r, jb.xtra) && !mate_start_reachable(r, p)) {
            cells += (unsigned long long)(r.qe + 1) * (unsigned)jb.tlen;
        } else if (mate_needs_start(r, jb.xtra)) {
            SeqView Q2{qseq + jb.q_off, r.qe}, T2{tseq + jb.t_off, r.te};
            const fa_kswr rr = sw_pass<P, SMAX>(Q2, r.qe + 1, T2, jb.tlen,
                                                FA_KSW_XSTOP | (uint32_t)r.score, p, gmask, l,
                                                blist, bcap, cells, st);
            if (rr.score >= r.score) { r.tb = r.te - rr.te; r.qb = r.qe - rr.qe; }
        }
        st = __reduce_or_sync(gmask, st);
        if (l == 0) {
            out[jid] = r;
            if (st) atomicOr(status, st);
        } else {
            cells = 0;
        }
    }
    if (cells_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, o);
        if (lane == 0 && cells) atomicAdd(cells_out, cells);
    }
}

// The profile row tables of the u8 engine in shared memory (mat + shift mod 256 for codes
// 0..4, shift for padding code 5, 0 in byte 7): rt[t] the low and rt[5 + t] the high word of
// target base t's table.  Threads 0-4 write them; the caller synchronises.
// With FAST (sw_pass_u8x2) the bytes are the signed matrix entries and padding scores 0.
template <bool FAST>
__device__ __forceinline__ void mate_row_tables(uint32_t *rt, const MateParams &p) {
    if (threadIdx.x < 5) {
        const int t = threadIdx.x;
        const uint32_t sh = FAST ? 0u : (uint32_t)p.shift;
        rt[t] = (uint8_t)(p.mat[t * 5] + sh) | (uint32_t)(uint8_t)(p.mat[t * 5 + 1] + sh) << 8 |
                (uint32_t)(uint8_t)(p.mat[t * 5 + 2] + sh) << 16 | (uint32_t)(uint8_t)(p.mat[t * 5 + 3] + sh) << 24;
        rt[5 + t] = (uint8_t)(p.mat[t * 5 + 4] + sh) | (uint32_t)(uint8_t)sh << 8;
    }
}

// u8 jobs: one 8-thread group per job, two reference lanes per thread (sw_pass_u8x2): the
// forward pass of every job.  A reverse pass that can reach the forward score is appended to
// `rev` (rev[0] the count, the job ids from rev[2]) for mate_rev_kernel_u8x2, which keeps
// all its groups busy with listed jobs.
template <int SMAX, bool FAST, bool FULL>
__global__ void __launch_bounds__(kMateThreads)
mate_sw_kernel_u8x2(const fa_mate_job *__restrict__ jobs, const uint32_t *__restrict__ order, uint32_t n,
                    const uint8_t *__restrict__ qseq, const uint8_t *__restrict__ tseq, const MateParams p,
                    int bcap, fa_kswr *__restrict__ out, unsigned long long *__restrict__ cells_out,
                    uint32_t *__restrict__ status, uint32_t *__restrict__ rev)
{
    constexpr int G = 8;
    extern __shared__ uint32_t bsm[];
    mate_row_tables<FAST>(bsm, p);
    __syncthreads();
    const uint32_t gtid = blockIdx.x * kMateThreads + threadIdx.x;
    const uint32_t gidx = gtid / G;
    const int lane = threadIdx.x & 31;
    const int l = lane % G;
    const uint32_t gmask = ((1u << G) - 1u) << (lane - l);
    unsigned long long cells = 0;
    uint32_t st = 0;
    if (gidx < n) {
        const uint32_t jid = order ? order[gidx] : gidx;
        const fa_mate_job jb = jobs[jid];
        // this group's run list, then its row snapshot (the block's lists come first)
        uint32_t *blist = bsm + 16 + (threadIdx.x / G) * bcap;
        uint32_t *hm = bsm + 16 + (kMateThreads / G) * bcap + (threadIdx.x / G) * (SMAX * G);
        SeqView Q{qseq + jb.q_off, -1}, Tg{tseq + jb.t_off, -1};
        fa_kswr r = sw_pass_u8x2<SMAX, false, FAST, FULL>(Q, jb.qlen, Tg, jb.tlen, jb.xtra, p, gmask, l, blist, bcap, hm, bsm,
                                              cells, st);
        if (mate_needs_start(r, jb.xtra)) {
            if (!mate_start_reachable(r, p)) {
                cells += (unsigned long long)(r.qe + 1) * (unsigned)jb.tlen;
            } else if (l == 0) {
                rev[2 + atomicAdd(rev, 1u)] = jid;
            }
        }
        st = __reduce_or_sync(gmask, st);
        if (l == 0) {
            out[jid] = r;
            if (st) atomicOr(status, st);
        } else {
            cells = 0;
        }
    }
    if (cells_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, o);
        if (lane == 0 && cells) atomicAdd(cells_out, cells);
    }
}

// The reverse passes listed by mate_sw_kernel_u8x2, four jobs per warp taken from a shared
// counter (rev[1]) as warps finish, the forward result read back from `out`.
template <int SMAX, bool FAST>
__global__ void __launch_bounds__(kMateThreads, 7)
mate_rev_kernel_u8x2(const fa_mate_job *__restrict__ jobs, const uint8_t *__restrict__ qseq,
                     const uint8_t *__restrict__ tseq, const MateParams p, fa_kswr *__restrict__ out,
                     unsigned long long *__restrict__ cells_out, uint32_t *__restrict__ status,
                     uint32_t *__restrict__ rev)
{
    constexpr int G = 8;
    extern __shared__ uint32_t bsm[];
    mate_row_tables<FAST>(bsm, p);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int l = lane % G;
    const uint32_t gmask = ((1u << G) - 1u) << (lane - l);
    uint32_t *hm = bsm + 16 + (threadIdx.x / G) * (SMAX * G);
    const uint32_t count = *(volatile uint32_t *)rev;
    unsigned long long cells = 0;
    uint32_t st = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(rev + 1, 32u / G);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t idx = base + lane / G;
        if (idx < count) {
            const uint32_t jid = rev[2 + idx];
            const fa_mate_job jb = jobs[jid];
            const fa_kswr r = out[jid];
            SeqView Q2{qseq + jb.q_off, r.qe}, T2{tseq + jb.t_off, r.te};
            const fa_kswr rr = sw_pass_u8x2<SMAX, true, FAST>(Q2, r.qe + 1, T2, jb.tlen, FA_KSW_XSTOP | (uint32_t)r.score, p,
                                                        gmask, l, nullptr, 0, hm, bsm, cells, st);
            if (l == 0 && rr.score >= r.score) {
                out[jid].tb = r.te - rr.te;
                out[jid].qb = r.qe - rr.qe;
            }
        }
        __syncwarp();
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if (lane == 0 && st) atomicOr(status, st);
    if (l != 0) cells = 0;
    if (cells_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, o);
        if (lane == 0 && cells) atomicAdd(cells_out, cells);
    }
}

template <int SMAX, bool FAST, bool FULL>
static cudaError_t launch_mate_u8x2(const fa_mate_job *d_jobs, const uint32_t *d_order, uint32_t n,
                                    const uint8_t *d_qseq, const uint8_t *d_tseq, const MateParams &p, int bcap,
                                    fa_kswr *d_out, unsigned long long *d_cells, uint32_t *d_status, uint32_t *d_rev,
                                    cudaStream_t stream)
{
    const size_t smem = (16 + (size_t)(kMateThreads / 8) * (bcap + SMAX * 8)) * sizeof(uint32_t);
    cudaError_t err = cudaFuncSetAttribute(mate_sw_kernel_u8x2<SMAX, FAST, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
    if (err != cudaSuccess) return err;
    if (!d_rev) return cudaErrorInvalidValue;
    err = cudaMemsetAsync(d_rev, 0, 2 * sizeof(uint32_t), stream);
    if (err != cudaSuccess) return err;
    const uint64_t threads = (uint64_t)n * 8;
    const uint32_t blocks = (uint32_t)((threads + kMateThreads - 1) / kMateThreads);
    mate_sw_kernel_u8x2<SMAX, FAST, FULL><<<blocks, kMateThreads, smem, stream>>>(d_jobs, d_order, n, d_qseq, d_tseq, p, bcap,
                                                                      d_out, d_cells, d_status, d_rev);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    // reverse passes: as many blocks as are resident at once (or as the jobs need), each warp
    // taking four listed jobs at a time until the list is done
    const size_t rsmem = (16 + (size_t)(kMateThreads / 8) * SMAX * 8) * sizeof(uint32_t);
    err = cudaFuncSetAttribute(mate_rev_kernel_u8x2<SMAX, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsmem);
    if (err != cudaSuccess) return err;
    int dev = 0, sms = 0, per_sm = 0;
    if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
    if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
    if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mate_rev_kernel_u8x2<SMAX, FAST>, kMateThreads,
                                                             rsmem)) != cudaSuccess)
        return err;
    const uint32_t rblocks = std::min<uint32_t>(blocks, (uint32_t)std::max(1, sms * std::max(per_sm, 1)));
    mate_rev_kernel_u8x2<SMAX, FAST><<<rblocks, kMateThreads, rsmem, stream>>>(d_jobs, d_qseq, d_tseq, p, d_out, d_cells,
                                                                         d_status, d_rev);
    return cudaGetLastError();
}

template <int P, int SMAX>
static cudaError_t launch_mate_t(const fa_mate_job *d_jobs, const uint32_t *d_order, uint32_t n,
                                 const uint8_t *d_qseq, const uint8_t *d_tseq, const MateParams &p,
                                 int bcap, fa_kswr *d_out, unsigned long long *d_cells,
                                 uint32_t *d_status, cudaStream_t stream)
{
    const size_t smem = (size_t)(kMateThreads / P) * bcap * sizeof(uint32_t);
    cudaError_t err = cudaFuncSetAttribute(mate_sw_kernel<P, SMAX>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const uint64_t threads = (uint64_t)n * P;
    const uint32_t blocks = (uint32_t)((threads + kMateThreads - 1) / kMateThreads);
    mate_sw_kernel<P, SMAX><<<blocks, kMateThreads, smem, stream>>>(d_jobs, d_order, n, d_qseq, d_tseq,
                                                                    p, bcap, d_out, d_cells, d_status);
    return cudaGetLastError();
}

cudaError_t launch_mate_sw(bool byte_lanes, const fa_mate_job *d_jobs, const uint32_t *d_order,
                           uint32_t n, const uint8_t *d_qseq, const uint8_t *d_tseq,
                           const MateParams &p, int min_qlen, int max_qlen, int max_tlen, fa_kswr *d_out,
                           unsigned long long *d_cells, uint32_t *d_status, uint32_t *d_rev,
                           cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int bcap = (max_tlen + 1) / 2 + 2;   // consecutive list rows differ by >= 2
    // the smallest register depth (segments per lane) that holds the longest query: slots
    // beyond a job's segment count are predicated off but still issue, so the depth tracks
    // the batch's query length (151-bp mates: 10 u8 segments, 19 i16 segments)
#define FA_MATE(PP, SS) launch_mate_t<PP, SS>(d_jobs, d_order, n, d_qseq, d_tseq, p, bcap, d_out, d_cells, d_status, \
                                              stream)
#define FA_MATE2_(SS, FA, FU) launch_mate_u8x2<SS, FA, FU>(d_jobs, d_order, n, d_qseq, d_tseq, p, bcap, d_out, \
                                                           d_cells, d_status, d_rev, stream)
#define FA_MATE2(SS)                                                                                             \
    (fast ? (full(SS) ? FA_MATE2_(SS, true, true) : FA_MATE2_(SS, true, false))                                 \
          : (full(SS) ? FA_MATE2_(SS, false, true) : FA_MATE2_(SS, false, false)))
    // sw_pass_u8x2's FAST form: no u8 saturation possible below the score cap, equal gap penalties
    const bool fast = (max_qlen + 1) * p.max + (p.shift & 0xff) <= 255 && p.o_del == p.o_ins && p.e_del == p.e_ins;
    // FULL form: every job's segment count equals the register depth
    auto full = [&](int smax) { return min_qlen > 16 * (smax - 1); };
    if (byte_lanes) {
        if (max_qlen <= 16 * 10) return FA_MATE2(10);
        if (max_qlen <= 16 * 12) return FA_MATE2(12);
        if (max_qlen <= 16 * 16) return FA_MATE2(16);
        if (max_qlen <= 16 * 24) return FA_MATE2(24);
        return FA_MATE2(32);
    }
#undef FA_MATE2
#undef FA_MATE2_
    if (max_qlen <= 8 * 16) return FA_MATE(8, 16);
    if (max_qlen <= 8 * 20) return FA_MATE(8, 20);
    if (max_qlen <= 8 * 24) return FA_MATE(8, 24);
    return FA_MATE(8, 32);
#undef FA_MATE
}

}  // namespace fa
