/*
 * ksw_oracle.c -- CPU restatement of the reference's seed-extension and
 * mate-rescue Smith-Waterman.  TEST INFRASTRUCTURE ONLY: the parity checker and
 * the timed CPU baseline.  The shipped library never links or calls this file.
 *
 * Followed line by line for behaviour (not structure):
 *   ksw_extend2   src/core/alignment/ksw_affine_gap.rs:952-1169
 *   ksw_qinit     src/core/alignment/ksw_affine_gap.rs:78-151
 *   ksw_u8_impl   src/core/alignment/ksw_affine_gap.rs:267-494
 *   ksw_i16_impl  src/core/alignment/ksw_affine_gap.rs:503-735
 *   ksw_align2    src/core/alignment/ksw_affine_gap.rs:773-861
 * The band-retry policy follows bwa-mem2's mem_chain2aln loop (MAX_BAND_TRY=2);
 * the reference itself has no retry, so that part is pinned by no reference test.
 */
#include "ksw_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* Rust `f64 as i32`: truncate toward zero, saturate, NaN -> 0. */
static int32_t rust_f64_as_i32(double x)
{
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (int32_t)x;
}

/* Band after the max_ins / max_del clamp (ksw_affine_gap.rs:999-1018). */
static int ext_band_clamp(int qlen, int m, const int8_t *mat, int o_del, int e_del,
                          int o_ins, int e_ins, int w, int end_bonus)
{
    int max_score = 0;
    for (int i = 0; i < m * m; ++i)
        if (mat[i] > (int8_t)max_score) max_score = mat[i];
    int max_ins = rust_f64_as_i32(((double)qlen * (double)max_score + (double)end_bonus -
                                   (double)o_ins) / (double)e_ins + 1.0);
    if (max_ins < 1) max_ins = 1;
    if (w > max_ins) w = max_ins;
    int max_del = rust_f64_as_i32(((double)qlen * (double)max_score + (double)end_bonus -
                                   (double)o_del) / (double)e_del + 1.0);
    if (max_del < 1) max_del = 1;
    if (w > max_del) w = max_del;
    return w;
}

typedef struct { int32_t h, e; } eh_t;

int ora_wide_clean(const fa_params *p, int qlen, int W, int init_reach)
{
    W = ext_band_clamp(qlen, p->m, p->mat, p->o_del, p->e_del, p->o_ins, p->e_ins, W, p->end_bonus);
    const int end0 = W + 1 < qlen ? W + 1 : qlen;
    return init_reach <= end0;
}

int ora_ksw_extend2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                    int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                    int w, int end_bonus, int zdrop, int h0,
                    fa_ext_result *out, ora_ext_trace *trace)
{
    return ora_ksw_extend2_flags(qlen, query, tlen, target, m, mat, o_del, e_del, o_ins, e_ins, w, end_bonus,
                                 zdrop, h0, 0, out, trace);
}

int ora_ksw_extend2_flags(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                          int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                          int w, int end_bonus, int zdrop, int h0, unsigned flags,
                          fa_ext_result *out, ora_ext_trace *trace)
{
    /* ksw_affine_gap.rs:968 asserts h0 > 0; FA_PARAM_H0_ZERO lifts that for h0 == 0 and the
     * recurrence below then runs on h0 = 0 exactly as written */
    if (h0 < 0 || (h0 == 0 && !(flags & FA_PARAM_H0_ZERO))) return FA_ERR_ARG;
    if (qlen <= 0 || tlen < 0 || m <= 0 || m > 5) return FA_ERR_ARG;
    for (int j = 0; j < qlen; ++j) if (query[j] >= m) return FA_ERR_ARG;
    for (int i = 0; i < tlen; ++i) if (target[i] >= m) return FA_ERR_ARG;

    const int oe_del = o_del + e_del, oe_ins = o_ins + e_ins;
    int8_t *qp = (int8_t *)malloc((size_t)qlen * m);
    eh_t *eh = (eh_t *)calloc((size_t)qlen + 1, sizeof(eh_t));
    if (!qp || !eh) { free(qp); free(eh); return FA_ERR_CAPACITY; }

    /* query profile: qp[k*qlen + j] = mat[k*m + query[j]] */
    for (int k = 0; k < m; ++k)
        for (int j = 0; j < qlen; ++j) qp[k * qlen + j] = mat[k * m + query[j]];

    /* first row */
    eh[0].h = h0;
    eh[1].h = h0 > oe_ins ? h0 - oe_ins : 0;
    for (int j = 2; j <= qlen && eh[j - 1].h > e_ins; ++j) eh[j].h = eh[j - 1].h - e_ins;
    int init_reach = 0;
    for (int j = 1; j <= qlen; ++j) if (eh[j].h > 0) init_reach = j;

    w = ext_band_clamp(qlen, m, mat, o_del, e_del, o_ins, e_ins, w, end_bonus);

    int max = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, max_off = 0;
    int beg = 0, end = qlen;
    int64_t cells = 0;
    int rows = 0, clamped = 0, label = 0;

    /* Exit-bound certificate.  Every path that leaves the computed region does so
     * through a gap cell the run itself computes (the F value past a row's end,
     * the E value of a column the band drops on the left, the first column or the
     * first row beyond the band).  From such an exit x at (ix, jx) the path can
     * reach row i with at most  min(x + a*(i-ix), x + a*D - e_del*(i-ix-D)),
     * D = qlen-1-jx.  P1 and P3 keep the maxima of the two lines' intercepts. */
    int a = 0;
    for (int k = 0; k < m * m; ++k) if (mat[k] > a) a = mat[k];
    const int NEG = -(1 << 29);
    /* [0]: exits on the right (F past the row end, first row), [1]: on the left
     * (dropped columns, first column); each side's tents peak near one row */
    int P1[2] = {NEG, NEG}, P3[2] = {NEG, NEG};
    int bmax = NEG, first_fail = INT32_MAX, row_ok = 1, stale = 0;
    int srun = 0, sev = 0, slast = 0;   /* bound shortfall: running max, at the last event, last row */
    int max_written = -1, broke = 0, zbreak = 0;
#define ORA_EXIT(side, x, ix, jx) do { const int x_ = (x), ix_ = (ix), D_ = qlen - 1 - (jx); \
        if (x_ > 0) { if (x_ - a * ix_ > P1[side]) P1[side] = x_ - a * ix_;                 \
            const int t_ = x_ + (a + e_del) * D_ + e_del * ix_; if (t_ > P3[side]) P3[side] = t_; } } while (0)

    for (int i = 0; i < tlen; ++i) {
        int f = 0, m_row = 0, mj = -1;
        const int8_t *q = &qp[target[i] * qlen];
        ++rows;
        /* band and constraint */
        int beg_a = beg, end_a = end;
        if (beg < i - w) beg = i - w;
        if (end > i + w + 1) end = i + w + 1;
        if (end > qlen) end = qlen;
        if (beg != beg_a) clamped = 1;
        if (end != (end_a < qlen ? end_a : qlen)) clamped = 1;
        if (i - beg > label) label = i - beg;
        if (end - 1 - i > label) label = end - 1 - i;
        if (end > beg) cells += end - beg;
        if (i == 0) {
            if (end < qlen) ORA_EXIT(0, eh[end].h, -1, end - 1);       /* first row past the band */
        } else {
            for (int j = beg_a; j < beg && j < qlen; ++j) ORA_EXIT(1, eh[j].e, i, j);  /* dropped column */
            if (beg_a == 0 && beg > 0) {                               /* first column leaves */
                const int x = h0 - (o_del + e_del * i);
                ORA_EXIT(1, x, i - 1, -1);
            }
            const int lo = beg > max_written + 1 ? beg : max_written + 1;
            const int hi = end - 1 < init_reach ? end - 1 : init_reach;
            if (lo <= hi) stale = 1;                                   /* reads a never-written cell */
        }

        /* first column */
        int h1;
        if (beg == 0) {
            h1 = h0 - (o_del + e_del * (i + 1));
            if (h1 < 0) h1 = 0;
        } else {
            h1 = 0;
        }
        for (int j = beg; j < end; ++j) {
            eh_t *p = &eh[j];
            int M = p->h, e = p->e;     /* H(i-1,j-1), E(i,j) */
            p->h = h1;                   /* H(i,j-1) for the next row */
            M = M ? M + q[j] : 0;        /* no I directly followed by D */
            int h = M > e ? M : e;
            h = h > f ? h : f;
            h1 = h;
            if (m_row < h) { mj = j; m_row = h; }   /* first column attaining the row max */
            int t = M - oe_del; if (t < 0) t = 0;
            e -= e_del; if (e < t) e = t;
            p->e = e;
            t = M - oe_ins; if (t < 0) t = 0;
            f -= e_ins; if (f < t) f = t;
        }
        eh[end].h = h1;
        eh[end].e = 0;

        /* whole query aligned: (beg..end).contains(qlen-1) || end == qlen */
        if ((qlen - 1 >= beg && qlen - 1 < end) || end == qlen) {
            int h_end = end == qlen ? h1 : eh[qlen - 1].h;
            if (gscore < h_end) { gscore = h_end; max_ie = i; }   /* earliest row wins ties */
        }
        if (end > max_written) max_written = end;
        if (end < qlen) ORA_EXIT(0, f, i, end);                        /* F past the row's end */
        {
            int b = NEG;
            for (int sd = 0; sd < 2; ++sd) {
                if (P1[sd] == NEG) continue;
                const int b1 = P1[sd] + a * i, b3 = P3[sd] - e_del * i;
                const int bs = b1 < b3 ? b1 : b3;
                if (bs > b) b = bs;
            }
            row_ok = m_row > 0 ? b < m_row : b <= 0;
            if (!row_ok && first_fail == INT32_MAX) first_fail = i;
            slast = row_ok ? 0 : b - m_row + 1;
            if (slast > srun) srun = slast;
            if (max_ie == i) sev = srun;
            if (b > bmax) bmax = b;
        }
        if (m_row == 0) { broke = 1; break; }
        if (m_row > max) {
            max = m_row; max_i = i; max_j = mj;
            sev = srun;
            int off = mj - i; if (off < 0) off = -off;
            if (max_off < off) max_off = off;
        } else if (zdrop > 0) {
            int di = i - max_i, dj = mj - max_j;
            if (di > dj) {
                if (max - m_row - (di - dj) * e_del > zdrop) { broke = zbreak = 1; break; }
            } else if (max - m_row - (dj - di) * e_ins > zdrop) {
                broke = zbreak = 1;
                break;
            }
        }
        /* adaptive band for the next row */
        int nb = beg;
        while (nb < end && eh[nb].h == 0 && eh[nb].e == 0) ++nb;
        beg = nb;
        int ne = end;
        while (ne > beg && eh[ne].h == 0 && eh[ne].e == 0) --ne;
        end = ne + 2 < qlen ? ne + 2 : qlen;
    }

    out->score = max;
    out->qle = max_j + 1;
    out->tle = max_i + 1;
    out->gtle = max_ie + 1;
    out->gscore = gscore;
    out->max_off = max_off;
    if (trace) {
        trace->cells = cells;
        trace->rows = rows;
        trace->clamped = clamped;
        trace->label = label < 0 ? 0 : label;
        trace->w_eff = w;
        /* outputs are fixed by the rows up to the last max or gscore event; the
         * break row must match too, so the wider run stops at the same row */
        const int i_ev = max_i > max_ie ? max_i : max_ie;
        const int lim = max < gscore ? max : gscore;
        /* after a zero row every live path has left the region: the rows a wider
         * run may still process are bounded by the tents over [rows-1, tlen-1] */
        int fut = NEG;
        if (broke && !zbreak) {
            const int i0 = rows - 1, i1 = tlen - 1;
            for (int sd = 0; sd < 2; ++sd) {
                if (P1[sd] == NEG) continue;
                /* tent peak where the two lines meet; its max over [i0, i1] */
                int lo = i0, hi = i1;
                while (lo < hi) {            /* first row where the falling line is lower */
                    const int mid = lo + (hi - lo) / 2;
                    if (P3[sd] - e_del * mid <= P1[sd] + a * mid) hi = mid; else lo = mid + 1;
                }
                int best_t = NEG;
                for (int k = lo - 1; k <= lo; ++k) {
                    if (k < i0 || k > i1) continue;
                    const int b1 = P1[sd] + a * k, b3 = P3[sd] - e_del * k;
                    const int v = b1 < b3 ? b1 : b3;
                    if (v > best_t) best_t = v;
                }
                if (best_t > fut) fut = best_t;
            }
        }
        const int tail_ok = !broke || (zbreak ? row_ok : fut < lim);
        trace->bound_ok = !stale && gscore > 0 && first_fail > i_ev && tail_ok && bmax < lim;
        /* how far the bound missed, in columns of extra band: widening the band moves
         * every exit at least one more gap extension away */
        int slack = sev;                                 /* rows up to the last event count */
        if (broke && zbreak && slast > slack) slack = slast;
        if (bmax >= lim && bmax - lim + 1 > slack) slack = bmax - lim + 1;
        if (broke && !zbreak && fut >= lim && fut - lim + 1 > slack) slack = fut - lim + 1;
        const int e_min = e_del < e_ins ? e_del : e_ins;
        int delta = ORA_HINT_NONE;
        if (!stale && gscore > 0 && e_min > 0) {
            const int sl = slack > 1 ? slack : 1;
            delta = (sl + e_min - 1) / e_min;
            if (delta > ORA_HINT_NONE) delta = ORA_HINT_NONE;
        }
        trace->hint = delta;
        trace->init_reach = init_reach;
    }
#undef ORA_EXIT
    free(qp);
    free(eh);
    return FA_OK;
}

/* ------------------------------------------------------------------------ */
/* ksw_align2: emulation of the 128-bit striped kernels lane by lane.        */

#define SW_MAX_LANES 16

typedef struct {
    int size;          /* 1: u8 lanes (16), 2: i16 lanes (8) */
    int qlen, slen, P;
    int shift, mdiff, max;
    int32_t *qp;       /* [m][slen][P] profile values (u8 already shifted) */
    int32_t *H0, *H1, *E, *Hmax;  /* [slen][P] */
} swq_t;

static void swq_free(swq_t *q)
{
    free(q->qp); free(q->H0); free(q->H1); free(q->E); free(q->Hmax);
}

/* ksw_qinit (ksw_affine_gap.rs:78-151) */
static int swq_init(swq_t *q, int size, int qlen, const uint8_t *query, int m, const int8_t *mat)
{
    memset(q, 0, sizeof(*q));
    q->size = size > 1 ? 2 : 1;
    q->P = q->size == 1 ? 16 : 8;
    q->qlen = qlen;
    q->slen = (qlen + q->P - 1) / q->P;
    int min_score = 127, max_score = 0;
    for (int i = 0; i < m * m; ++i) {
        if (mat[i] < min_score) min_score = mat[i];
        if (mat[i] > max_score) max_score = mat[i];
    }
    q->shift = (uint8_t)(256 - min_score);
    q->mdiff = (uint8_t)(max_score + q->shift);
    q->max = (uint8_t)max_score;
    size_t cells = (size_t)q->slen * q->P;
    q->qp = (int32_t *)malloc(sizeof(int32_t) * cells * m);
    q->H0 = (int32_t *)calloc(cells ? cells : 1, sizeof(int32_t));
    q->H1 = (int32_t *)calloc(cells ? cells : 1, sizeof(int32_t));
    q->E = (int32_t *)calloc(cells ? cells : 1, sizeof(int32_t));
    q->Hmax = (int32_t *)calloc(cells ? cells : 1, sizeof(int32_t));
    if (!q->qp || !q->H0 || !q->H1 || !q->E || !q->Hmax) { swq_free(q); return -1; }
    for (int a = 0; a < m; ++a)
        for (int j = 0; j < q->slen; ++j)
            for (int l = 0; l < q->P; ++l) {
                int k = j + l * q->slen;
                int s = k < qlen ? mat[a * m + query[k]] : 0;
                int v = q->size == 1 ? (uint8_t)(int8_t)(s + (int8_t)q->shift) : (int16_t)s;
                q->qp[((size_t)a * q->slen + j) * q->P + l] = v;
            }
    return 0;
}

static inline int sat_u8(int x) { return x < 0 ? 0 : x > 255 ? 255 : x; }
static inline int sat_i16(int x) { return x < -32768 ? -32768 : x > 32767 ? 32767 : x; }

/* ksw_u8_impl / ksw_i16_impl (ksw_affine_gap.rs:267-494, 503-735) */
static fa_kswr sw_kernel(swq_t *q, int tlen, const uint8_t *target, int o_del, int e_del,
                         int o_ins, int e_ins, uint32_t xtra, int64_t *cells)
{
    fa_kswr r = {0, -1, -1, -1, -1, -1, -1};
    const uint32_t minsc = (xtra & FA_KSW_XSUBO) ? (xtra & 0xffff) : 0x10000;
    const uint32_t endsc = (xtra & FA_KSW_XSTOP) ? (xtra & 0xffff) : 0x10000;
    const int P = q->P, slen = q->slen, u8 = q->size == 1;
    const int oe_del = o_del + e_del, oe_ins = o_ins + e_ins;
    int gmax = 0, te = -1;
    int64_t *b = NULL;
    size_t nb = 0, cb = 0;
    const size_t ncell = (size_t)slen * P;

    memset(q->E, 0, sizeof(int32_t) * ncell);
    memset(q->H0, 0, sizeof(int32_t) * ncell);
    memset(q->Hmax, 0, sizeof(int32_t) * ncell);

    int32_t *H0 = q->H0, *H1 = q->H1;
    for (int i = 0; i < tlen; ++i) {
        int f[SW_MAX_LANES] = {0}, mx[SW_MAX_LANES] = {0}, h[SW_MAX_LANES];
        if (cells) *cells += q->qlen;
        /* h = H0[slen-1] shifted up one lane */
        h[0] = 0;
        for (int l = 1; l < P; ++l) h[l] = H0[(slen - 1) * P + l - 1];
        const int32_t *S = &q->qp[(size_t)target[i] * ncell];
        for (int j = 0; j < slen; ++j) {
            for (int l = 0; l < P; ++l) {
                int s = S[j * P + l], e = q->E[j * P + l], hv;
                if (u8) {
                    hv = sat_u8(sat_u8(h[l] + s) - q->shift);
                    hv = hv > e ? hv : e;
                    hv = hv > f[l] ? hv : f[l];
                    mx[l] = mx[l] > hv ? mx[l] : hv;
                    H1[j * P + l] = hv;
                    int ee = sat_u8(e - e_del), eo = sat_u8(hv - oe_del);
                    q->E[j * P + l] = ee > eo ? ee : eo;
                    int fe = sat_u8(f[l] - e_ins), fo = sat_u8(hv - oe_ins);
                    f[l] = fe > fo ? fe : fo;
                } else {
                    hv = sat_i16(h[l] + s);
                    hv = hv > e ? hv : e;
                    hv = hv > f[l] ? hv : f[l];
                    mx[l] = mx[l] > hv ? mx[l] : hv;
                    H1[j * P + l] = hv;
                    int ee = sat_i16(e - e_del), eo = sat_i16(hv - oe_del);
                    q->E[j * P + l] = ee > eo ? ee : eo;
                    int fe = sat_i16(f[l] - e_ins), fo = sat_i16(hv - oe_ins);
                    f[l] = fe > fo ? fe : fo;
                }
                h[l] = H0[j * P + l];
            }
        }
        /* lazy-F: shift f one lane per pass; stop after a pass that changed nothing */
        for (int k = 0; k < P; ++k) {
            for (int l = P - 1; l > 0; --l) f[l] = f[l - 1];
            f[0] = 0;
            int changed = 0;
            for (int j = 0; j < slen; ++j)
                for (int l = 0; l < P; ++l) {
                    int hb = H1[j * P + l];
                    int hn = hb > f[l] ? hb : f[l];
                    H1[j * P + l] = hn;
                    f[l] = u8 ? sat_u8(f[l] - e_ins) : sat_i16(f[l] - e_ins);
                    if (hn != hb) changed = 1;
                }
            if (!changed) break;
        }
        int imax = 0;
        for (int l = 0; l < P; ++l) {
            int v = u8 ? mx[l] : (mx[l] & 0xffff);   /* max_epu16 of non-negative lanes */
            if (v > imax) imax = v;
        }
        if ((uint32_t)imax >= minsc) {
            if (nb == 0 || (int32_t)(b[nb - 1] & 0xffffffff) + 1 != i) {
                if (nb == cb) {
                    cb = cb ? cb * 2 : 8;
                    b = (int64_t *)realloc(b, cb * sizeof(int64_t));
                }
                b[nb++] = ((int64_t)imax << 32) | (uint32_t)i;
            } else if ((int32_t)(b[nb - 1] >> 32) < imax) {
                b[nb - 1] = ((int64_t)imax << 32) | (uint32_t)i;
            }
        }
        if (imax > gmax) {
            gmax = imax;
            te = i;
            memcpy(q->Hmax, H1, sizeof(int32_t) * ncell);
            if (u8) {
                if (gmax + q->shift >= 255 || (uint32_t)gmax >= endsc) break;
            } else {
                if ((uint32_t)gmax >= 0x7FFF || (uint32_t)gmax >= endsc) break;
            }
        }
        int32_t *tmp = H0; H0 = H1; H1 = tmp;
    }
    q->H0 = H0; q->H1 = H1;

    const int sat = u8 ? 255 : 0x7FFF;
    r.score = u8 ? (gmax + q->shift < 255 ? gmax : 255) : gmax;
    r.te = te;
    if (r.score != sat) {
        int max_qe = -1, max_val = -1;
        for (size_t k = 0; k < ncell; ++k) {
            int seg = (int)(k / P), lane = (int)(k % P);
            int cand = seg + lane * slen;
            if (cand >= q->qlen) continue;
            /* extract_epi8 / extract_epi16 return signed lanes */
            int val = u8 ? (int)(int8_t)(uint8_t)q->Hmax[k] : (int)(int16_t)q->Hmax[k];
            if (val > max_val) { max_val = val; max_qe = cand; }
            else if (val == max_val && cand < max_qe) max_qe = cand;
        }
        r.qe = max_qe;
        if (nb) {
            int iv = (r.score + q->max - 1) / q->max;
            int low = te - iv, high = te + iv;
            for (size_t k = 0; k < nb; ++k) {
                int e_idx = (int32_t)(b[k] & 0xffffffff);
                int sc = (int32_t)(b[k] >> 32);
                if ((e_idx < low || e_idx > high) && sc > r.score2) { r.score2 = sc; r.te2 = e_idx; }
            }
        }
    }
    free(b);
    return r;
}

int ora_ksw_align2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                   int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                   uint32_t xtra, fa_kswr *out, int64_t *cells)
{
    if (qlen <= 0 || tlen < 0 || m <= 0 || m > 5) return FA_ERR_ARG;
    for (int j = 0; j < qlen; ++j) if (query[j] >= m) return FA_ERR_ARG;
    for (int i = 0; i < tlen; ++i) if (target[i] >= m) return FA_ERR_ARG;
    int max_score = 0;
    for (int i = 0; i < m * m; ++i) if (mat[i] > max_score) max_score = mat[i];
    if (max_score <= 0) return FA_ERR_ARG;   /* the reference divides by q.max */

    int size = (xtra & FA_KSW_XBYTE) ? 1 : 2;
    swq_t q;
    if (swq_init(&q, size, qlen, query, m, mat)) return FA_ERR_CAPACITY;
    if (cells) *cells = 0;
    fa_kswr r = sw_kernel(&q, tlen, target, o_del, e_del, o_ins, e_ins, xtra, cells);
    int find_start = (xtra & FA_KSW_XSTART) &&
                     !((xtra & FA_KSW_XSUBO) && r.score < (int)(xtra & 0xffff));
    if (find_start && r.qe >= 0 && r.te >= 0) {
        int ql = r.qe + 1, tl = r.te + 1;
        uint8_t *rq = (uint8_t *)malloc(ql);
        uint8_t *rt = (uint8_t *)malloc(tlen ? tlen : 1);
        for (int k = 0; k < ql; ++k) rq[k] = query[ql - 1 - k];
        for (int k = 0; k < tlen; ++k) rt[k] = k < tl ? target[tl - 1 - k] : target[k];
        swq_t q2;
        if (swq_init(&q2, q.size, ql, rq, m, mat) == 0) {
            fa_kswr rr = sw_kernel(&q2, tlen, rt, o_del, e_del, o_ins, e_ins,
                                   FA_KSW_XSTOP | (uint32_t)r.score, cells);
            if (rr.score >= r.score) { r.tb = r.te - rr.te; r.qb = r.qe - rr.qe; }
            swq_free(&q2);
        }
        free(rq);
        free(rt);
    }
    swq_free(&q);
    *out = r;
    return FA_OK;
}

/* ------------------------------------------------------------------------ */
/* Batch drivers                                                             */

typedef struct {
    int kind;  /* 0 ext, 1 policy, 2 mate */
    const fa_params *p;
    const fa_policy *pol;
    const fa_mate_params *mp;
    const fa_job *jobs;
    const fa_mate_job *mjobs;
    const uint8_t *qseq, *tseq;
    const int32_t *w_first;
    fa_ext_result *out;
    fa_kswr *mout;
    ora_ext_trace *traces;
    int32_t *w_final, *tries;
    int64_t *cells;
    uint32_t n, next;
    pthread_mutex_t mu;
    int err;
} batch_t;

static int run_ext(const fa_params *p, const fa_job *jb, const uint8_t *qseq, const uint8_t *tseq,
                   int w, fa_ext_result *o, ora_ext_trace *tr)
{
    return ora_ksw_extend2_flags(jb->qlen, qseq + jb->q_off, jb->tlen, tseq + jb->t_off, p->m, p->mat,
                                 p->o_del, p->e_del, p->o_ins, p->e_ins, w, p->end_bonus, p->zdrop,
                                 jb->h0, p->flags, o, tr);
}

/* Smallest band of the ladder 1, 2, 3, 4, 6, 8, 12, 16, ... (2^k, 3*2^(k-1)) >= b. */
static int ladder_ceil(int b)
{
    if (b <= 2) return b;
    int p2 = 1;
    while (p2 < b) p2 <<= 1;
    return 3 * p2 / 4 >= b ? 3 * p2 / 4 : p2;
}

/* bwa-mem2 mem_chain2aln retry loop, starting from try k0 with `prev` given. */
static int policy_bwa(const fa_params *p, const fa_job *jb, const uint8_t *qs, const uint8_t *ts,
                      int max_tries, fa_ext_result *o, int32_t *wfin, int32_t *ntries, int64_t *cx)
{
    int prev = jb->dir == FA_DIR_RIGHT ? jb->h0 : 0;
    for (int k = 0; k < max_tries; ++k) {
        int w = jb->w << k;
        ora_ext_trace tr;
        int rc = run_ext(p, jb, qs, ts, w, o, &tr);
        if (rc) return rc;
        *cx += tr.cells;
        *ntries += 1;
        *wfin = w;
        if (o->score == prev || o->max_off < (w >> 1) + (w >> 2)) break;
        prev = o->score;
    }
    return FA_OK;
}

static int policy_one(const batch_t *B, uint32_t i)
{
    const fa_job *jb = &B->jobs[i];
    const fa_policy *pol = B->pol;
    int32_t wfin = jb->w, ntries = 0;
    int64_t cx = 0;
    int rc = FA_OK;
    if (pol->mode == FA_POLICY_SINGLE) {
        ora_ext_trace tr;
        rc = run_ext(B->p, jb, B->qseq, B->tseq, jb->w, &B->out[i], &tr);
        cx = tr.cells; ntries = 1;
    } else if (pol->mode == FA_POLICY_BWA) {
        rc = policy_bwa(B->p, jb, B->qseq, B->tseq, pol->max_tries, &B->out[i], &wfin, &ntries, &cx);
    } else {
        int w = B->w_first ? B->w_first[i] : jb->w;
        if (w < pol->w_min) w = pol->w_min;
        int accepted = 0;
        while (w < jb->w) {
            ora_ext_trace tr;
            rc = run_ext(B->p, jb, B->qseq, B->tseq, w, &B->out[i], &tr);
            if (rc) break;
            cx += tr.cells; ntries += 1;
            int ok = !tr.clamped, jump = 0;
            if (!ok && (pol->judge & FA_JUDGE_BOUND)) {
                const int prev0 = jb->dir == FA_DIR_RIGHT ? jb->h0 : 0;
                ok = tr.bound_ok && ora_wide_clean(B->p, jb->qlen, jb->w, tr.init_reach) &&
                     (B->out[i].score == prev0 || B->out[i].max_off < (jb->w >> 1) + (jb->w >> 2));
            }
            if (!ok && (pol->judge & FA_JUDGE_MAXOFF)) {
                int off_ok = B->out[i].max_off < (w >> 1) + (w >> 2);
                int global = B->out[i].gscore == B->out[i].score;
                ok = off_ok && (!(pol->judge & FA_JUDGE_GLOBAL) || global);
                jump = off_ok && !ok;
            }
            if (ok) { accepted = 1; wfin = w; break; }
            if (!jump && (pol->judge & FA_JUDGE_BOUND) && (pol->judge & FA_JUDGE_ONCE) &&
                (pol->judge & FA_JUDGE_HINT) && ntries == 1 &&
                tr.hint < ORA_HINT_NONE && ora_wide_clean(B->p, jb->qlen, jb->w, tr.init_reach)) {
                const int nw = ladder_ceil(w + tr.hint);     /* one retry at the suggested band */
                if (2 * nw <= jb->w) { w = nw; continue; }
            }
            if (jump || (pol->judge & FA_JUDGE_ONCE)) break;   /* straight to the configured band */
            w <<= 1;
        }
        if (!rc && !accepted)
            rc = policy_bwa(B->p, jb, B->qseq, B->tseq, pol->max_tries, &B->out[i], &wfin, &ntries, &cx);
    }
    if (B->w_final) B->w_final[i] = wfin;
    if (B->tries) B->tries[i] = ntries;
    if (B->cells) B->cells[i] = cx;
    return rc;
}

static void *batch_worker(void *arg)
{
    batch_t *B = (batch_t *)arg;
    for (;;) {
        pthread_mutex_lock(&B->mu);
        uint32_t s = B->next;
        B->next = s + 64 < B->n ? s + 64 : B->n;
        uint32_t e = B->next;
        pthread_mutex_unlock(&B->mu);
        if (s >= e) break;
        for (uint32_t i = s; i < e; ++i) {
            int rc;
            if (B->kind == 0) {
                rc = run_ext(B->p, &B->jobs[i], B->qseq, B->tseq, B->jobs[i].w, &B->out[i],
                             B->traces ? &B->traces[i] : NULL);
            } else if (B->kind == 1) {
                rc = policy_one(B, i);
            } else {
                const fa_mate_job *mj = &B->mjobs[i];
                rc = ora_ksw_align2(mj->qlen, B->qseq + mj->q_off, mj->tlen, B->tseq + mj->t_off,
                                    B->mp->m, B->mp->mat, B->mp->o_del, B->mp->e_del,
                                    B->mp->o_ins, B->mp->e_ins, mj->xtra, &B->mout[i],
                                    B->cells ? &B->cells[i] : NULL);
            }
            if (rc) {
                pthread_mutex_lock(&B->mu);
                if (!B->err) B->err = rc;
                pthread_mutex_unlock(&B->mu);
            }
        }
    }
    return NULL;
}

static int run_batch(batch_t *B, int nthreads)
{
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_mutex_init(&B->mu, NULL);
    B->next = 0;
    B->err = 0;
    if (nthreads == 1) {
        batch_worker(B);
    } else {
        pthread_t th[256];
        for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, batch_worker, B);
        for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    }
    pthread_mutex_destroy(&B->mu);
    return B->err;
}

int ora_ext_batch(const fa_params *p, const fa_job *jobs, uint32_t n,
                  const uint8_t *qseq, const uint8_t *tseq,
                  fa_ext_result *out, ora_ext_trace *traces, int nthreads)
{
    batch_t B;
    memset(&B, 0, sizeof(B));
    B.kind = 0; B.p = p; B.jobs = jobs; B.qseq = qseq; B.tseq = tseq;
    B.out = out; B.traces = traces; B.n = n;
    return run_batch(&B, nthreads);
}

int ora_ext_batch_policy(const fa_params *p, const fa_policy *pol,
                         const fa_job *jobs, uint32_t n,
                         const uint8_t *qseq, const uint8_t *tseq,
                         const int32_t *w_first, fa_ext_result *out,
                         int32_t *w_final, int32_t *tries, int64_t *cells_exec,
                         int nthreads)
{
    batch_t B;
    memset(&B, 0, sizeof(B));
    B.kind = 1; B.p = p; B.pol = pol; B.jobs = jobs; B.qseq = qseq; B.tseq = tseq;
    B.w_first = w_first; B.out = out; B.w_final = w_final; B.tries = tries;
    B.cells = cells_exec; B.n = n;
    return run_batch(&B, nthreads);
}

int ora_mate_batch(const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                   const uint8_t *qseq, const uint8_t *tseq, fa_kswr *out,
                   int64_t *cells, int nthreads)
{
    batch_t B;
    memset(&B, 0, sizeof(B));
    B.kind = 2; B.mp = p; B.mjobs = jobs; B.qseq = qseq; B.tseq = tseq;
    B.mout = out; B.cells = cells; B.n = n;
    return run_batch(&B, nthreads);
}
