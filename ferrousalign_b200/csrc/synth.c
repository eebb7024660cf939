/*
 * synth.c -- seeded synthetic workloads for the extension and mate-rescue paths.
 *
 * The reference measures on real reads it does not ship; these generators stand in
 * with the shapes, sizes and error models of the workloads the library is timed on:
 *   - a reference of i.i.d. uniform A/C/G/T with a fraction of positions set to N
 *     and optional low-complexity dinucleotide-repeat tracts;
 *   - reads sampled at uniform positions with substitutions and geometric-length
 *     indels;
 *   - extension jobs cut the way the reference cuts them
 *     (src/pipelines/linear/batch_extension/collect_soa.rs:150-209): the right job is
 *     the read suffix after an exact seed against the reference window that follows
 *     it, the left job the reversed prefix against the reversed window before it;
 *   - mate-rescue jobs pair a read with a window of the insert-size range on the
 *     opposite strand (src/pipelines/linear/paired/mate_rescue.rs:1975-2021).
 * Every read has its own generator stream (xoshiro256** seeded through splitmix64 from
 * the batch seed and the read index), so output is identical for any thread count.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../../include/ferrous_b200.h"
#include "fa_synth.h"

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed ^ (stream * 0xd1342543de82ef95ull + 0x2545f4914f6cdd1dull);
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&x);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    const uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return res;
}
static double rng_unif(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t rng_below(rng_t *r, uint32_t n) { return n ? (uint32_t)((rng_next(r) >> 32) * (uint64_t)n >> 32) : 0; }
/* geometric length >= 1 with the given mean */
static int rng_geom(rng_t *r, double mean) {
    double p = 1.0 / mean;
    int k = 1;
    while (rng_unif(r) > p && k < 64) ++k;
    return k;
}
static double rng_normal(rng_t *r) {
    double u1 = rng_unif(r), u2 = rng_unif(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

int fa_synth_reference(uint64_t seed, uint64_t len, double n_rate, double repeat_frac, uint8_t *out)
{
    if (!out) return FA_ERR_ARG;
    rng_t r;
    rng_seed(&r, seed, 0xFEEDull);
    for (uint64_t i = 0; i < len; ++i) out[i] = (uint8_t)(rng_next(&r) >> 62);
    if (repeat_frac > 0) {
        uint64_t target = (uint64_t)(repeat_frac * (double)len), done = 0;
        while (done < target) {
            uint64_t tl = 20 + rng_below(&r, 181);          /* tract length 20-200 */
            uint64_t pos = (uint64_t)(rng_unif(&r) * (double)(len > tl ? len - tl : 1));
            uint8_t a = (uint8_t)rng_below(&r, 4), b = (uint8_t)((a + 1 + rng_below(&r, 3)) & 3);
            for (uint64_t k = 0; k < tl && pos + k < len; ++k) out[pos + k] = (k & 1) ? b : a;
            done += tl;
        }
    }
    if (n_rate > 0)
        for (uint64_t i = 0; i < len; ++i)
            if (rng_unif(&r) < n_rate) out[i] = 4;
    return FA_OK;
}

/* Walks the reference from `start`, emitting a read of length L with substitutions and
 * indels; positions < exact_lo or in [exact_from, exact_to) are copied without errors.
 * rpos[k] = reference position aligned to read position k (rpos[L] = end). */
static int make_read(rng_t *r, const uint8_t *ref, uint64_t ref_len, uint64_t start, int L,
                     double sub, double indel, double indel_mean, int exact_from, int exact_to,
                     uint8_t *read, uint64_t *rpos)
{
    uint64_t p = start;
    int k = 0;
    while (k < L) {
        if (p >= ref_len) return -1;
        const int exact = k >= exact_from && k < exact_to;
        if (!exact && indel > 0 && rng_unif(r) < indel) {
            int len = rng_geom(r, indel_mean);
            if (rng_unif(r) < 0.5) {             /* insertion in the read */
                for (int t = 0; t < len && k < L; ++t) {
                    rpos[k] = p;
                    read[k++] = (uint8_t)rng_below(r, 4);
                }
            } else {                              /* deletion from the read */
                p += (uint64_t)len;
            }
            continue;
        }
        if (p >= ref_len) return -1;
        uint8_t b = ref[p];
        if (!exact && rng_unif(r) < sub) {
            uint8_t c = b > 3 ? (uint8_t)rng_below(r, 4) : (uint8_t)((b + 1 + rng_below(r, 3)) & 3);
            b = c;
        }
        rpos[k] = p;
        read[k++] = b;
        ++p;
    }
    rpos[L] = p;
    return 0;
}

typedef struct {
    const uint8_t *ref;
    uint64_t ref_len, seed;
    const fa_synth_ext_cfg *cfg;
    uint32_t n_reads;
    int qcap, tcap, jobs_per_read;
    fa_job *jobs;
    fa_synth_ext_info *info;
    uint8_t *qslot, *tslot;
    int32_t *ok;
    uint32_t next;
    pthread_mutex_t mu;
} ext_work_t;

/* one read -> 1 right job (seed at start) or up to 2 jobs (left + right) */
static void ext_read(ext_work_t *W, uint32_t ridx)
{
    const fa_synth_ext_cfg *c = W->cfg;
    rng_t r;
    rng_seed(&r, W->seed, ridx + 1);
    uint8_t read[FA_SYNTH_MAX_READ];
    uint64_t rpos[FA_SYNTH_MAX_READ + 1];
    for (int j = 0; j < W->jobs_per_read; ++j) W->ok[(size_t)ridx * W->jobs_per_read + j] = 0;
    for (int attempt = 0; attempt < 8; ++attempt) {
        int L = c->read_len_min + (int)rng_below(&r, (uint32_t)(c->read_len_max - c->read_len_min + 1));
        double indel = c->n_indel_rates > 0 ? c->indel_rates[rng_below(&r, (uint32_t)c->n_indel_rates)] : 0.0;
        int sl = c->seed_len_min + (int)rng_below(&r, (uint32_t)(c->seed_len_max - c->seed_len_min + 1));
        if (sl > L - 1) sl = L - 1;
        int spos = c->seed_at_start ? 0 : (int)rng_below(&r, (uint32_t)(L - sl + 1));
        uint64_t margin = (uint64_t)(2 * L + c->w + 64);
        if (W->ref_len <= 2 * margin) return;
        uint64_t start = margin + (uint64_t)(rng_unif(&r) * (double)(W->ref_len - 2 * margin));
        if (make_read(&r, W->ref, W->ref_len, start, L, c->sub_rate, indel, c->indel_mean, spos, spos + sl,
                      read, rpos))
            continue;
        /* second exact seed (chain partner): last 19-mer after the seed that matches the
           reference exactly at its true position */
        int spread = 0, have2 = 0;
        for (int k = L - 19; k >= spos + sl; --k) {
            int okm = 1;
            for (int t = 0; t < 19 && okm; ++t)
                okm = rpos[k + t] + 1 == rpos[k + t + 1] && W->ref[rpos[k + t]] == read[k + t] && read[k + t] < 4;
            if (okm) {
                long d1 = (long)rpos[spos] - spos, d2 = (long)rpos[k] - k;
                spread = (int)labs(d2 - d1);
                have2 = 1;
                break;
            }
        }
        int jslot = 0;
        const int h0 = sl * c->match_score;
        /* left job: reversed prefix vs reversed window before the seed */
        if (!c->seed_at_start && spos > 0 && jslot < W->jobs_per_read) {
            size_t s = (size_t)ridx * W->jobs_per_read + jslot;
            int ql = spos;
            uint64_t rend = rpos[spos];
            int tl = ql + c->w;
            if ((uint64_t)tl > rend) tl = (int)rend;
            if (ql <= W->qcap && tl <= W->tcap && tl >= 0) {
                uint8_t *q = W->qslot + s * W->qcap, *t = W->tslot + s * W->tcap;
                for (int k = 0; k < ql; ++k) q[k] = read[ql - 1 - k];
                for (int k = 0; k < tl; ++k) t[k] = W->ref[rend - 1 - k];
                W->jobs[s].qlen = ql; W->jobs[s].tlen = tl; W->jobs[s].h0 = h0;
                W->jobs[s].w = c->w; W->jobs[s].dir = FA_DIR_LEFT; W->jobs[s]._pad = 0;
                W->info[s].seed_len = sl; W->info[s].diag_spread = spread; W->info[s].has_partner = have2;
                W->info[s].read_idx = ridx; W->info[s].indel_rate_ppm = (int)(indel * 1e6);
                W->ok[s] = 1;
            }
            ++jslot;
        }
        /* right job: suffix after the seed vs the window that follows it */
        if (spos + sl < L && jslot < W->jobs_per_read) {
            size_t s = (size_t)ridx * W->jobs_per_read + jslot;
            int ql = L - (spos + sl);
            uint64_t rb = rpos[spos + sl];
            int tl = ql + c->w;
            if (rb + (uint64_t)tl > W->ref_len) tl = (int)(W->ref_len - rb);
            if (ql <= W->qcap && tl <= W->tcap && tl >= 0) {
                uint8_t *q = W->qslot + s * W->qcap, *t = W->tslot + s * W->tcap;
                memcpy(q, read + spos + sl, (size_t)ql);
                memcpy(t, W->ref + rb, (size_t)tl);
                W->jobs[s].qlen = ql; W->jobs[s].tlen = tl; W->jobs[s].h0 = h0;
                W->jobs[s].w = c->w; W->jobs[s].dir = FA_DIR_RIGHT; W->jobs[s]._pad = 0;
                W->info[s].seed_len = sl; W->info[s].diag_spread = spread; W->info[s].has_partner = have2;
                W->info[s].read_idx = ridx; W->info[s].indel_rate_ppm = (int)(indel * 1e6);
                W->ok[s] = 1;
            }
        }
        return;
    }
}

static void *ext_worker(void *arg)
{
    ext_work_t *W = (ext_work_t *)arg;
    for (;;) {
        pthread_mutex_lock(&W->mu);
        uint32_t s = W->next, e = s + 256 < W->n_reads ? s + 256 : W->n_reads;
        W->next = e;
        pthread_mutex_unlock(&W->mu);
        if (s >= e) break;
        for (uint32_t i = s; i < e; ++i) ext_read(W, i);
    }
    return NULL;
}

static int n_threads(int t) {
    if (t <= 0) t = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (t < 1) t = 1;
    if (t > 128) t = 128;
    return t;
}

int64_t fa_synth_ext_jobs(const uint8_t *ref, uint64_t ref_len, uint64_t seed,
                          const fa_synth_ext_cfg *cfg, uint32_t n_jobs, int nthreads,
                          fa_job *jobs, fa_synth_ext_info *info,
                          uint8_t *qseq, uint64_t qseq_cap, uint8_t *tseq, uint64_t tseq_cap,
                          uint64_t *q_used, uint64_t *t_used)
{
    if (!ref || !cfg || !jobs || !qseq || !tseq || cfg->read_len_max > FA_SYNTH_MAX_READ ||
        cfg->read_len_min < 2 || cfg->read_len_max < cfg->read_len_min || cfg->seed_len_min < 1 ||
        cfg->seed_len_max < cfg->seed_len_min || cfg->n_indel_rates > 4)
        return -FA_ERR_ARG;
    ext_work_t W;
    memset(&W, 0, sizeof(W));
    W.ref = ref; W.ref_len = ref_len; W.seed = seed; W.cfg = cfg;
    W.jobs_per_read = cfg->seed_at_start ? 1 : 2;
    W.qcap = cfg->read_len_max;
    W.tcap = cfg->read_len_max + cfg->w;
    uint64_t q_off = 0, t_off = 0;
    uint32_t produced = 0, round = 0;
    while (produced < n_jobs && round < 64) {
        uint32_t need = n_jobs - produced;
        W.n_reads = cfg->seed_at_start ? need : (need + 1) / 2 + 16;
        size_t slots = (size_t)W.n_reads * W.jobs_per_read;
        W.jobs = (fa_job *)calloc(slots, sizeof(fa_job));
        W.info = (fa_synth_ext_info *)calloc(slots, sizeof(fa_synth_ext_info));
        W.qslot = (uint8_t *)malloc(slots * W.qcap);
        W.tslot = (uint8_t *)malloc(slots * W.tcap);
        W.ok = (int32_t *)calloc(slots, sizeof(int32_t));
        if (!W.jobs || !W.info || !W.qslot || !W.tslot || !W.ok) {
            free(W.jobs); free(W.info); free(W.qslot); free(W.tslot); free(W.ok);
            return -FA_ERR_CAPACITY;
        }
        W.seed = seed + 0x1000003ull * round;
        W.next = 0;
        pthread_mutex_init(&W.mu, NULL);
        int nt = n_threads(nthreads);
        pthread_t th[128];
        for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, ext_worker, &W);
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
        pthread_mutex_destroy(&W.mu);
        for (size_t s = 0; s < slots && produced < n_jobs; ++s) {
            if (!W.ok[s]) continue;
            fa_job jb = W.jobs[s];
            if (q_off + (uint64_t)jb.qlen > qseq_cap || t_off + (uint64_t)jb.tlen > tseq_cap) {
                produced = n_jobs + 1;   /* signal overflow */
                break;
            }
            memcpy(qseq + q_off, W.qslot + s * W.qcap, (size_t)jb.qlen);
            memcpy(tseq + t_off, W.tslot + s * W.tcap, (size_t)jb.tlen);
            jb.q_off = q_off; jb.t_off = t_off;
            q_off += (uint64_t)jb.qlen; t_off += (uint64_t)jb.tlen;
            jobs[produced] = jb;
            if (info) info[produced] = W.info[s];
            ++produced;
        }
        free(W.jobs); free(W.info); free(W.qslot); free(W.tslot); free(W.ok);
        ++round;
        if (produced > n_jobs) return -FA_ERR_CAPACITY;
    }
    if (q_used) *q_used = q_off;
    if (t_used) *t_used = t_off;
    return (int64_t)produced;
}

/* ---- mate rescue -------------------------------------------------------- */

typedef struct {
    const uint8_t *ref;
    uint64_t ref_len, seed;
    const fa_synth_mate_cfg *cfg;
    uint32_t n;
    int tcap;
    fa_mate_job *jobs;
    uint8_t *qseq, *tseq;   /* fixed slots: qseq n*read_len, tseq n*tcap */
    uint32_t next;
    pthread_mutex_t mu;
} mate_work_t;

static void mate_pair(mate_work_t *W, uint32_t i)
{
    const fa_synth_mate_cfg *c = W->cfg;
    rng_t r;
    rng_seed(&r, W->seed, (uint64_t)i + 7);
    const int L = c->read_len;
    uint8_t frag[4096], read[FA_SYNTH_MAX_READ];
    uint64_t rpos[FA_SYNTH_MAX_READ + 1];
    const int lo = (int)(c->insert_mean - 4 * c->insert_sd), hi = (int)(c->insert_mean + 4 * c->insert_sd);
    for (;;) {
        int ins = (int)lround(c->insert_mean + c->insert_sd * rng_normal(&r));
        if (ins < L) ins = L;
        if (ins > 4000) ins = 4000;
        uint64_t margin = (uint64_t)(hi + 2 * L + 64);
        uint64_t p1 = margin + (uint64_t)(rng_unif(&r) * (double)(W->ref_len - 2 * margin));
        memcpy(frag, W->ref + p1, (size_t)ins);
        /* mate read: last L bases of the fragment, sequenced from the opposite strand;
           the rescue query is its reverse complement, i.e. forward-strand bases with errors */
        uint64_t mstart = p1 + (uint64_t)(ins - L);
        if (make_read(&r, W->ref, W->ref_len, mstart, L, c->sub_rate, c->indel_rate, 2.0, 0, 0, read, rpos))
            continue;
        (void)frag;
        /* window: every mate start the insert-size range allows, plus the read length */
        uint64_t wb = p1 + (uint64_t)(lo > L ? lo - L : 0);
        uint64_t we = p1 + (uint64_t)hi;
        int tl = (int)(we - wb);
        if (tl > W->tcap) tl = W->tcap;
        uint8_t *q = W->qseq + (size_t)i * L, *t = W->tseq + (size_t)i * W->tcap;
        memcpy(q, read, (size_t)L);
        memcpy(t, W->ref + wb, (size_t)tl);
        W->jobs[i].qlen = L;
        W->jobs[i].tlen = tl;
        W->jobs[i].xtra = fa_mate_xtra_host(L, c->match_score, c->min_seed_len);
        W->jobs[i]._pad = 0;
        return;
    }
}

static void *mate_worker(void *arg)
{
    mate_work_t *W = (mate_work_t *)arg;
    for (;;) {
        pthread_mutex_lock(&W->mu);
        uint32_t s = W->next, e = s + 256 < W->n ? s + 256 : W->n;
        W->next = e;
        pthread_mutex_unlock(&W->mu);
        if (s >= e) break;
        for (uint32_t i = s; i < e; ++i) mate_pair(W, i);
    }
    return NULL;
}

uint32_t fa_mate_xtra_host(int32_t mate_len, int32_t match_score, int32_t min_seed_len)
{
    uint32_t x = FA_KSW_XSUBO | FA_KSW_XSTART;
    if (mate_len * match_score < 250) x |= FA_KSW_XBYTE;
    return x | (uint32_t)(min_seed_len * match_score);
}

int64_t fa_synth_mate_jobs(const uint8_t *ref, uint64_t ref_len, uint64_t seed,
                           const fa_synth_mate_cfg *cfg, uint32_t n, int nthreads,
                           fa_mate_job *jobs, uint8_t *qseq, uint64_t qseq_cap,
                           uint8_t *tseq, uint64_t tseq_cap, uint64_t *q_used, uint64_t *t_used)
{
    if (!ref || !cfg || !jobs || !qseq || !tseq || cfg->read_len > FA_SYNTH_MAX_READ || cfg->read_len < 2)
        return -FA_ERR_ARG;
    mate_work_t W;
    memset(&W, 0, sizeof(W));
    W.ref = ref; W.ref_len = ref_len; W.seed = seed; W.cfg = cfg; W.n = n; W.jobs = jobs;
    W.tcap = (int)(8 * cfg->insert_sd) + cfg->read_len + 8;
    if ((uint64_t)n * cfg->read_len > qseq_cap || (uint64_t)n * W.tcap > tseq_cap) return -FA_ERR_CAPACITY;
    W.qseq = qseq; W.tseq = tseq;
    pthread_mutex_init(&W.mu, NULL);
    int nt = n_threads(nthreads);
    pthread_t th[128];
    for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, mate_worker, &W);
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&W.mu);
    /* compact the target slots */
    uint64_t t_off = 0;
    for (uint32_t i = 0; i < n; ++i) {
        jobs[i].q_off = (uint64_t)i * cfg->read_len;
        memmove(tseq + t_off, tseq + (size_t)i * W.tcap, (size_t)jobs[i].tlen);
        jobs[i].t_off = t_off;
        t_off += (uint64_t)jobs[i].tlen;
    }
    if (q_used) *q_used = (uint64_t)n * cfg->read_len;
    if (t_used) *t_used = t_off;
    return (int64_t)n;
}
