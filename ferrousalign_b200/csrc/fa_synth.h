/* fa_synth.h -- seeded synthetic workloads (libfa_synth.so, host only). */
#ifndef FA_SYNTH_H
#define FA_SYNTH_H

#include <stdint.h>
#include "../../include/ferrous_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FA_SYNTH_MAX_READ 1024

typedef struct {
    int32_t read_len_min, read_len_max;
    int32_t seed_len_min, seed_len_max;
    int32_t seed_at_start;        /* 1: one right job per read (seed = read prefix)   */
    int32_t w;                    /* band; target window = query length + w           */
    int32_t match_score;          /* h0 = seed length * match_score                   */
    int32_t n_indel_rates;        /* per-read indel rate drawn from indel_rates[]     */
    double  indel_rates[4];
    double  sub_rate;
    double  indel_mean;           /* geometric indel length mean                      */
} fa_synth_ext_cfg;

/* generator-side facts about each job (features for the band predictor) */
typedef struct {
    int32_t seed_len;
    int32_t diag_spread;          /* |diagonal difference| to the chain partner seed  */
    int32_t has_partner;
    int32_t read_idx;
    int32_t indel_rate_ppm;
    int32_t _pad;
} fa_synth_ext_info;

typedef struct {
    int32_t read_len;
    int32_t match_score, min_seed_len;
    int32_t _pad;
    double  insert_mean, insert_sd;
    double  sub_rate, indel_rate;
} fa_synth_mate_cfg;

int fa_synth_reference(uint64_t seed, uint64_t len, double n_rate, double repeat_frac, uint8_t *out);

/* Returns the number of jobs written (n_jobs) or -FA_ERR_*. */
int64_t fa_synth_ext_jobs(const uint8_t *ref, uint64_t ref_len, uint64_t seed,
                          const fa_synth_ext_cfg *cfg, uint32_t n_jobs, int nthreads,
                          fa_job *jobs, fa_synth_ext_info *info,
                          uint8_t *qseq, uint64_t qseq_cap, uint8_t *tseq, uint64_t tseq_cap,
                          uint64_t *q_used, uint64_t *t_used);

int64_t fa_synth_mate_jobs(const uint8_t *ref, uint64_t ref_len, uint64_t seed,
                           const fa_synth_mate_cfg *cfg, uint32_t n, int nthreads,
                           fa_mate_job *jobs, uint8_t *qseq, uint64_t qseq_cap,
                           uint8_t *tseq, uint64_t tseq_cap, uint64_t *q_used, uint64_t *t_used);

uint32_t fa_mate_xtra_host(int32_t mate_len, int32_t match_score, int32_t min_seed_len);

#ifdef __cplusplus
}
#endif
#endif
