/*
 * ksw_oracle.h -- CPU restatement of FerrousAlign's seed-extension and
 * mate-rescue Smith-Waterman, used ONLY as a test checker and as the timed
 * CPU baseline.  Nothing in the shipped library links against this code.
 *
 * Parity status: the reference is Rust and cannot be built here.  The oracle
 * is pinned against the reference's own known-answer tests
 * (src/core/alignment/ksw_affine_gap.rs:1252-1277: ACGT/ACGT -> qle=4,
 * tle=4) plus hand-derived known answers and an independent pure-Python
 * restatement (tests/golden/make_golden.py).  All other reference tests assert
 * only bounds.
 */
#ifndef FA_KSW_ORACLE_H
#define FA_KSW_ORACLE_H

#include <stdint.h>
#include "../include/ferrous_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-extension trace used for the GCUPS numerator and the band certificate. */
typedef struct {
    int64_t cells;     /* sum over processed rows of (end - beg)            */
    int32_t rows;      /* rows processed (including the row that breaks)    */
    int32_t clamped;   /* 1 if the band clamp narrowed [beg,end) in any row */
    int32_t label;     /* max over rows of max(i-beg, end-1-i, 0): the
                          smallest band that reproduces this run exactly    */
    int32_t w_eff;     /* band after the max_ins / max_del clamp             */
    int32_t bound_ok;  /* exit-bound certificate: no path that leaves this
                          run's computed region can change any output       */
    int32_t init_reach;/* last column whose first-row value is positive     */
    int32_t hint;      /* extra band columns the certificate asks for when it
                          fails (ORA_HINT_NONE: none suggested)            */
    int32_t _pad;
} ora_ext_trace;

#define ORA_HINT_NONE 63

/* The exit-bound certificate of a narrow run at band w transfers to a run at
 * configured band W >= w when W's first row covers every positive first-row
 * cell (so W never reads an unwritten column).  Returns 1 if so. */
int ora_wide_clean(const fa_params *p, int qlen, int W, int init_reach);

/* ksw_extend2 (ksw_affine_gap.rs:952-1169).  Returns FA_OK, or FA_ERR_ARG
 * where the reference panics (h0 <= 0, qlen <= 0, code >= m). */
int ora_ksw_extend2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                    int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                    int w, int end_bonus, int zdrop, int h0,
                    fa_ext_result *out, ora_ext_trace *trace);
/* Same, with fa_params.flags: FA_PARAM_H0_ZERO accepts h0 == 0 and runs the recurrence on it
 * as written (the reference's assert at ksw_affine_gap.rs:968 lifted). */
int ora_ksw_extend2_flags(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                          int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                          int w, int end_bonus, int zdrop, int h0, unsigned flags,
                          fa_ext_result *out, ora_ext_trace *trace);

/* ksw_align2 (ksw_affine_gap.rs:773-861) with the 128-bit striped engine the
 * reference instantiates it with (16 u8 lanes, 8 i16 lanes). */
int ora_ksw_align2(int qlen, const uint8_t *query, int tlen, const uint8_t *target,
                   int m, const int8_t *mat, int o_del, int e_del, int o_ins, int e_ins,
                   uint32_t xtra, fa_kswr *out, int64_t *cells);

/* Batch drivers over fa_job / fa_mate_job arrays (nthreads <= 0: all cores). */
int ora_ext_batch(const fa_params *p, const fa_job *jobs, uint32_t n,
                  const uint8_t *qseq, const uint8_t *tseq,
                  fa_ext_result *out, ora_ext_trace *traces, int nthreads);

/* Band-retry policy (bwa-mem2 mem_chain2aln semantics, see fa_policy). */
int ora_ext_batch_policy(const fa_params *p, const fa_policy *pol,
                         const fa_job *jobs, uint32_t n,
                         const uint8_t *qseq, const uint8_t *tseq,
                         const int32_t *w_first, fa_ext_result *out,
                         int32_t *w_final, int32_t *tries, int64_t *cells_exec,
                         int nthreads);

int ora_mate_batch(const fa_mate_params *p, const fa_mate_job *jobs, uint32_t n,
                   const uint8_t *qseq, const uint8_t *tseq, fa_kswr *out,
                   int64_t *cells, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
