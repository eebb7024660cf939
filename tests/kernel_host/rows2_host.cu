// Test harness: the two-rows-per-thread extension kernel's thread body compiled for the
// host, so the CPU test suite can run the exact kernel code against the oracle.  The other
// extension sources come along because the rows2 launcher calls into them.
#include "../../ferrousalign_b200/csrc/extend_kernel.cu"
#include "../../ferrousalign_b200/csrc/extend_pair_kernel.cu"
#include "../../ferrousalign_b200/csrc/extend_rows2_kernel.cu"

namespace {
template <bool SYM, bool CERT, int RING>
uint32_t run_one(uint32_t jid, uint16_t *eh, uint8_t *sb, const fa_job *jobs, const fa::SeqBuf &qs,
                 const fa::SeqBuf &ts, const fa::ExtParams &k, int qcap, const int32_t *w_try, fa_ext_result *out,
                 uint8_t *flags, uint32_t *status, uint32_t *ovf, uint32_t *ovf_n) {
    if (qs.packed)
        return fa::rows2_thread<1, SYM, CERT, RING, true>(jid, eh, sb, jobs, qs, ts, k, qcap, w_try, out, flags,
                                                          nullptr, status, ovf, ovf_n);
    return fa::rows2_thread<1, SYM, CERT, RING, false>(jid, eh, sb, jobs, qs, ts, k, qcap, w_try, out, flags, nullptr,
                                                       status, ovf, ovf_n);
}
}  // namespace

// Runs every job of `order` through rows2_thread (shared-memory stride 1).  Jobs whose
// scores can pass 255 are listed in ovf[0..*ovf_n) instead, as the kernel hands them on.
// cert: evaluate the certificate into flags[jid]; ring: 0, 32 or 64 column slots.
// w_try (optional): per-job band of this run, as the learned rounds pass it.
// Sequences: byte codes (qpk / tpk NULL), or 2-bit packed buffers (fa_packed_seq, host
// memory) read through the kernels' packed reader.
extern "C" int rows2_host_run(const fa_params *prm, const fa_job *jobs, const uint32_t *order, uint32_t n,
                              const uint8_t *qseq, const uint8_t *tseq, int qcap, int cert, int ring,
                              const int32_t *w_try, fa_ext_result *out, uint8_t *flags, uint32_t *cells,
                              uint32_t *status, uint32_t *ovf, uint32_t *ovf_n, const fa_packed_seq *qpk,
                              const fa_packed_seq *tpk) {
    fa::SeqBuf qs{qseq, ~0ull, nullptr, 0, 0}, ts{tseq, ~0ull, nullptr, 0, 0};
    if (qpk && tpk) {
        qs = fa::SeqBuf{qpk->bases, (qpk->n_bases + 3) / 4, qpk->n_runs, (uint32_t)qpk->n_nruns, 1};
        ts = fa::SeqBuf{tpk->bases, (tpk->n_bases + 3) / 4, tpk->n_runs, (uint32_t)tpk->n_nruns, 1};
    }
    fa::ExtParams k;
    for (int i = 0; i < 25; ++i) k.mat[i] = prm->mat[i];
    k.m = prm->m;
    k.o_del = prm->o_del; k.e_del = prm->e_del; k.o_ins = prm->o_ins; k.e_ins = prm->e_ins;
    k.zdrop = prm->zdrop; k.end_bonus = prm->end_bonus;
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (prm->mat[i] > ms) ms = prm->mat[i];
    k.max_score = ms;
    k.flags = prm->flags;
    if (!fa::ext_rows2_eligible(k, qcap) || (ring != 0 && ring != 32 && ring != 64)) return -1;
    std::vector<uint16_t> eh((size_t)(ring > 0 ? ring : qcap + 1));
    std::vector<uint8_t> sb((size_t)qcap + 1);
    const bool sym = fa::ext_rows2_sym(k);
    for (uint32_t g = 0; g < n; ++g) {
        const uint32_t j = order[g];
        uint32_t c = 0;
#define RUN(S, C, R) c = run_one<S, C, R>(j, eh.data(), sb.data(), jobs, qs, ts, k, qcap, w_try, out, flags, \
                                          status, ovf, ovf_n)
        if (cert) {
            if (ring == 32) { if (sym) RUN(true, true, 32); else RUN(false, true, 32); }
            else if (ring == 64) { if (sym) RUN(true, true, 64); else RUN(false, true, 64); }
            else { if (sym) RUN(true, true, 0); else RUN(false, true, 0); }
        } else {
            if (ring == 32) { if (sym) RUN(true, false, 32); else RUN(false, false, 32); }
            else if (ring == 64) { if (sym) RUN(true, false, 64); else RUN(false, false, 64); }
            else { if (sym) RUN(true, false, 0); else RUN(false, false, 0); }
        }
#undef RUN
        cells[j] = c;
    }
    return 0;
}

// The listing predicate of the early overflow pass (rows2_int32_job), per job of jobs[0..n):
// listed[j] = 1 where the two-row launch with that list skips job j and the int32 pass runs it.
extern "C" void rows2_host_int32_jobs(const fa_params *prm, const fa_job *jobs, uint32_t n, int qcap,
                                      uint8_t *listed) {
    int a = 0;
    for (int i = 0; i < 25; ++i) if (prm->mat[i] > a) a = prm->mat[i];
    for (uint32_t j = 0; j < n; ++j) listed[j] = fa::rows2_int32_job(jobs[j], qcap, a) ? 1 : 0;
}
