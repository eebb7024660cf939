// Test harness: the two-rows-per-thread extension kernel's thread body compiled for the
// host, so the CPU test suite can run the exact kernel code against the oracle.  The other
// extension sources come along because the rows2 launcher calls into them.
#include "../../ferrousalign_b200/csrc/extend_kernel.cu"
#include "../../ferrousalign_b200/csrc/extend_pair_kernel.cu"
#include "../../ferrousalign_b200/csrc/extend_rows2_kernel.cu"

// Runs every job of `order` through rows2_thread (shared-memory stride 1).  Jobs whose
// scores can pass 255 are listed in ovf[0..*ovf_n) instead, as the kernel hands them on.
extern "C" int rows2_host_run(const fa_params *prm, const fa_job *jobs, const uint32_t *order, uint32_t n,
                              const uint8_t *qseq, const uint8_t *tseq, int qcap, fa_ext_result *out,
                              uint32_t *cells, uint32_t *status, uint32_t *ovf, uint32_t *ovf_n) {
    fa::ExtParams k;
    for (int i = 0; i < 25; ++i) k.mat[i] = prm->mat[i];
    k.m = prm->m;
    k.o_del = prm->o_del; k.e_del = prm->e_del; k.o_ins = prm->o_ins; k.e_ins = prm->e_ins;
    k.zdrop = prm->zdrop; k.end_bonus = prm->end_bonus;
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (prm->mat[i] > ms) ms = prm->mat[i];
    k.max_score = ms;
    if (!fa::ext_rows2_eligible(k, qcap)) return -1;
    std::vector<uint16_t> eh((size_t)qcap + 1);
    std::vector<uint8_t> sb((size_t)qcap + 1);
    const bool sym = fa::ext_rows2_sym(k);
    for (uint32_t g = 0; g < n; ++g)
        cells[order[g]] = sym ? fa::rows2_thread<1, true>(order[g], eh.data(), sb.data(), jobs, qseq, tseq, k, qcap,
                                                          nullptr, out, nullptr, nullptr, status, ovf, ovf_n)
                              : fa::rows2_thread<1, false>(order[g], eh.data(), sb.data(), jobs, qseq, tseq, k, qcap,
                                                           nullptr, out, nullptr, nullptr, status, ovf, ovf_n);
    return 0;
}
