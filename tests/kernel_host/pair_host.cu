// Test harness: the int16x2 extension kernel's thread body compiled for the host, so
// the CPU test suite can run the exact kernel code against the oracle.
#define FA_HOST_KERNEL_TESTS 1
#include "../../ferrousalign_b200/csrc/extend_pair_kernel.cu"

namespace fa {
// launch_* bodies reference these; the harness never launches anything
}

extern "C" int pair_host_run(const fa_params *prm, const fa_job *jobs, const uint32_t *order, uint32_t n,
                             const uint8_t *qseq, const uint8_t *tseq, int qcap, fa_ext_result *out,
                             uint32_t *status) {
    fa::ExtParams k;
    for (int i = 0; i < 25; ++i) k.mat[i] = prm->mat[i];
    k.m = prm->m;
    k.o_del = prm->o_del; k.e_del = prm->e_del; k.o_ins = prm->o_ins; k.e_ins = prm->e_ins;
    k.zdrop = prm->zdrop; k.end_bonus = prm->end_bonus;
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (prm->mat[i] > ms) ms = prm->mat[i];
    k.max_score = ms;
    k.flags = prm->flags;
    if (!fa::ext_pair_eligible(k)) return -1;
    return fa::ext_pair_host(jobs, order, n, qseq, tseq, k, qcap, out, status);
}
