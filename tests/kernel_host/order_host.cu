// Test harness: the job-ordering kernels' bin mapping compiled for the host.  The histogram
// and the scatter kernels both map a job to fa::qlen_bin(qlen); order_host_run replays the
// scatter's cursor walk on the CPU with that same function, so a CPU test can check that
// every order slot is written exactly once whatever the query lengths (negative and
// oversized ones included).
#include "../../ferrousalign_b200/csrc/order_kernel.cu"

extern "C" int order_host_bin(int qlen) { return fa::qlen_bin(qlen); }

// hist[FA_MAX_QLEN + 1] from the lengths, start offsets longest first (as the host launcher
// computes them), then one cursor step per job in job order.  Returns the number of order
// slots written more than once or outside [0, n), and fills order[] (unwritten slots keep
// their incoming value).
extern "C" int order_host_run(const int *qlen, uint32_t n, uint32_t *order) {
    std::vector<uint32_t> hist(FA_MAX_QLEN + 1, 0), cursor(FA_MAX_QLEN + 1, 0), seen(n, 0);
    for (uint32_t i = 0; i < n; ++i) ++hist[fa::qlen_bin(qlen[i])];
    uint32_t acc = 0;
    for (int q = FA_MAX_QLEN; q >= 0; --q) { cursor[q] = acc; acc += hist[q]; }
    int bad = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t slot = cursor[fa::qlen_bin(qlen[i])]++;
        if (slot >= n || seen[slot]++) { ++bad; continue; }
        order[slot] = i;
    }
    return bad;
}
