// Test harness: the packed-sequence reader (fa_packed.cuh) compiled for the host.  Reads a
// job's bases at a sequence of positions both as multi-word spans (getw) and four at a time
// (get4), each through its own reader, so the CPU tests can compare the two and the codes.
#include "../../ferrousalign_b200/csrc/fa_packed.cuh"

namespace {
template <int NW>
void read_spans(const fa::SeqBuf &b, uint64_t off, int len, int r0, int step, int nsteps, uint32_t *out_w,
                uint32_t *out_4) {
    fa::PackedReader a, c;
    a.init(b, off, len);
    c.init(b, off, len);
    for (int s = 0; s < nsteps; ++s) {
        const int r = r0 + s * step;
        uint32_t v[NW];
        a.getw<NW>(r, v);
        for (int m = 0; m < NW; ++m) {
            out_w[s * NW + m] = v[m];
            out_4[s * NW + m] = c.get4(r + 4 * m);
        }
    }
}
}  // namespace

// nw: 2, 4 or 7 words (8, 16 or 28 bases) per read; out_w / out_4: nsteps * nw words.
extern "C" int packed_host_read(const fa_packed_seq *pk, uint64_t off, int len, int r0, int step, int nsteps, int nw,
                                uint32_t *out_w, uint32_t *out_4) {
    const fa::SeqBuf b{pk->bases, (pk->n_bases + 3) / 4, pk->n_runs, (uint32_t)pk->n_nruns, 1};
    switch (nw) {
    case 2: read_spans<2>(b, off, len, r0, step, nsteps, out_w, out_4); return 0;
    case 4: read_spans<4>(b, off, len, r0, step, nsteps, out_w, out_4); return 0;
    case 7: read_spans<7>(b, off, len, r0, step, nsteps, out_w, out_4); return 0;
    default: return 1;
    }
}
