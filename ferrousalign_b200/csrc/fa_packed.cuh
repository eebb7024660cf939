// fa_packed.cuh -- sequence buffers as the extension kernels read them: byte codes or
// 2-bit packed bases with their N runs (fa_packed_seq in the C ABI).
//
// Packed layout: base k is bits 2*(k % 4) .. 2*(k % 4) + 1 of byte k / 4 (codes A0 C1 G2 T3),
// so a little-endian 32-bit word w holds bases 16w .. 16w + 15.  A 2-bit code cannot hold N
// (code 4); N bases are listed as sorted, non-overlapping runs, as the reference's index
// keeps its ambiguous stretches beside the 2-bit .pac (bntseq.rs:451-535).  A reader keeps
// a cursor on the first run that can still touch what it reads, so a job with no N nearby
// pays one compare per four bases.
#pragma once

#include <cstdint>

#include "fa_device.cuh"

namespace fa {

// One sequence buffer on the device.  packed == 0: p holds byte codes 0-4 (runs unused);
// packed == 1: p holds 2-bit bases (nbytes bytes, 4-byte aligned) and runs the N runs.
struct SeqBuf {
    const uint8_t *p;
    uint64_t nbytes;
    const fa_nrun *runs;
    uint32_t n_runs;
    uint32_t packed;
};

__host__ __device__ __forceinline__ uint32_t funnel_r(uint32_t lo, uint32_t hi, uint32_t sh) {
#ifdef __CUDA_ARCH__
    return __funnelshift_r(lo, hi, sh);
#else
    return (uint32_t)((((uint64_t)hi << 32) | lo) >> (sh & 31));
#endif
}

// Four 2-bit codes (8 bits) spread to four bytes, code k in byte k.
__host__ __device__ __forceinline__ uint32_t spread4(uint32_t x8) {
    uint32_t t = (x8 | (x8 << 12)) & 0x000F000Fu;   // codes 0,1 in bits 0-3, codes 2,3 in bits 16-19
    return (t | (t << 6)) & 0x03030303u;            // code 1 to bits 8-9, code 3 to bits 24-25
}

// Reader over one job's sequence in a packed buffer: get4(r) returns the codes of positions
// r .. r+3 of the job (N runs applied) as bytes, zero for positions outside [0, len).
// Positions asked for may go back by up to kBack bases from the furthest one asked so far
// (the band-feature kernel re-reads a window that overlaps the previous one).
struct PackedReader {
    static constexpr int64_t kBack = 32;
    const uint32_t *w;
    uint64_t nwords;
    const fa_nrun *runs;
    uint32_t nr, k;
    uint64_t base, nxt;   // the job's first base; runs[k].pos (or ~0 when no run is left)
    int len;

    __host__ __device__ __forceinline__ void init(const SeqBuf &b, uint64_t off, int len_) {
        w = reinterpret_cast<const uint32_t *>(b.p);
        nwords = (b.nbytes + 3) >> 2;
        runs = b.runs;
        nr = b.n_runs;
        base = off;
        len = len_;
        // first run that ends past the job's start (binary search over the sorted runs)
        uint32_t lo = 0, hi = nr;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (runs[mid].pos + runs[mid].len <= off) lo = mid + 1;
            else hi = mid;
        }
        k = lo;
        nxt = k < nr ? runs[k].pos : ~0ull;
    }

    __host__ __device__ __forceinline__ uint32_t word(uint64_t i) const { return i < nwords ? w[i] : 0u; }

    // codes of the four bases at absolute positions pos .. pos+3, N runs applied
    __host__ __device__ __forceinline__ uint32_t raw4(uint64_t pos) {
        const uint64_t wi = pos >> 4;
        const uint32_t x = funnel_r(word(wi), word(wi + 1), (uint32_t)(pos & 15) * 2u) & 0xFFu;
        uint32_t v = spread4(x);
        if (nxt < pos + 4) {   // an N run starts before the end of these four bases: rare
            for (uint32_t j = k; j < nr && runs[j].pos < pos + 4; ++j) {
                const uint64_t a = runs[j].pos > pos ? runs[j].pos : pos;
                const uint64_t e = runs[j].pos + runs[j].len;
                const uint64_t b = e < pos + 4 ? e : pos + 4;
                for (uint64_t q = a; q < b; ++q) {
                    const uint32_t sh = (uint32_t)(q - pos) * 8u;
                    v = (v & ~(0xFFu << sh)) | (4u << sh);
                }
            }
            // runs ending kBack bases before this read can no longer be asked for
            while (k < nr && runs[k].pos + runs[k].len + kBack <= pos) ++k;
            nxt = k < nr ? runs[k].pos : ~0ull;
        }
        return v;
    }

    // word at a signed index: 0 outside the buffer
    __host__ __device__ __forceinline__ uint32_t word_s(int64_t i) const {
        return i >= 0 && (uint64_t)i < nwords ? w[i] : 0u;
    }

    // codes of positions r .. r + 4*NW - 1 of the job, four per word (same bytes as NW calls
    // of get4): ceil(NW / 4) + 1 word loads, one funnel shift per 16 bases
    template <int NW>
    __host__ __device__ __forceinline__ void getw(int r, uint32_t (&out)[NW]) {
        constexpr int NA = (NW + 3) / 4;   // aligned 16-base words
        const int64_t pos = (int64_t)base + r;
        const int64_t wi = pos >> 4;       // floor, also below zero
        const uint32_t sh = (uint32_t)(pos & 15) * 2u;
        uint32_t wv[NA + 1];
#pragma unroll
        for (int m = 0; m <= NA; ++m) wv[m] = word_s(wi + m);
#pragma unroll
        for (int m = 0; m < NA; ++m) wv[m] = funnel_r(wv[m], wv[m + 1], sh);
#pragma unroll
        for (int m = 0; m < NW; ++m) out[m] = spread4((wv[m / 4] >> (8 * (m % 4))) & 0xFFu);
        const int64_t end = pos + 4 * NW;
        if (end > 0 && nxt < (uint64_t)end) {   // an N run starts before the end of the span: rare
            for (uint32_t j = k; j < nr && (int64_t)runs[j].pos < end; ++j) {
                const int64_t a = (int64_t)runs[j].pos, e = a + (int64_t)runs[j].len;
#pragma unroll
                for (int m = 0; m < NW; ++m) {
                    const int64_t p0 = pos + 4 * m;
                    const int lo = (int)(a > p0 ? (a - p0 < 4 ? a - p0 : 4) : 0);
                    const int hi = (int)(e > p0 ? (e - p0 < 4 ? e - p0 : 4) : 0);
                    if (hi > lo) {
                        const uint32_t bm = (hi >= 4 ? 0xFFFFFFFFu : (1u << (8 * hi)) - 1u) & ~((1u << (8 * lo)) - 1u);
                        out[m] = (out[m] & ~bm) | (0x04040404u & bm);
                    }
                }
            }
            while (k < nr && (int64_t)(runs[k].pos + runs[k].len) + kBack <= pos) ++k;
            nxt = k < nr ? runs[k].pos : ~0ull;
        }
        // zero outside [0, len)
#pragma unroll
        for (int m = 0; m < NW; ++m) {
            const int p0 = r + 4 * m;
            if (p0 < 0 || p0 + 4 > len) {
                const int lo = p0 >= 0 ? 0 : (-p0 < 4 ? -p0 : 4);
                const int hi = len - p0 <= 0 ? 0 : (len - p0 < 4 ? len - p0 : 4);
                const uint32_t bm = (hi >= 4 ? 0xFFFFFFFFu : (1u << (8 * hi)) - 1u) & ~(lo >= 4 ? 0xFFFFFFFFu : (1u << (8 * lo)) - 1u);
                out[m] &= bm;
            }
        }
    }

    __host__ __device__ __forceinline__ uint32_t get4(int r) {
        if (r >= len || r + 4 <= 0) return 0u;
        // -3 <= r < 0: the bytes of positions r .. -1 are 0, the rest come from position 0 on
        uint32_t v = r < 0 ? raw4(base) << (8u * (uint32_t)(-r)) : raw4(base + (uint64_t)r);
        if (r + 4 > len) v &= 0xFFFFFFFFu >> (8 * (uint32_t)(r + 4 - len));
        return v;
    }
};

// Sequential four-base reads of positions p, p + 4, p + 8, ... through a PackedReader: one
// 16-base span read per four calls.
struct PackedStream4 {
    uint32_t b[4];
    int left, next;

    __host__ __device__ __forceinline__ void start(int pos) { next = pos; left = 0; }

    __host__ __device__ __forceinline__ uint32_t next4(PackedReader &r) {
        if (left == 0) {
            r.getw<4>(next, b);
            next += 16;
            left = 4;
        }
        const uint32_t v = b[0];
        b[0] = b[1];
        b[1] = b[2];
        b[2] = b[3];
        --left;
        return v;
    }
};

}  // namespace fa
