// simd_baseline.cpp -- the reference's SIMD CPU path, restated in C++ as a timed baseline.
//
// Test and benchmark infrastructure only: nothing in the product links it.  It restates
// the three inter-sequence SIMD kernels the reference's pipeline runs on the host, with the
// chunk loops that feed them, so the GPU path can be timed against that CPU path on the
// same host cores:
//
//   ext_i16  sw_kernel_i16 (src/core/alignment/banded_swa/kernel_i16.rs:44-272): saturating
//            int16 lanes, the full qmax x tmax rectangle of a chunk under a band mask, row-max
//            z-drop, 0-based end positions.  16 lanes with AVX2, 32 with AVX-512BW.
//   ext_i8   sw_kernel_with_ws (banded_swa/kernel.rs:29-284): the same shape in saturating
//            int8 lanes, taken when no job of the batch is longer than 128 (the dispatcher's
//            rule, batch_extension/dispatch.rs:100-107).  32 lanes AVX2, 64 AVX-512BW.
//   kswv     batch_ksw_align_avx2 (src/core/alignment/kswv_avx2.rs:93-641): the mate-rescue
//            u8 local SW with the XOR/shuffle score table, per-row maxima, the every-other-lane
//            second best and the estimated tb/qb.  32 lanes AVX2, 64 AVX-512BW.
//
// Chunking follows the intended all-jobs loop (banded_swa/dispatch.rs:13-138,
// batch_extension/dispatch.rs:270-395): consecutive jobs in chunks of the vector width, each
// chunk transposed to a position-major SoA padded with 0xFF (soa.rs:11-71,
// workspace.rs:768-857), chunks spread over host threads as rayon spreads them.  Two
// deliberate departures from the code as written, both toward the intended behaviour the
// comments there state: every chunk is scored (the pipeline's dispatcher scores only the
// first W jobs, dispatch.rs:120-146), and lengths are carried at full width instead of being
// clamped to 127 in int8 fields (soa.rs:30-41, workspace.rs:789-790).  The kernels' outputs
// are not ksw_extend2's (their z-drop, band and end positions differ by design), so these
// runs are throughput baselines; their own correctness is pinned by the reference's kernel
// tests (tests/kernel_optimization_test.rs) and by agreement between vector widths.
//
// Built twice by build_oracle.py: with -DFA_ISA=2 -mavx512bw (the AVX-512BW engines) and
// with -DFA_ISA=1 -mavx2 -mno-avx512f (the AVX2 engines and the portable 8-lane engine), so
// the AVX2 numbers come from code that cannot use AVX-512 instructions.

#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "../include/ferrous_b200.h"

#ifndef FA_ISA
#define FA_ISA 1
#endif

namespace {

// ------------------------------------------------------------------ vector engines
// Each engine: W lanes; V a vector; M a lane mask.  blend(a, b, m) = m ? b : a;
// keep(a, m) = m ? a : 0.

#if FA_ISA == 1
struct I16Avx2 {
    static constexpr int W = 16;
    using V = __m256i;
    using M = __m256i;
    static V zero() { return _mm256_setzero_si256(); }
    static V set1(int16_t x) { return _mm256_set1_epi16(x); }
    static V load(const int16_t *p) { return _mm256_loadu_si256((const __m256i *)p); }
    static void store(int16_t *p, V v) { _mm256_storeu_si256((__m256i *)p, v); }
    static V adds(V a, V b) { return _mm256_adds_epi16(a, b); }
    static V subs(V a, V b) { return _mm256_subs_epi16(a, b); }
    static V max(V a, V b) { return _mm256_max_epi16(a, b); }
    static V min(V a, V b) { return _mm256_min_epi16(a, b); }
    static M eq(V a, V b) { return _mm256_cmpeq_epi16(a, b); }
    static M gt(V a, V b) { return _mm256_cmpgt_epi16(a, b); }
    static M mand(M a, M b) { return _mm256_and_si256(a, b); }
    static M mor(M a, M b) { return _mm256_or_si256(a, b); }
    static M mload(const int16_t *p) { return load(p); }
    static V blend(V a, V b, M m) { return _mm256_blendv_epi8(a, b, m); }
    static V keep(V a, M m) { return _mm256_and_si256(a, m); }
};

struct I8Avx2 {
    static constexpr int W = 32;
    using V = __m256i;
    using M = __m256i;
    static V zero() { return _mm256_setzero_si256(); }
    static V set1(int8_t x) { return _mm256_set1_epi8(x); }
    static V load(const int8_t *p) { return _mm256_loadu_si256((const __m256i *)p); }
    static void store(int8_t *p, V v) { _mm256_storeu_si256((__m256i *)p, v); }
    static V adds(V a, V b) { return _mm256_adds_epi8(a, b); }
    static V subs(V a, V b) { return _mm256_subs_epi8(a, b); }
    static V max(V a, V b) { return _mm256_max_epi8(a, b); }
    static V minu(V a, V b) { return _mm256_min_epu8(a, b); }
    static M eq(V a, V b) { return _mm256_cmpeq_epi8(a, b); }
    static M gt(V a, V b) { return _mm256_cmpgt_epi8(a, b); }
    static V vor(V a, V b) { return _mm256_or_si256(a, b); }
    static M msb(V a) { return a; }   // blendv reads each byte's top bit
    static M mand(M a, M b) { return _mm256_and_si256(a, b); }
    static M mload(const int8_t *p) { return load(p); }
    static V blend(V a, V b, M m) { return _mm256_blendv_epi8(a, b, m); }
    static V keep(V a, M m) { return _mm256_and_si256(a, m); }
};

struct U8Avx2 {
    static constexpr int W = 32;
    using V = __m256i;
    using M = __m256i;
    static V zero() { return _mm256_setzero_si256(); }
    static V set1(uint8_t x) { return _mm256_set1_epi8((char)x); }
    static V table(const int8_t *t16) {   // the 16-byte table in both 128-bit halves
        const __m128i t = _mm_loadu_si128((const __m128i *)t16);
        return _mm256_broadcastsi128_si256(t);
    }
    static V load(const uint8_t *p) { return _mm256_loadu_si256((const __m256i *)p); }
    static void store(uint8_t *p, V v) { _mm256_storeu_si256((__m256i *)p, v); }
    static V vxor(V a, V b) { return _mm256_xor_si256(a, b); }
    static V vor(V a, V b) { return _mm256_or_si256(a, b); }
    static V shuffle(V t, V idx) { return _mm256_shuffle_epi8(t, idx); }
    static V addsu(V a, V b) { return _mm256_adds_epu8(a, b); }
    static V subsu(V a, V b) { return _mm256_subs_epu8(a, b); }
    static V maxu(V a, V b) { return _mm256_max_epu8(a, b); }
    static V add(V a, V b) { return _mm256_add_epi8(a, b); }
    static M eq(V a, V b) { return _mm256_cmpeq_epi8(a, b); }
    static M gtu(V a, V b) {   // unsigned a > b: flip the sign bits, compare signed
        const V s = _mm256_set1_epi8((char)0x80);
        return _mm256_cmpgt_epi8(_mm256_xor_si256(a, s), _mm256_xor_si256(b, s));
    }
    static M geu(V a, V b) { return _mm256_cmpeq_epi8(_mm256_max_epu8(a, b), a); }
    static M msb(V a) { return a; }
    static M mand(M a, M b) { return _mm256_and_si256(a, b); }
    static M mor(M a, M b) { return _mm256_or_si256(a, b); }
    static M mandnot(M a, M b) { return _mm256_andnot_si256(a, b); }   // ~a & b
    static M all() { return _mm256_set1_epi8(-1); }
    static M none() { return _mm256_setzero_si256(); }
    static bool any(M m) { return _mm256_movemask_epi8(m) != 0; }
    static V blend(V a, V b, M m) { return _mm256_blendv_epi8(a, b, m); }
    static uint64_t bits(M m) { return (uint32_t)_mm256_movemask_epi8(m); }
};
#endif

#if FA_ISA == 2
struct I16Avx512 {
    static constexpr int W = 32;
    using V = __m512i;
    using M = __mmask32;
    static V zero() { return _mm512_setzero_si512(); }
    static V set1(int16_t x) { return _mm512_set1_epi16(x); }
    static V load(const int16_t *p) { return _mm512_loadu_si512((const void *)p); }
    static void store(int16_t *p, V v) { _mm512_storeu_si512((void *)p, v); }
    static V adds(V a, V b) { return _mm512_adds_epi16(a, b); }
    static V subs(V a, V b) { return _mm512_subs_epi16(a, b); }
    static V max(V a, V b) { return _mm512_max_epi16(a, b); }
    static V min(V a, V b) { return _mm512_min_epi16(a, b); }
    static M eq(V a, V b) { return _mm512_cmpeq_epi16_mask(a, b); }
    static M gt(V a, V b) { return _mm512_cmpgt_epi16_mask(a, b); }
    static M mand(M a, M b) { return a & b; }
    static M mor(M a, M b) { return a | b; }
    static M mload(const int16_t *p) { return _mm512_movepi16_mask(load(p)); }
    static V blend(V a, V b, M m) { return _mm512_mask_blend_epi16(m, a, b); }
    static V keep(V a, M m) { return _mm512_maskz_mov_epi16(m, a); }
};

struct I8Avx512 {
    static constexpr int W = 64;
    using V = __m512i;
    using M = __mmask64;
    static V zero() { return _mm512_setzero_si512(); }
    static V set1(int8_t x) { return _mm512_set1_epi8(x); }
    static V load(const int8_t *p) { return _mm512_loadu_si512((const void *)p); }
    static void store(int8_t *p, V v) { _mm512_storeu_si512((void *)p, v); }
    static V adds(V a, V b) { return _mm512_adds_epi8(a, b); }
    static V subs(V a, V b) { return _mm512_subs_epi8(a, b); }
    static V max(V a, V b) { return _mm512_max_epi8(a, b); }
    static V minu(V a, V b) { return _mm512_min_epu8(a, b); }
    static M eq(V a, V b) { return _mm512_cmpeq_epi8_mask(a, b); }
    static M gt(V a, V b) { return _mm512_cmpgt_epi8_mask(a, b); }
    static V vor(V a, V b) { return _mm512_or_si512(a, b); }
    static M msb(V a) { return _mm512_movepi8_mask(a); }
    static M mand(M a, M b) { return a & b; }
    static M mload(const int8_t *p) { return _mm512_movepi8_mask(load(p)); }
    static V blend(V a, V b, M m) { return _mm512_mask_blend_epi8(m, a, b); }
    static V keep(V a, M m) { return _mm512_maskz_mov_epi8(m, a); }
};

struct U8Avx512 {
    static constexpr int W = 64;
    using V = __m512i;
    using M = __mmask64;
    static V zero() { return _mm512_setzero_si512(); }
    static V set1(uint8_t x) { return _mm512_set1_epi8((char)x); }
    static V table(const int8_t *t16) {
        const __m128i t = _mm_loadu_si128((const __m128i *)t16);
        return _mm512_broadcast_i32x4(t);
    }
    static V load(const uint8_t *p) { return _mm512_loadu_si512((const void *)p); }
    static void store(uint8_t *p, V v) { _mm512_storeu_si512((void *)p, v); }
    static V vxor(V a, V b) { return _mm512_xor_si512(a, b); }
    static V vor(V a, V b) { return _mm512_or_si512(a, b); }
    static V shuffle(V t, V idx) { return _mm512_shuffle_epi8(t, idx); }
    static V addsu(V a, V b) { return _mm512_adds_epu8(a, b); }
    static V subsu(V a, V b) { return _mm512_subs_epu8(a, b); }
    static V maxu(V a, V b) { return _mm512_max_epu8(a, b); }
    static V add(V a, V b) { return _mm512_add_epi8(a, b); }
    static M eq(V a, V b) { return _mm512_cmpeq_epi8_mask(a, b); }
    static M gtu(V a, V b) { return _mm512_cmpgt_epu8_mask(a, b); }
    static M geu(V a, V b) { return _mm512_cmpge_epu8_mask(a, b); }
    static M msb(V a) { return _mm512_movepi8_mask(a); }
    static M mand(M a, M b) { return a & b; }
    static M mor(M a, M b) { return a | b; }
    static M mandnot(M a, M b) { return ~a & b; }
    static M all() { return ~(M)0; }
    static M none() { return 0; }
    static bool any(M m) { return m != 0; }
    static V blend(V a, V b, M m) { return _mm512_mask_blend_epi8(m, a, b); }
    static uint64_t bits(M m) { return m; }
};
#endif

#if FA_ISA == 1
// Portable 8-lane int16 engine (the width of the reference's SSE/NEON engine): plain loops,
// used to check that the vector engines agree with a lane-by-lane evaluation.
struct I16Port {
    static constexpr int W = 8;
    struct V { int16_t x[W]; };
    using M = V;
    static int16_t sat(int v) { return (int16_t)std::min(32767, std::max(-32768, v)); }
    template <class F> static V map2(V a, V b, F f) { V r; for (int k = 0; k < W; ++k) r.x[k] = f(a.x[k], b.x[k]); return r; }
    static V zero() { V r; memset(&r, 0, sizeof r); return r; }
    static V set1(int16_t v) { V r; for (int k = 0; k < W; ++k) r.x[k] = v; return r; }
    static V load(const int16_t *p) { V r; memcpy(r.x, p, sizeof r.x); return r; }
    static void store(int16_t *p, V v) { memcpy(p, v.x, sizeof v.x); }
    static V adds(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return sat(x + y); }); }
    static V subs(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return sat(x - y); }); }
    static V max(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return std::max(x, y); }); }
    static V min(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return std::min(x, y); }); }
    static M eq(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return (int16_t)(x == y ? -1 : 0); }); }
    static M gt(V a, V b) { return map2(a, b, [](int16_t x, int16_t y) { return (int16_t)(x > y ? -1 : 0); }); }
    static M mand(M a, M b) { return map2(a, b, [](int16_t x, int16_t y) { return (int16_t)(x & y); }); }
    static M mor(M a, M b) { return map2(a, b, [](int16_t x, int16_t y) { return (int16_t)(x | y); }); }
    static M mload(const int16_t *p) { return load(p); }
    static V blend(V a, V b, M m) { V r; for (int k = 0; k < W; ++k) r.x[k] = m.x[k] ? b.x[k] : a.x[k]; return r; }
    static V keep(V a, M m) { V r; for (int k = 0; k < W; ++k) r.x[k] = m.x[k] ? a.x[k] : 0; return r; }
};
#endif

struct OutScore {   // banded_swa/types.rs:77-85 (the three fields the kernels set)
    int32_t score, te, qe;
};

struct ChunkIn {    // one chunk of jobs, transposed (SoA, position-major, stride W)
    int lanes, max_q, max_t;
};

// ------------------------------------------------------------- sw_kernel_i16 restatement
// kernel_i16.rs:44-272, one chunk.  q/t: SoA int16 codes (0xFF padding), qlen/tlen/h0/w per
// lane; h/e: DP rows of qmax * W int16.
template <class E>
void kernel_i16(const int16_t *q_soa, const int16_t *t_soa, const int16_t *qlen, const int16_t *tlen,
                const int16_t *h0, const int16_t *w, int lanes, int qmax, int tmax, const fa_params &p,
                int16_t *h, int16_t *e, OutScore *out) {
    constexpr int W = E::W;
    using V = typename E::V;
    using M = typename E::M;
    if (qmax == 0 || tmax == 0 || lanes == 0) return;
    const V zero = E::zero();
    const V match_v = E::set1(p.mat[0]), mis_v = E::set1(p.mat[1]), amb_v = E::set1(p.mat[24]);
    const V three = E::set1(3), one = E::set1(1);
    const V oe_del = E::set1((int16_t)(p.o_del + p.e_del)), oe_ins = E::set1((int16_t)(p.o_ins + p.e_ins));
    const V e_del = E::set1((int16_t)p.e_del), e_ins = E::set1((int16_t)p.e_ins);
    memset(e, 0, sizeof(int16_t) * (size_t)qmax * W);
    // first row: h0, max(h0 - oe_ins, 0), then -e_ins clamped at 0 (kernel_i16.rs:86-101)
    const V h0v = E::load(h0);
    E::store(h, h0v);
    V hp = E::max(E::subs(h0v, oe_ins), zero);
    if (qmax > 1) E::store(h + W, hp);
    for (int j = 2; j < qmax; ++j) {
        hp = E::max(E::subs(hp, e_ins), zero);
        E::store(h + (size_t)j * W, hp);
    }
    V max_s = h0v, max_i = E::set1(-1), max_j = E::set1(-1);
    alignas(64) int16_t beg[W], end[W], term[W], ms[W], rm[W];
    bool done[W];
    int n_done = 0;
    for (int l = 0; l < W; ++l) { beg[l] = 0; end[l] = l < lanes ? qlen[l] : 0; done[l] = false; }
    const V qlen_v = E::load(qlen);
    const V w_v = E::load(w);
    for (int i = 0; i < tmax; ++i) {
        if (n_done == lanes) break;
        V f = zero;
        V hd = E::load(h);
        const V s1 = E::load(t_soa + (size_t)i * W);
        const V iv = E::set1((int16_t)i);
        // band bounds, kept from row to row (kernel_i16.rs:149-161)
        const V cb = E::max(E::load(beg), E::subs(iv, w_v));
        const V ce = E::min(E::min(E::load(end), E::adds(E::adds(iv, w_v), one)), qlen_v);
        E::store(beg, cb);
        E::store(end, ce);
        for (int l = 0; l < W; ++l) term[l] = (l < lanes && !done[l] && i < tlen[l]) ? -1 : 0;
        const M tm = E::mload(term);
        const V cbm1 = E::subs(cb, one);
        V row_max = zero;
        for (int j = 0; j < qmax; ++j) {
            int16_t *hj = h + (size_t)j * W, *ej = e + (size_t)j * W;
            const V ht = E::load(hj), ep = E::load(ej);
            const V hdc = hd;
            hd = ht;
            const V s2 = E::load(q_soa + (size_t)j * W);
            V sc = E::blend(mis_v, match_v, E::eq(s1, s2));
            sc = E::blend(sc, amb_v, E::mor(E::gt(s2, three), E::gt(s1, three)));
            const V m = E::max(E::adds(hdc, sc), zero);
            const V ev = E::max(E::max(E::subs(m, oe_del), zero), E::subs(ep, e_del));
            f = E::max(E::max(E::subs(m, oe_ins), zero), E::subs(f, e_ins));
            V hv = E::max(E::max(E::max(m, ev), f), zero);
            const V jv = E::set1((int16_t)j);
            const M band = E::mand(E::gt(jv, cbm1), E::gt(ce, jv));
            const M keep = E::mand(band, tm);
            hv = E::keep(hv, keep);
            E::store(hj, hv);
            E::store(ej, E::keep(ev, keep));
            const M up = E::gt(hv, max_s);
            max_s = E::max(hv, max_s);
            max_i = E::blend(max_i, iv, up);
            max_j = E::blend(max_j, jv, up);
            row_max = E::max(row_max, hv);
        }
        if (p.zdrop > 0) {   // kernel_i16.rs:229-247
            E::store(ms, max_s);
            E::store(rm, row_max);
            for (int l = 0; l < lanes; ++l)
                if (!done[l] && i > 0 && i < tlen[l] && ms[l] - rm[l] > p.zdrop) { done[l] = true; ++n_done; }
        }
    }
    alignas(64) int16_t s[W], ti[W], tj[W];
    E::store(s, max_s);
    E::store(ti, max_i);
    E::store(tj, max_j);
    for (int l = 0; l < lanes; ++l) out[l] = OutScore{s[l], ti[l], tj[l]};
}

// -------------------------------------------------------- sw_kernel_with_ws restatement
// banded_swa/kernel.rs:29-284, one chunk, int8 lanes (every length <= 128).
template <class E>
void kernel_i8(const int8_t *q_soa, const int8_t *t_soa, const int8_t *qlen, const int8_t *tlen, const int8_t *h0,
               const int8_t *w, int lanes, int qmax, int tmax, const fa_params &p, int8_t *h, int8_t *e,
               OutScore *out) {
    constexpr int W = E::W;
    using V = typename E::V;
    using M = typename E::M;
    if (qmax == 0 || tmax == 0 || lanes == 0) return;
    const V zero = E::zero();
    const V match_v = E::set1(p.mat[0]), mis_v = E::set1(p.mat[1]);
    const V oe_del = E::set1((int8_t)(p.o_del + p.e_del)), oe_ins = E::set1((int8_t)(p.o_ins + p.e_ins));
    const V e_del = E::set1((int8_t)p.e_del), e_ins = E::set1((int8_t)p.e_ins), one = E::set1(1);
    memset(e, 0, (size_t)qmax * W);
    const V h0v = E::load(h0);
    E::store(h, h0v);
    V hp = E::subs(h0v, oe_ins);
    if (qmax > 1) E::store(h + W, hp);
    for (int j = 2; j < qmax; ++j) {
        hp = E::subs(hp, e_ins);
        E::store(h + (size_t)j * W, hp);
    }
    V max_s = h0v, max_i = zero, max_j = zero;
    alignas(64) int8_t beg[W], end[W], cur_b[W], cur_e[W], term[W], ms[W];
    bool done[W];
    int n_done = 0;
    for (int l = 0; l < W; ++l) { beg[l] = 0; end[l] = l < lanes ? qlen[l] : 0; done[l] = false; }
    const V qlen_v = E::load(qlen), w_v = E::load(w), beg_v = E::load(beg), end_v = E::load(end);
    for (int i = 0; i < tmax; ++i) {
        if (n_done > lanes / 2) break;   // kernel.rs:143-147
        V f = zero;
        V hd = E::load(h);
        const V s1 = E::load(t_soa + (size_t)i * W);
        const V iv = E::set1((int8_t)i);
        const V cb = E::max(beg_v, E::subs(iv, w_v));
        const V ce = E::minu(E::minu(end_v, E::adds(E::adds(iv, w_v), one)), qlen_v);
        E::store(cur_b, cb);
        E::store(cur_e, ce);
        for (int l = 0; l < W; ++l) term[l] = (l < lanes && !done[l] && i < (uint8_t)tlen[l]) ? -1 : 0;
        const M tm = E::mload(term);
        const V cbm1 = E::subs(cb, one);
        for (int j = 0; j < qmax; ++j) {
            int8_t *hj = h + (size_t)j * W, *ej = e + (size_t)j * W;
            const V ht = E::load(hj), ep = E::load(ej);
            const V hdc = hd;
            hd = ht;
            const V s2 = E::load(q_soa + (size_t)j * W);
            const V sc = E::blend(mis_v, match_v, E::eq(s1, s2));
            V m = E::adds(hdc, sc);
            m = E::blend(m, zero, E::msb(E::vor(s1, s2)));   // padding (0xFF) zeroes M
            m = E::max(m, zero);
            const V ev = E::max(E::subs(m, oe_del), E::subs(ep, e_del));
            f = E::max(E::subs(m, oe_ins), E::subs(f, e_ins));
            V hv = E::max(E::max(m, ev), f);
            const V jv = E::set1((int8_t)j);
            const M keep = E::mand(E::mand(E::gt(jv, cbm1), E::gt(ce, jv)), tm);
            hv = E::keep(hv, keep);
            E::store(hj, hv);
            E::store(ej, E::keep(ev, keep));
            const M up = E::gt(hv, max_s);
            max_s = E::max(hv, max_s);
            max_i = E::blend(max_i, iv, up);
            max_j = E::blend(max_j, jv, up);
        }
        E::store(ms, max_s);
        if (p.zdrop > 0) {   // kernel.rs:227-256: row max over the row's band from the stored row
            for (int l = 0; l < lanes; ++l) {
                if (done[l] || i == 0 || i >= (uint8_t)tlen[l]) continue;
                int8_t row_max = 0;
                for (int j = cur_b[l]; j < (uint8_t)cur_e[l]; ++j) row_max = std::max(row_max, h[(size_t)j * W + l]);
                if (row_max == 0 || (int)ms[l] - (int)row_max > p.zdrop) { done[l] = true; ++n_done; }
            }
        }
    }
    alignas(64) int8_t s[W], ti[W], tj[W];
    E::store(s, max_s);
    E::store(ti, max_i);
    E::store(tj, max_j);
    for (int l = 0; l < lanes; ++l) out[l] = OutScore{s[l], ti[l], tj[l]};
}

// ----------------------------------------------------- batch_ksw_align_avx2 restatement
// kswv_avx2.rs:93-641, one chunk: ref (target) and query SoA u8 (0xFF padding), nrow = the
// chunk's longest target, ncol its longest query; xtra = 0 for every lane (mate rescue passes
// h0 = 0, mate_rescue.rs:739).  Scoring: match / mismatch / ambiguous scores as the reference's
// mate-rescue batch passes them (mate_rescue.rs:713-719, ambig 0).
template <class E>
void kernel_kswv(const uint8_t *t_soa, const uint8_t *q_soa, int nrow, int ncol, const int32_t *rlen, int lanes,
                 int8_t w_match, int8_t w_mis, int8_t w_amb, int o_del, int e_del, int o_ins, int e_ins,
                 uint8_t *h0b, uint8_t *h1b, uint8_t *fb, uint8_t *rowmax, int16_t *te_all, fa_kswr *out) {
    constexpr int W = E::W;
    using V = typename E::V;
    using M = typename E::M;
    const V zero = E::zero(), one = E::set1(1);
    const int8_t mdiff = std::max(std::max(w_match, w_mis), w_amb);
    const int8_t shift_val = std::min(std::min(w_match, w_mis), w_amb);
    const uint8_t shift = (uint8_t)(256 - shift_val);
    int8_t tab[16] = {w_match, w_mis, w_mis, w_mis, w_amb, w_amb, w_amb, w_amb,
                      w_amb, w_amb, w_amb, w_amb, w_amb, 0, 0, 0};
    for (int k = 0; k < 16; ++k) tab[k] = (int8_t)(tab[k] + (int8_t)shift);
    const V perm = E::table(tab), sft = E::set1(shift), cmax = E::set1(255), five = E::set1(5);
    const V e_del_v = E::set1((uint8_t)e_del), oe_del_v = E::set1((uint8_t)(o_del + e_del));
    const V e_ins_v = E::set1((uint8_t)e_ins), oe_ins_v = E::set1((uint8_t)(o_ins + e_ins));
    const V minsc = zero, endsc = E::set1(255);   // xtra = 0: no XSUBO threshold, no XSTOP
    V gmax = zero;
    for (int l = 0; l < W; ++l) te_all[l] = -1;
    memset(h0b, 0, (size_t)(ncol + 1) * W);
    memset(h1b, 0, (size_t)(ncol + 1) * W);
    memset(fb, 0, (size_t)(ncol + 1) * W);
    memset(rowmax, 0, (size_t)(nrow + 1) * W);
    V pimax = zero, qe = zero;
    M mask = E::none(), minsc_m = E::none(), exit0 = E::all();
    int limit = nrow;
    for (int i = 0; i < nrow; ++i) {
        V e11 = zero, imax = zero, iqe = E::set1(255), lv = zero;
        const V s1 = E::load(t_soa + (size_t)i * W);
        for (int j = 0; j < ncol; ++j) {
            const V h00 = E::load(h0b + (size_t)j * W);
            const V s2 = E::load(q_soa + (size_t)j * W);
            const V f11 = E::load(fb + (size_t)(j + 1) * W);
            V sbt = E::shuffle(perm, E::vxor(s1, s2));
            sbt = E::blend(sbt, sft, E::eq(s2, five));
            V m11 = E::addsu(h00, sbt);
            m11 = E::blend(m11, zero, E::msb(E::vor(s1, s2)));
            m11 = E::subsu(m11, sft);
            V h11 = E::maxu(E::maxu(m11, e11), f11);
            const M up = E::gtu(h11, imax);
            imax = E::maxu(imax, h11);
            iqe = E::blend(iqe, lv, up);
            e11 = E::maxu(E::subsu(h11, oe_ins_v), E::subsu(e11, e_ins_v));
            const V f21 = E::maxu(E::subsu(h11, oe_del_v), E::subsu(f11, e_del_v));
            E::store(h1b + (size_t)(j + 1) * W, h11);
            E::store(fb + (size_t)(j + 1) * W, f21);
            lv = E::add(lv, one);
        }
        if (i > 0) {   // row maxima for the second best (kswv_avx2.rs:356-372)
            const M msk = E::mor(E::gtu(imax, pimax), mask);
            V pt = E::blend(pimax, zero, msk);
            pt = E::blend(pt, zero, exit0);
            E::store(rowmax + (size_t)(i - 1) * W, pt);
            mask = E::mandnot(msk, E::all());
        }
        pimax = imax;
        minsc_m = E::mor(minsc_m, E::geu(imax, minsc));
        const M upd = E::mand(E::gtu(imax, gmax), exit0);
        gmax = E::blend(gmax, imax, upd);
        qe = E::blend(qe, iqe, upd);
        uint64_t b = E::bits(upd);
        while (b) {   // te in 16-bit lanes (kswv_avx2.rs:381-420)
            const int l = __builtin_ctzll(b);
            te_all[l] = (int16_t)i;
            b &= b - 1;
        }
        const M stop = E::mor(E::geu(gmax, endsc), E::geu(E::addsu(gmax, sft), cmax));
        exit0 = E::mandnot(stop, exit0);
        if (!E::any(exit0)) {
            limit = i + 1;
            break;
        }
        std::swap(h0b, h1b);
    }
    {
        const V pf = E::blend(pimax, zero, mask);
        E::store(rowmax + (size_t)(limit - 1) * W, pf);
    }
    alignas(64) uint8_t sc[W], qa[W];
    E::store(sc, gmax);
    E::store(qa, qe);
    int live = 0;
    for (int l = 0; l < lanes; ++l) {
        const int s = (int)sc[l] + (int)shift < 255 ? sc[l] : 255;
        out[l] = fa_kswr{s, te_all[l], qa[l], 0, 0, 0, 0};
        if (s != 255) ++live;
    }
    if (live == 0) return;
    // second best over every other lane (kswv_avx2.rs:528-603): lane 2k's window sets the
    // bounds of the 16-bit slot k, which covers byte lanes 2k and 2k+1
    constexpr int H = W / 2;
    int16_t low[H], high[H], rl[H];
    int maxl = 0, minh = nrow;
    for (int k = 0; k < H; ++k) { low[k] = high[k] = rl[k] = 0; }
    for (int k = 0; k < H; ++k) {   // every slot, padding lanes included, as the reference
        const int li = 2 * k;
        const int val = ((int)sc[li] + mdiff - 1) / mdiff;
        low[k] = (int16_t)std::max(te_all[li] - val, 0);
        high[k] = (int16_t)std::min(te_all[li] + val, nrow - 1);
        rl[k] = (int16_t)rlen[li];
        if (qa[li] != 0) {
            maxl = std::max(maxl, (int)low[k]);
            minh = std::min(minh, (int)high[k]);
        }
    }
    uint8_t mx[W];
    int16_t te2[H];
    memset(mx, 0, sizeof mx);
    for (int k = 0; k < H; ++k) te2[k] = -1;
    // blendv on bytes: a row updates byte lane l when its slot's 16-bit test and the byte
    // test hold; te2's 16-bit slot takes the row in the byte halves whose byte test held
    auto scan_row = [&](int i, bool fwd) {
        const uint8_t *r = rowmax + (size_t)i * W;
        for (int l = 0; l < W; ++l) {
            const int k = l >> 1;
            const bool slot = fwd ? low[k] > i : (i > high[k] && rl[k] > i);
            if (slot && r[l] > mx[l]) {
                mx[l] = r[l];
                const uint16_t v = (uint16_t)te2[k];
                te2[k] = (int16_t)((l & 1) ? ((v & 0x00FFu) | ((uint16_t)i & 0xFF00u))
                                           : ((v & 0xFF00u) | ((uint16_t)i & 0x00FFu)));
            }
        }
    };
    for (int i = 0; i < maxl; ++i) scan_row(i, true);
    for (int i = std::max(minh + 1, 0); i < limit; ++i) scan_row(i, false);
    for (int l = 0; l < lanes; ++l) {
        fa_kswr &o = out[l];
        if (qa[l] != 0) {
            o.score2 = mx[l] == 0 ? -1 : mx[l];
            o.te2 = te2[l / 2];
        } else {
            o.score2 = -1;
            o.te2 = -1;
        }
        if (o.score > 0 && o.te >= 0 && o.qe >= 0) {   // tb/qb estimated (kswv_avx2.rs:627-637)
            o.qb = 0;
            o.tb = std::max(o.te - o.qe, 0);
        } else {
            o.tb = -1;
            o.qb = -1;
        }
    }
}

// ------------------------------------------------------------------ chunk drivers

template <class F>
void parallel_chunks(uint32_t n_chunks, int nthreads, F &&body) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    nthreads = (int)std::min<uint32_t>((uint32_t)nthreads, std::max(1u, n_chunks));
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const uint32_t c = next.fetch_add(1);
            if (c >= n_chunks) break;
            body(c);
        }
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < nthreads; ++t) ts.emplace_back(worker);
    worker();
    for (auto &t : ts) t.join();
}

// Banded extension over all jobs: the i8 kernel when no job is longer than 128 (query or
// target), else the i16 kernel; chunks of W consecutive jobs.
template <class E16, class E8>
int ext_batch(const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq, const uint8_t *tseq,
              int32_t *out3, int nthreads, int force_i16) {
    int max_len = 0;
    for (uint32_t k = 0; k < n; ++k) max_len = std::max(max_len, std::max(jobs[k].qlen, jobs[k].tlen));
    const bool use_i8 = max_len <= 128 && !force_i16;
    const int W = use_i8 ? E8::W : E16::W;
    const uint32_t n_chunks = (n + W - 1) / W;
    parallel_chunks(n_chunks, nthreads, [&](uint32_t c) {
        thread_local std::vector<int16_t> q16, t16, h16, e16;
        thread_local std::vector<int8_t> q8, t8, h8, e8;
        const uint32_t b = c * (uint32_t)W;
        const int lanes = (int)std::min<uint32_t>((uint32_t)W, n - b);
        int mq = 0, mt = 0;
        for (int l = 0; l < lanes; ++l) { mq = std::max(mq, jobs[b + l].qlen); mt = std::max(mt, jobs[b + l].tlen); }
        OutScore os[64];
        if (use_i8) {
            alignas(64) int8_t ql[64] = {}, tl[64] = {}, hh[64] = {}, ww[64] = {};
            q8.assign((size_t)mq * W, (int8_t)0xFF);
            t8.assign((size_t)mt * W, (int8_t)0xFF);
            h8.resize((size_t)std::max(mq, 1) * W);
            e8.resize((size_t)std::max(mq, 1) * W);
            for (int l = 0; l < lanes; ++l) {
                const fa_job &jb = jobs[b + l];
                for (int j = 0; j < jb.qlen; ++j) q8[(size_t)j * W + l] = (int8_t)qseq[jb.q_off + j];
                for (int i = 0; i < jb.tlen; ++i) t8[(size_t)i * W + l] = (int8_t)tseq[jb.t_off + i];
                // int8 lane scalars, lengths clamped to 127 (batch_extension/dispatch.rs:126-131)
                ql[l] = (int8_t)std::min(jb.qlen, 127); tl[l] = (int8_t)std::min(jb.tlen, 127);
                hh[l] = (int8_t)jb.h0; ww[l] = (int8_t)jb.w;
            }
            kernel_i8<E8>(q8.data(), t8.data(), ql, tl, hh, ww, lanes, mq, mt, *p, h8.data(), e8.data(), os);
        } else {
            alignas(64) int16_t ql[64] = {}, tl[64] = {}, hh[64] = {}, ww[64] = {};
            q16.assign((size_t)mq * W, (int16_t)0xFF);
            t16.assign((size_t)mt * W, (int16_t)0xFF);
            h16.resize((size_t)std::max(mq, 1) * W);
            e16.resize((size_t)std::max(mq, 1) * W);
            for (int l = 0; l < lanes; ++l) {
                const fa_job &jb = jobs[b + l];
                for (int j = 0; j < jb.qlen; ++j) q16[(size_t)j * W + l] = qseq[jb.q_off + j];
                for (int i = 0; i < jb.tlen; ++i) t16[(size_t)i * W + l] = tseq[jb.t_off + i];
                ql[l] = (int16_t)jb.qlen; tl[l] = (int16_t)jb.tlen; hh[l] = (int16_t)jb.h0;
                ww[l] = (int16_t)(int8_t)jb.w;   // band carried as the reference's int8 field
            }
            kernel_i16<E16>(q16.data(), t16.data(), ql, tl, hh, ww, lanes, mq, mt, *p, h16.data(), e16.data(), os);
        }
        for (int l = 0; l < lanes; ++l) {
            out3[3 * (size_t)(b + l)] = os[l].score;
            out3[3 * (size_t)(b + l) + 1] = os[l].te;
            out3[3 * (size_t)(b + l) + 2] = os[l].qe;
        }
    });
    return use_i8 ? 8 : 16;
}

template <class E>
void kswv_batch(const fa_mate_job *jobs, uint32_t n, const uint8_t *qseq, const uint8_t *tseq, fa_kswr *out,
                int nthreads) {
    constexpr int W = E::W;
    const uint32_t n_chunks = (n + W - 1) / W;
    parallel_chunks(n_chunks, nthreads, [&](uint32_t c) {
        thread_local std::vector<uint8_t> q, t, h0, h1, f, rm;
        const uint32_t b = c * (uint32_t)W;
        const int lanes = (int)std::min<uint32_t>((uint32_t)W, n - b);
        int mq = 0, mt = 0;
        int32_t rl[W] = {};
        int16_t te[W];
        for (int l = 0; l < lanes; ++l) { mq = std::max(mq, jobs[b + l].qlen); mt = std::max(mt, jobs[b + l].tlen); }
        if (mq == 0 || mt == 0) {
            for (int l = 0; l < lanes; ++l) out[b + l] = fa_kswr{0, -1, 0, -1, -1, -1, -1};
            return;
        }
        q.assign((size_t)mq * W, 0xFF);
        t.assign((size_t)mt * W, 0xFF);
        h0.resize((size_t)(mq + 1) * W);
        h1.resize((size_t)(mq + 1) * W);
        f.resize((size_t)(mq + 1) * W);
        rm.resize((size_t)(mt + 1) * W);
        for (int l = 0; l < lanes; ++l) {
            const fa_mate_job &jb = jobs[b + l];
            for (int j = 0; j < jb.qlen; ++j) q[(size_t)j * W + l] = qseq[jb.q_off + j];
            for (int i = 0; i < jb.tlen; ++i) t[(size_t)i * W + l] = tseq[jb.t_off + i];
            rl[l] = jb.tlen;
        }
        kernel_kswv<E>(t.data(), q.data(), mt, mq, rl, lanes, 1, -4, 0, 6, 1, 6, 1, h0.data(), h1.data(), f.data(),
                       rm.data(), te, out + b);
    });
}

}  // namespace

// ------------------------------------------------------------------ C entry points
// Per build: FA_ISA 1 exports the *_avx2 and *_port entries, FA_ISA 2 the *_avx512 ones.

extern "C" {

#if FA_ISA == 1
int simd_ext_batch_avx2(const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq,
                        const uint8_t *tseq, int32_t *out3, int nthreads, int force_i16) {
    return ext_batch<I16Avx2, I8Avx2>(p, jobs, n, qseq, tseq, out3, nthreads, force_i16);
}
// int16 kernel on the portable 8-lane engine (no int8 path): the lane-by-lane check
int simd_ext_batch_port(const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq,
                        const uint8_t *tseq, int32_t *out3, int nthreads) {
    return ext_batch<I16Port, I8Avx2>(p, jobs, n, qseq, tseq, out3, nthreads, 1);
}
void simd_kswv_batch_avx2(const fa_mate_job *jobs, uint32_t n, const uint8_t *qseq, const uint8_t *tseq,
                          fa_kswr *out, int nthreads) {
    kswv_batch<U8Avx2>(jobs, n, qseq, tseq, out, nthreads);
}
// One chunk of the int8 kernel on caller-made SoA inputs, as the reference's kernel tests
// call sw_kernel (tests/kernel_optimization_test.rs); lanes <= 32, out3 = score, te, qe.
int simd_i8_chunk_avx2(const uint8_t *q_soa, const uint8_t *t_soa, const int8_t *qlen, const int8_t *tlen,
                       const int8_t *h0, const int8_t *w, int lanes, int max_q, int max_t, const fa_params *p,
                       int32_t *out3) {
    if (lanes < 0 || lanes > I8Avx2::W) return -1;
    alignas(64) int8_t ql[I8Avx2::W] = {}, tl[I8Avx2::W] = {}, hh[I8Avx2::W] = {}, ww[I8Avx2::W] = {};
    for (int l = 0; l < lanes; ++l) { ql[l] = qlen[l]; tl[l] = tlen[l]; hh[l] = h0[l]; ww[l] = w[l]; }
    std::vector<int8_t> h((size_t)std::max(max_q, 1) * I8Avx2::W), e(h.size());
    std::vector<int8_t> q((size_t)max_q * I8Avx2::W, (int8_t)0xFF), t((size_t)max_t * I8Avx2::W, (int8_t)0xFF);
    // the caller's SoA has stride `lanes`; re-stride it to the engine's width
    for (int j = 0; j < max_q; ++j)
        for (int l = 0; l < lanes; ++l) q[(size_t)j * I8Avx2::W + l] = (int8_t)q_soa[(size_t)j * lanes + l];
    for (int i = 0; i < max_t; ++i)
        for (int l = 0; l < lanes; ++l) t[(size_t)i * I8Avx2::W + l] = (int8_t)t_soa[(size_t)i * lanes + l];
    OutScore os[I8Avx2::W];
    for (auto &o : os) o = OutScore{0, 0, 0};
    kernel_i8<I8Avx2>(q.data(), t.data(), ql, tl, hh, ww, lanes, max_q, max_t, *p, h.data(), e.data(), os);
    for (int l = 0; l < lanes; ++l) { out3[3 * l] = os[l].score; out3[3 * l + 1] = os[l].te; out3[3 * l + 2] = os[l].qe; }
    return 0;
}
#endif

#if FA_ISA == 2
int simd_ext_batch_avx512(const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq,
                          const uint8_t *tseq, int32_t *out3, int nthreads, int force_i16) {
    return ext_batch<I16Avx512, I8Avx512>(p, jobs, n, qseq, tseq, out3, nthreads, force_i16);
}
void simd_kswv_batch_avx512(const fa_mate_job *jobs, uint32_t n, const uint8_t *qseq, const uint8_t *tseq,
                            fa_kswr *out, int nthreads) {
    kswv_batch<U8Avx512>(jobs, n, qseq, tseq, out, nthreads);
}
#endif

}  // extern "C"
