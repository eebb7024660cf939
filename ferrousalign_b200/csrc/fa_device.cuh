// fa_device.cuh -- device-side types and helpers shared by the B200 kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ferrous_b200.h"

namespace fa {

// Device status word bits (written with atomicOr, read back by the host).
enum : uint32_t {
    ST_BAD_CODE = 1u << 0,   // a sequence byte >= alphabet size
    ST_CAPACITY = 1u << 1,   // a job exceeded the launch's length limit
    ST_BLIST    = 1u << 2,   // mate-SW run list overflowed its buffer
    ST_ARG      = 1u << 3,   // a job violates an argument rule (h0 <= 0, qlen <= 0, tlen < 0)
    ST_RANGE    = 1u << 4,   // a chain's seed range is malformed (region merge)
    ST_RUNS     = 1u << 5,   // a packed buffer's N runs are empty, unsorted, overlapping or past its bases
};

// Base (0-3) of FM-index position x < 2 l_pac in a 2-bit packed reference (the .pac layout:
// base k in bits 7-6 of byte k/4 when k % 4 == 0 down to bits 1-0 when k % 4 == 3; positions
// at or past l_pac are the reverse complement of forward position 2 l_pac - 1 - x).
__device__ __forceinline__ uint8_t pac_base(const uint8_t *__restrict__ pac, uint64_t l_pac, uint64_t x) {
    const bool rev = x >= l_pac;
    const uint64_t f = rev ? (l_pac << 1) - 1 - x : x;
    const uint8_t b = (pac[f >> 2] >> ((~(uint32_t)f & 3u) << 1)) & 3u;
    return rev ? (uint8_t)(3u - b) : b;
}

// Scoring parameters in the form the extension kernel consumes.
struct ExtParams {
    int8_t  mat[25];
    int32_t m;
    int32_t o_del, e_del, o_ins, e_ins;
    int32_t zdrop, end_bonus;
    int32_t max_score;      // max(0, max(mat))  (ksw_affine_gap.rs:1000-1005)
    int32_t flags;          // fa_params.flags (FA_PARAM_*)
};

struct MateParams {
    int8_t  mat[25];
    int32_t m;
    int32_t o_del, e_del, o_ins, e_ins;
    int32_t shift, max;     // ksw_qinit shift / max (ksw_affine_gap.rs:88-101)
};

// Rust `f64 as i32`: truncation toward zero with saturation, NaN -> 0.
__host__ __device__ inline int32_t rust_f64_as_i32(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return static_cast<int32_t>(x);
}

// Band after the max_ins / max_del clamp of ksw_extend2 (ksw_affine_gap.rs:1007-1018),
// evaluated in the same double-precision order as the reference.
__host__ __device__ inline int32_t ext_band_clamp(int32_t qlen, int32_t w, const ExtParams &p) {
    int32_t max_ins = rust_f64_as_i32(((double)qlen * (double)p.max_score + (double)p.end_bonus -
                                       (double)p.o_ins) / (double)p.e_ins + 1.0);
    if (max_ins < 1) max_ins = 1;
    if (w > max_ins) w = max_ins;
    int32_t max_del = rust_f64_as_i32(((double)qlen * (double)p.max_score + (double)p.end_bonus -
                                       (double)p.o_del) / (double)p.e_del + 1.0);
    if (max_del < 1) max_del = 1;
    if (w > max_del) w = max_del;
    return w;
}

// ksw_extend2 run as written on a job with h0 == 0 (FA_PARAM_H0_ZERO; the reference asserts
// h0 > 0 at ksw_affine_gap.rs:968).  The first row is then all zero (eh[0].h = h0 = 0 and
// eh[1].h = 0, :1017-1025), so every M is 0 (`M ? M + s : 0`, :1066-1071) and every H, E
// and F of row 0 is 0: the row maximum is 0 and the loop breaks after row 0 (:1122), which
// sets gscore = 0 and max_ie = 0 only when row 0's band reaches the query end (:1109-1120,
// end = min(qlen, w + 1) with the clamped band w).  `w` is the band after ext_band_clamp.
// Returns the cells row 0 visited (end - beg), 0 when tlen == 0 (no row runs).
__host__ __device__ inline uint32_t ext_h0_zero_result(int32_t qlen, int32_t tlen, int32_t w, fa_ext_result *r) {
    r->score = 0;
    r->qle = 0;
    r->tle = 0;
    r->max_off = 0;
    r->gscore = -1;
    r->gtle = 0;
    if (tlen <= 0) return 0;
    const int32_t end = qlen < w + 1 ? qlen : w + 1;
    if (end == qlen) {
        r->gscore = 0;
        r->gtle = 1;
    }
    return (uint32_t)end;
}

}  // namespace fa
