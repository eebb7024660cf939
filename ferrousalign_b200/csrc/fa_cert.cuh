// fa_cert.cuh -- the exit-bound certificate's accumulator, shared by the extension kernels.
#pragma once

#include <cstdint>

namespace fa {

// Exit-bound certificate (CERT = true).  A path that leaves the run's computed
// region first steps onto a gap cell the run itself evaluates: the F value just past
// a row's end, the E value of a column the band drops on the left, the first column
// when the band leaves it, or the first row beyond the band.  From such an exit of
// value x at (ix, jx) the path reaches row i with a score of at most
//     min(x + a*(i-ix), x + a*D - e_del*(i-ix-D)),   D = qlen-1-jx,  a = max(mat),
// a tent in i.  P1/P3 hold, per side (right exits, left exits), the maxima of the
// two lines' intercepts.  The run's outputs are those of every wider run when:
//   * every row up to the last max / gscore event has its row max above the bound
//     (so row maxima, their first columns and the z-drop decisions agree),
//   * the bound stays below min(score, gscore) on every processed row, and on the
//     rows a wider run could still process after a zero row,
//   * a z-drop break row passes the first test too (a wider run breaks there),
//   * the run never read a column no earlier row wrote (a first-row value standing in
//     for a later row), and the wider band's first row covers every positive
//     first-row value (so neither run does).
// Widening is monotone in every cell, so the wider run sees the same values inside
// this run's region, raised only by exiting paths, which the tents bound.
struct ExitBound {
    static constexpr int NEG = -(1 << 29);
    int p1[2], p3[2];
    __host__ __device__ __forceinline__ void init() { p1[0] = p1[1] = p3[0] = p3[1] = NEG; }
    __host__ __device__ __forceinline__ void add(int side, int x, int ix, int jx, int qlen, int a, int e_del) {
        if (x > 0) {
            const int D = qlen - 1 - jx;
            p1[side] = max(p1[side], x - a * ix);
            p3[side] = max(p3[side], x + (a + e_del) * D + e_del * ix);
        }
    }
    __host__ __device__ __forceinline__ void merge(const ExitBound &o) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            p1[s] = max(p1[s], o.p1[s]);
            p3[s] = max(p3[s], o.p3[s]);
        }
    }
    __host__ __device__ __forceinline__ int at(int i, int a, int e_del) const {
        int b = NEG;
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (p1[s] != NEG) b = max(b, min(p1[s] + a * i, p3[s] - e_del * i));
        return b;
    }
    // max over integer rows i0..i1 of at(i): each tent is concave, so its maximum over
    // the interval sits at the integer rows beside the crossing of its two lines
    __host__ __device__ __forceinline__ int max_over(int i0, int i1, int a, int e_del) const {
        int b = NEG;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (p1[s] == NEG) continue;
            int c = i1;
            if (a + e_del > 0) {
                const int num = p3[s] - p1[s], den = a + e_del;
                c = num >= 0 ? num / den : -((-num + den - 1) / den);   // floor
            }
#pragma unroll
            for (int d = 0; d < 2; ++d) {
                const int k = min(max(c + d, i0), i1);
                b = max(b, min(p1[s] + a * k, p3[s] - e_del * k));
            }
        }
        return b;
    }
};

}  // namespace fa
