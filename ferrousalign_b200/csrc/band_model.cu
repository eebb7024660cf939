// band_model.cu -- the learned band predictor: feature extraction, a 16-64-32-1 MLP
// (BF16 weights, FP32 accumulation) and its training kernels.
//
// The predictor guesses, per extension, the narrowest band that reproduces the full-band
// result, from facts available before the DP runs: seed length, query/target lengths,
// h0, the chain's seed-diagonal spread and mismatch counts along the seed diagonal and
// its neighbours.  The extension kernels then start at the predicted band and the
// band-retry policy (policy_kernel.cu) accepts or widens it.
//
// Training: quantile (pinball) loss on log2(band) so the prediction sits above most
// labels; per-block minibatch backward with the activations in shared memory and
// gradient products computed from them, then Adam on FP32 master weights with a BF16
// copy for inference.

#include <cuda_bf16.h>

#include "fa_device.cuh"
#include "fa_kernels.h"

namespace fa {

// ---------------------------------------------------------------- features
// x[0..15] per job (raw, normalised later by the model):
//  0 seed length (h0 / max score)   1 qlen
//  2 query end - last mismatch on the seed diagonal     3 the same on the best shifted diagonal
//  4 seed-diagonal spread (hint)    5 has partner     6 mismatching 8-blocks on the diagonal
//  7 their fraction                 8 first mismatching block / blocks
//  9 mismatching blocks in the last quarter           10 diagonal mismatches / positions
// 11 longest matching block run / blocks              12 N bases in the query
// 13 tlen - qlen                    14 |best shift| of the second half (diagonals -4..4)
// 15 mismatch fraction of the second half on that best shifted diagonal
// One thread per job, 16 positions per step as four 32-bit words: the query bytes and a
// 28-byte target window are read as aligned words and realigned with funnel shifts;
// byte-wise SIMD compares (__vcmpne4, __vcmpgtu4) give one 0xFF byte per mismatching
// position, masked to the valid position range, and counts / last positions come from
// popc / clz.  The valid range of each shifted diagonal is known in closed form, so only
// its mismatches are counted.  Sequence buffers carry kSeqPad bytes of padding, so the
// word holding a buffer's last byte is always inside the allocation.
__device__ __forceinline__ uint32_t byte_range_mask(int p0, int lo, int hi)
{
    const int a = min(max(lo - p0, 0), 4), b = min(max(hi - p0, 0), 4);
    const uint32_t hm = b >= 4 ? 0xFFFFFFFFu : (1u << (8 * b)) - 1u;
    const uint32_t lm = a >= 4 ? 0xFFFFFFFFu : (1u << (8 * a)) - 1u;
    return hm & ~lm;
}

__device__ __forceinline__ uint32_t word_at(const uint8_t *__restrict__ base, long long byte_addr, uint64_t bytes)
{
    return (byte_addr >= 0 && (uint64_t)byte_addr < bytes)
               ? __ldg(reinterpret_cast<const uint32_t *>(base + byte_addr)) : 0u;
}

__device__ __forceinline__ int last_byte(uint32_t m) { return (31 - __clz(m)) >> 3; }

// PK: 2-bit packed sequences, read through PackedReader (positions outside the job come
// back as 0 there, where the byte form reads the neighbouring bytes; every use below masks
// them, so the features are the same).
// order (optional): a permutation of the n jobs that the threads take in turn -- a
// length-sorted one keeps a warp's 32 loops the same length.
template <bool PK>
__global__ void __launch_bounds__(128) band_features_kernel(const fa_job *__restrict__ jobs, uint32_t n,
                                                            const SeqBuf qs, const SeqBuf ts,
                                                            const fa_band_hint *__restrict__ hints, int max_score,
                                                            float *__restrict__ x, const uint32_t *__restrict__ order)
{
    const uint8_t *__restrict__ qseq = qs.p;
    const uint8_t *__restrict__ tseq = ts.p;
    const uint64_t qbytes = qs.nbytes, tbytes = ts.nbytes;
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= n) return;
    const uint32_t i = order ? order[gi] : gi;
    const fa_job jb = jobs[i];
    const int qlen = jb.qlen, tlen = jb.tlen;
    const int L = min(qlen, tlen);
    const int nblk = (L + 7) / 8;
    const int half = qlen / 2;
    int lo[9], hi[9], c[9], last_s[9];
#pragma unroll
    for (int s = 0; s < 9; ++s) {
        const int sh = s - 4;
        lo[s] = max(half, -sh);
        hi[s] = min(qlen, tlen - sh);
        c[s] = 0;
        last_s[s] = -1;
    }
    int mm = 0, last_mm = -1, nq = 0, mmblk = 0, first = -1, lastq = 0, best_run = 0, run = 0;
    PackedReader qr, tr;
    if (PK) {
        qr.init(qs, jb.q_off, qlen);
        tr.init(ts, jb.t_off, tlen);
    }
    for (int k0 = 0; k0 < qlen; k0 += 16) {
        uint32_t q4[4], nm[4], t7[7];
        if (PK) {
            qr.getw<4>(k0, q4);
            tr.getw<7>(k0 - 4, t7);   // target positions k0-4 .. k0+23
        } else {
            {
                const long long a = (long long)jb.q_off + k0, a0 = a & ~3LL;
                const int sh = (int)(a - a0) * 8;
                uint32_t w[5];
#pragma unroll
                for (int m = 0; m < 5; ++m) w[m] = word_at(qseq, a0 + 4 * m, qbytes);
#pragma unroll
                for (int m = 0; m < 4; ++m) q4[m] = __funnelshift_r(w[m], w[m + 1], sh);
            }
            {
                const long long a = (long long)jb.t_off + k0 - 4, a0 = a & ~3LL;   // target bytes k0-4 .. k0+23
                const int sh = (int)(a - a0) * 8;
                uint32_t w[8];
#pragma unroll
                for (int m = 0; m < 8; ++m) w[m] = word_at(tseq, a0 + 4 * m, tbytes);
#pragma unroll
                for (int m = 0; m < 7; ++m) t7[m] = __funnelshift_r(w[m], w[m + 1], sh);
            }
        }
        uint32_t dmask[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int p0 = k0 + 4 * m;
            nm[m] = __vcmpgtu4(q4[m], 0x03030303u);                     // N in the query
            nq += __popc(nm[m] & byte_range_mask(p0, 0, qlen)) >> 3;
            const uint32_t d = (__vcmpne4(q4[m], t7[m + 1]) | nm[m]) & byte_range_mask(p0, 0, L);
            dmask[m] = d;
            mm += __popc(d) >> 3;
            if (d) last_mm = p0 + last_byte(d);
        }
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) {                                // 8-position blocks
            const int bidx = k0 / 8 + bb;
            if (bidx < nblk) {
                if (dmask[2 * bb] | dmask[2 * bb + 1]) {
                    ++mmblk;
                    if (first < 0) first = bidx;
                    if (bidx * 4 >= nblk * 3) ++lastq;
                    run = 0;
                } else {
                    best_run = max(best_run, ++run);
                }
            }
        }
        if (k0 + 16 > half) {
#pragma unroll
            for (int s = 0; s < 9; ++s) {                               // target shifted by s - 4
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int p0 = k0 + 4 * m;
                    const uint32_t rm = byte_range_mask(p0, lo[s], hi[s]);
                    // bytes T[p0 + s - 4 ..]: offset 4m + s in the window
                    const int wi = m + s / 4;
                    const uint32_t tw = __funnelshift_r(t7[wi], t7[wi + 1], 8 * (s % 4));
                    const uint32_t dd = (__vcmpne4(q4[m], tw) | nm[m]) & rm;
                    c[s] += __popc(dd) >> 3;
                    if (dd) last_s[s] = p0 + last_byte(dd);
                }
            }
        }
    }
    // shifted diagonal with the lowest mismatch fraction (ties: the smaller shift)
    int best_s = 0, best_c = -1, best_n = 1, best_last = -1;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
        const int ns = max(0, hi[s] - lo[s]);
        const int sh = s - 4;
        const long long lhs = (long long)c[s] * best_n, rhs = (long long)best_c * ns;
        if (ns > 0 && (best_c < 0 || lhs < rhs || (lhs == rhs && abs(sh) < abs(best_s)))) {
            best_c = c[s]; best_n = ns; best_s = sh; best_last = last_s[s];
        }
    }
    float o[16];
    const float fb = (float)max(nblk, 1);
    o[0] = max_score > 0 ? (float)jb.h0 / (float)max_score : (float)jb.h0;
    o[1] = (float)qlen;
    o[2] = (float)(qlen - last_mm);
    o[3] = (float)(qlen - max(best_last, half - 1));
    o[4] = hints ? (float)hints[i].diag_spread : 0.f;
    o[5] = hints ? (float)(hints[i].has_partner != 0) : 0.f;
    o[6] = (float)mmblk;
    o[7] = (float)mmblk / fb;
    o[8] = first < 0 ? 1.f : (float)first / fb;
    o[9] = (float)lastq;
    o[10] = (float)mm / (float)max(L, 1);
    o[11] = (float)best_run / fb;
    o[12] = (float)nq;
    o[13] = (float)(tlen - qlen);
    o[14] = (float)abs(best_s);
    o[15] = best_c < 0 ? 1.f : (float)best_c / (float)best_n;
    float4 *xo = reinterpret_cast<float4 *>(x + (size_t)i * 16);
#pragma unroll
    for (int k = 0; k < 4; ++k) xo[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
}

cudaError_t launch_band_features(const fa_job *d_jobs, uint32_t n, const SeqBuf &d_q, const SeqBuf &d_t,
                                 const fa_band_hint *d_hints, int max_score, float *d_x, cudaStream_t s,
                                 const uint32_t *d_order)
{
    if (n == 0) return cudaSuccess;
    if (d_q.packed)
        band_features_kernel<true><<<(n + 127) / 128, 128, 0, s>>>(d_jobs, n, d_q, d_t, d_hints, max_score, d_x,
                                                                   d_order);
    else
        band_features_kernel<false><<<(n + 127) / 128, 128, 0, s>>>(d_jobs, n, d_q, d_t, d_hints, max_score, d_x,
                                                                    d_order);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- MLP
// Parameter layout (floats): W1[64][16] b1[64] W2[32][64] b2[32] W3[32] b3[1]
constexpr int kIn = 16, kH1 = 64, kH2 = 32;
constexpr int oW1 = 0, oB1 = oW1 + kH1 * kIn, oW2 = oB1 + kH1, oB2 = oW2 + kH2 * kH1, oW3 = oB2 + kH2,
              oB3 = oW3 + kH2, kNParams = oB3 + 1;
static_assert(kNParams == FA_BAND_NPARAMS, "parameter count");

struct NormConsts {
    float mean[kIn], inv_std[kIn];
};

// forward of one sample with weights staged in shared memory as float
// Every loop is fully unrolled so h1/h2 stay in registers.
__device__ __forceinline__ float mlp_forward(const float *__restrict__ w, const float *x, float *h1, float *h2)
{
#pragma unroll
    for (int u = 0; u < kH1; ++u) {
        float a = w[oB1 + u];
#pragma unroll
        for (int k = 0; k < kIn; ++k) a = fmaf(w[oW1 + u * kIn + k], x[k], a);
        h1[u] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int u = 0; u < kH2; ++u) {
        float a = w[oB2 + u];
#pragma unroll
        for (int k = 0; k < kH1; ++k) a = fmaf(w[oW2 + u * kH1 + k], h1[k], a);
        h2[u] = fmaxf(a, 0.f);
    }
    float y = w[oB3];
#pragma unroll
    for (int k = 0; k < kH2; ++k) y = fmaf(w[oW3 + k], h2[k], y);
    return y;
}

__device__ __forceinline__ void load_norm(const float *__restrict__ xr, const NormConsts &nc, float *x)
{
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[k] = (xr[k] - nc.mean[k]) * nc.inv_std[k];
}

// Forward of two samples at once: every weight comes from shared memory once for both, and
// layer 2 accumulates as each layer-1 unit is done (W2 transposed in w2t, so its reads are
// contiguous).  Each sum runs in the same order as mlp_forward's, so the outputs are the same.
__device__ __forceinline__ void mlp_forward2(const float *__restrict__ w, const float *__restrict__ w2t,
                                             const float *x0, const float *x1, float &y0, float &y1)
{
    float a0[kH2], a1[kH2];
#pragma unroll
    for (int v = 0; v < kH2; ++v) a0[v] = a1[v] = w[oB2 + v];
#pragma unroll 2
    for (int u = 0; u < kH1; ++u) {
        float s0 = w[oB1 + u], s1 = s0;
#pragma unroll
        for (int k = 0; k < kIn; ++k) {
            const float wk = w[oW1 + u * kIn + k];
            s0 = fmaf(wk, x0[k], s0);
            s1 = fmaf(wk, x1[k], s1);
        }
        s0 = fmaxf(s0, 0.f);
        s1 = fmaxf(s1, 0.f);
#pragma unroll
        for (int v = 0; v < kH2; ++v) {
            const float wv = w2t[u * kH2 + v];
            a0[v] = fmaf(wv, s0, a0[v]);
            a1[v] = fmaf(wv, s1, a1[v]);
        }
    }
    y0 = y1 = w[oB3];
#pragma unroll
    for (int k = 0; k < kH2; ++k) {
        const float wk = w[oW3 + k];
        y0 = fmaf(wk, fmaxf(a0[k], 0.f), y0);
        y1 = fmaf(wk, fmaxf(a1[k], 0.f), y1);
    }
}

// Inference: y = MLP(x) in log2(band) units; band = ceil(2^(y + margin)) raised to
// w_min and rounded up to the ladder 2, 3, 4, 6, 8, 12, ... (bands of one launch fall
// into few classes, which the band partition turns into uniform warps; doubling after a
// rejection stays on the ladder).  A band above half the configured band starts at the
// configured band: its narrow run would save less than half the cells, and a rejected one
// costs more than starting wide.  Each thread predicts two jobs, i and i + blockDim.x.
constexpr int kPredThreads = 128;
__global__ void __launch_bounds__(kPredThreads) band_predict_kernel(
    const __nv_bfloat16 *__restrict__ wbf, NormConsts nc, const float *__restrict__ x,
    const fa_job *__restrict__ jobs, uint32_t n, float margin, int w_min, float *__restrict__ y_out,
    int32_t *__restrict__ w_out)
{
    __shared__ __align__(16) float w[kNParams];
    __shared__ __align__(16) float w2t[kH1 * kH2];
    for (int k = threadIdx.x; k < kNParams; k += blockDim.x) w[k] = __bfloat162float(wbf[k]);
    for (int k = threadIdx.x; k < kH1 * kH2; k += blockDim.x) {
        const int u = k / kH2, v = k % kH2;
        w2t[k] = __bfloat162float(wbf[oW2 + v * kH1 + u]);
    }
    __syncthreads();
    const uint32_t i0 = blockIdx.x * (2 * kPredThreads) + threadIdx.x, i1 = i0 + kPredThreads;
    if (i0 >= n) return;
    float x0[kIn], x1[kIn];
    load_norm(x + (size_t)i0 * kIn, nc, x0);
    if (i1 < n) load_norm(x + (size_t)i1 * kIn, nc, x1);
    else
#pragma unroll
        for (int k = 0; k < kIn; ++k) x1[k] = 0.f;
    float y0, y1;
    mlp_forward2(w, w2t, x0, x1, y0, y1);
    auto put = [&](uint32_t i, float y) {
        if (y_out) y_out[i] = y;
        if (w_out) {
            const int wj = jobs ? jobs[i].w : 100;
            const float e = fminf(fmaxf(y + margin, 0.f), 16.f);
            int band = (int)ceilf(exp2f(e));
            band = max(band, w_min);
            if (band > 2) {                 // up to the ladder 2^k, 3*2^(k-1): few distinct bands per launch
                const int p2 = 1 << (32 - __clz(band - 1));
                band = 3 * p2 / 4 >= band ? 3 * p2 / 4 : p2;
            }
            if (2 * band > wj) band = wj;   // a narrow run above half the configured band saves too little
            band = min(band, wj);
            w_out[i] = band;
        }
    };
    put(i0, y0);
    if (i1 < n) put(i1, y1);
}

// Backward over one minibatch of up to kMB samples per block: activations in shared
// memory, then every thread accumulates a slice of the gradient as sums over the
// block's samples.  Loss: pinball(tau) on y - target, averaged over `n_total`.
constexpr int kMB = 128;
struct BwdSmem {             // rows padded by one float so per-sample rows map to distinct banks
    float w[kNParams];
    float x[kMB][kIn + 1];
    float h1[kMB][kH1 + 1];
    float h2[kMB][kH2 + 1];
    float d2[kMB][kH2 + 1];   // dL/d(pre-activation of layer 2)
    float d1[kMB][kH1 + 1];   // dL/d(pre-activation of layer 1)
    float dy[kMB];
};

__global__ void __launch_bounds__(kMB) band_backward_kernel(const __nv_bfloat16 *__restrict__ wbf, NormConsts nc,
                                                            const float *__restrict__ x, const float *__restrict__ target,
                                                            uint32_t n, float tau, float inv_total,
                                                            float *__restrict__ grad, float *__restrict__ loss_sum)
{
    extern __shared__ __align__(16) unsigned char bsm_raw[];
    BwdSmem &S = *reinterpret_cast<BwdSmem *>(bsm_raw);
    for (int k = threadIdx.x; k < kNParams; k += blockDim.x) S.w[k] = __bfloat162float(wbf[k]);
    __syncthreads();
    const int t = threadIdx.x;
    const uint32_t i = blockIdx.x * kMB + t;
    const bool live = i < n;
    float loss = 0.f;
    {
        float xi[kIn], h1[kH1], h2[kH2];
        if (live) {
            load_norm(x + (size_t)i * kIn, nc, xi);
        } else {
#pragma unroll
            for (int k = 0; k < kIn; ++k) xi[k] = 0.f;
        }
        const float y = mlp_forward(S.w, xi, h1, h2);
        float dy = 0.f;
        if (live) {
            const float r = target[i] - y;
            loss = r >= 0.f ? tau * r : (tau - 1.f) * r;
            dy = (r > 0.f ? -tau : (r < 0.f ? 1.f - tau : 0.f)) * inv_total;
        }
#pragma unroll
        for (int k = 0; k < kIn; ++k) S.x[t][k] = xi[k];
#pragma unroll
        for (int k = 0; k < kH1; ++k) S.h1[t][k] = h1[k];
#pragma unroll
        for (int k = 0; k < kH2; ++k) {
            S.h2[t][k] = h2[k];
            S.d2[t][k] = h2[k] > 0.f ? dy * S.w[oW3 + k] : 0.f;
        }
        S.dy[t] = dy;
        // d1 = W2^T d2, masked by ReLU'; h1 read back from shared memory so the loop
        // can stay rolled without indexing a register array
        for (int u = 0; u < kH1; ++u) {
            float a = 0.f;
#pragma unroll
            for (int v = 0; v < kH2; ++v) a = fmaf(S.w[oW2 + v * kH1 + u], S.d2[t][v], a);
            S.d1[t][u] = S.h1[t][u] > 0.f ? a : 0.f;
        }
    }
    __syncthreads();
    // gradient slices: each thread owns parameters p = t, t + kMB, ...
    for (int p = t; p < kNParams; p += kMB) {
        float g = 0.f;
        if (p < oB1) {                       // W1[u][k] = sum d1[u] * x[k]
            const int u = (p - oW1) / kIn, k = (p - oW1) % kIn;
            for (int s = 0; s < kMB; ++s) g = fmaf(S.d1[s][u], S.x[s][k], g);
        } else if (p < oW2) {                // b1[u]
            const int u = p - oB1;
            for (int s = 0; s < kMB; ++s) g += S.d1[s][u];
        } else if (p < oB2) {                // W2[u][k] = sum d2[u] * h1[k]
            const int u = (p - oW2) / kH1, k = (p - oW2) % kH1;
            for (int s = 0; s < kMB; ++s) g = fmaf(S.d2[s][u], S.h1[s][k], g);
        } else if (p < oW3) {                // b2[u]
            const int u = p - oB2;
            for (int s = 0; s < kMB; ++s) g += S.d2[s][u];
        } else if (p < oB3) {                // W3[k] = sum dy * h2[k]
            const int k = p - oW3;
            for (int s = 0; s < kMB; ++s) g = fmaf(S.dy[s], S.h2[s][k], g);
        } else {                             // b3
            for (int s = 0; s < kMB; ++s) g += S.dy[s];
        }
        atomicAdd(&grad[p], g);
    }
    // block loss
    float l = loss;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((t & 31) == 0 && loss_sum) atomicAdd(loss_sum, l);
}

// Adam on FP32 master weights; writes the BF16 copy used by forward/backward.
__global__ void band_adam_kernel(float *__restrict__ w, __nv_bfloat16 *__restrict__ wbf, float *__restrict__ m,
                                 float *__restrict__ v, const float *__restrict__ grad, float lr, float b1, float b2,
                                 float eps, float bc1, float bc2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNParams) return;
    const float g = grad[p];
    const float mp = b1 * m[p] + (1.f - b1) * g;
    const float vp = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mp;
    v[p] = vp;
    const float upd = lr * (mp / bc1) / (sqrtf(vp / bc2) + eps);
    const float wn = w[p] - upd;
    w[p] = wn;
    wbf[p] = __float2bfloat16_rn(wn);
}

size_t band_bwd_smem_bytes() { return sizeof(BwdSmem); }

static NormConsts norm_of(const float *mean, const float *std_) {
    NormConsts nc;
    for (int k = 0; k < kIn; ++k) {
        nc.mean[k] = mean[k];
        nc.inv_std[k] = std_[k] > 1e-12f ? 1.f / std_[k] : 1.f;
    }
    return nc;
}

cudaError_t launch_band_predict(const __nv_bfloat16 *d_wbf, const float *mean, const float *std_, const float *d_x,
                                const fa_job *d_jobs, uint32_t n, float margin, int w_min, float *d_y,
                                int32_t *d_w, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + 2 * kPredThreads - 1) / (2 * kPredThreads);
    band_predict_kernel<<<blocks, kPredThreads, 0, s>>>(d_wbf, norm_of(mean, std_), d_x, d_jobs, n, margin, w_min,
                                                        d_y, d_w);
    return cudaGetLastError();
}

cudaError_t launch_band_backward(const __nv_bfloat16 *d_wbf, const float *mean, const float *std_, const float *d_x,
                                 const float *d_target, uint32_t n, float tau, float inv_total, float *d_grad,
                                 float *d_loss, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const size_t smem = band_bwd_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(band_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    band_backward_kernel<<<(n + kMB - 1) / kMB, kMB, smem, s>>>(d_wbf, norm_of(mean, std_), d_x, d_target, n, tau,
                                                                inv_total, d_grad, d_loss);
    return cudaGetLastError();
}

cudaError_t launch_band_adam(float *d_w, __nv_bfloat16 *d_wbf, float *d_m, float *d_v, const float *d_grad, float lr,
                             int step, cudaStream_t s)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    band_adam_kernel<<<(kNParams + 255) / 256, 256, 0, s>>>(d_w, d_wbf, d_m, d_v, d_grad, lr, b1, b2, 1e-8f, bc1, bc2);
    return cudaGetLastError();
}

}  // namespace fa
