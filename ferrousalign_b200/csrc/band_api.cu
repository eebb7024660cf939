// band_api.cu -- C ABI of the learned band predictor and the learned extension call.

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "fa_kernels.h"

using namespace fa;

struct fa_band_model {
    std::vector<float> w;          // FP32 master weights (FA_BAND_NPARAMS)
    float mean[16], std_[16];      // feature normalisation
    std::vector<float> m, v;       // Adam moments
    int step = 0;
};

namespace {

int err(int code, const char *msg) { return set_last_error(code, msg); }

#define BA_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            char m_[256];                                                              \
            snprintf(m_, sizeof(m_), "%s failed: %s", #call, cudaGetErrorString(e_));  \
            return set_last_error(FA_ERR_CUDA, m_);                                    \
        }                                                                              \
    } while (0)

// A small RAII device buffer for the band calls (their sizes are modest).
struct DBuf {
    void *p = nullptr;
    explicit DBuf(size_t bytes) { if (bytes) cudaMalloc(&p, bytes); }
    ~DBuf() { if (p) cudaFree(p); }
    bool ok() const { return p != nullptr; }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

uint64_t fnv1a(const void *d, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char *b = static_cast<const unsigned char *>(d);
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

std::vector<__nv_bfloat16> to_bf16(const std::vector<float> &w) {
    std::vector<__nv_bfloat16> r(w.size());
    for (size_t i = 0; i < w.size(); ++i) r[i] = __float2bfloat16_rn(w[i]);
    return r;
}

}  // namespace

void fa::band_model_export(const fa_band_model *m, std::vector<__nv_bfloat16> &wbf, float *mean, float *std_) {
    wbf = to_bf16(m->w);
    memcpy(mean, m->mean, sizeof(m->mean));
    memcpy(std_, m->std_, sizeof(m->std_));
}

extern "C" {

int fa_band_model_create(uint64_t seed, fa_band_model **out) {
    if (!out) return err(FA_ERR_ARG, "null out");
    fa_band_model *m = new fa_band_model();
    m->w.assign(FA_BAND_NPARAMS, 0.f);
    m->m.assign(FA_BAND_NPARAMS, 0.f);
    m->v.assign(FA_BAND_NPARAMS, 0.f);
    for (int k = 0; k < 16; ++k) { m->mean[k] = 0.f; m->std_[k] = 1.f; }
    std::mt19937_64 rng(seed);
    // He-normal initialisation per layer; biases zero (the output bias starts at log2(16))
    auto fill = [&](int off, int fan_in, int count) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (float)fan_in));
        for (int i = 0; i < count; ++i) m->w[off + i] = nd(rng);
    };
    fill(0, 16, 64 * 16);
    fill(64 * 16 + 64, 64, 32 * 64);
    fill(64 * 16 + 64 + 32 * 64 + 32, 32, 32);
    m->w[FA_BAND_NPARAMS - 1] = 4.f;
    *out = m;
    return FA_OK;
}

void fa_band_model_destroy(fa_band_model *m) { delete m; }

int fa_band_model_get(const fa_band_model *m, float *weights, float *mean, float *std_) {
    if (!m) return err(FA_ERR_ARG, "null model");
    if (weights) memcpy(weights, m->w.data(), sizeof(float) * FA_BAND_NPARAMS);
    if (mean) memcpy(mean, m->mean, sizeof(m->mean));
    if (std_) memcpy(std_, m->std_, sizeof(m->std_));
    return FA_OK;
}

int fa_band_model_set(fa_band_model *m, const float *weights, const float *mean, const float *std_) {
    if (!m) return err(FA_ERR_ARG, "null model");
    if (weights) memcpy(m->w.data(), weights, sizeof(float) * FA_BAND_NPARAMS);
    if (mean) memcpy(m->mean, mean, sizeof(m->mean));
    if (std_) memcpy(m->std_, std_, sizeof(m->std_));
    return FA_OK;
}

// File: "FABM" | u32 version=1 | u32 nparams | f32 mean[16] | f32 std[16] | f32 w[n] | u64 fnv1a(all before)
int fa_band_model_save(const fa_band_model *m, const char *path) {
    if (!m || !path) return err(FA_ERR_ARG, "null argument");
    std::string buf("FABM", 4);
    const uint32_t ver = 1, np = FA_BAND_NPARAMS;
    buf.append((const char *)&ver, 4);
    buf.append((const char *)&np, 4);
    buf.append((const char *)m->mean, sizeof(m->mean));
    buf.append((const char *)m->std_, sizeof(m->std_));
    buf.append((const char *)m->w.data(), sizeof(float) * np);
    const uint64_t h = fnv1a(buf.data(), buf.size());
    buf.append((const char *)&h, 8);
    FILE *f = fopen(path, "wb");
    if (!f) return err(FA_ERR_ARG, "cannot open the model file for writing");
    const size_t wr = fwrite(buf.data(), 1, buf.size(), f);
    fclose(f);
    return wr == buf.size() ? FA_OK : err(FA_ERR_ARG, "short write of the model file");
}

int fa_band_model_load(const char *path, fa_band_model **out) {
    if (!path || !out) return err(FA_ERR_ARG, "null argument");
    FILE *f = fopen(path, "rb");
    if (!f) return err(FA_ERR_ARG, "cannot open the model file");
    std::string buf;
    char tmp[65536];
    size_t r;
    while ((r = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, r);
    fclose(f);
    const size_t need = 4 + 4 + 4 + 64 + 64 + 4 * (size_t)FA_BAND_NPARAMS + 8;
    if (buf.size() != need || memcmp(buf.data(), "FABM", 4) != 0) return err(FA_ERR_ARG, "not a band model file");
    uint32_t ver, np;
    memcpy(&ver, buf.data() + 4, 4);
    memcpy(&np, buf.data() + 8, 4);
    if (ver != 1 || np != FA_BAND_NPARAMS) return err(FA_ERR_ARG, "unsupported band model version");
    uint64_t h;
    memcpy(&h, buf.data() + need - 8, 8);
    if (h != fnv1a(buf.data(), need - 8)) return err(FA_ERR_ARG, "band model checksum mismatch");
    fa_band_model *m = nullptr;
    fa_band_model_create(0, &m);
    memcpy(m->mean, buf.data() + 12, 64);
    memcpy(m->std_, buf.data() + 76, 64);
    memcpy(m->w.data(), buf.data() + 140, 4 * (size_t)FA_BAND_NPARAMS);
    *out = m;
    return FA_OK;
}

int fa_band_features(fa_ctx *ctx, const fa_params *p, const fa_job *jobs, uint32_t n, const uint8_t *qseq,
                     uint64_t qseq_len, const uint8_t *tseq, uint64_t tseq_len, const fa_band_hint *hints, float *x) {
    if (!ctx || !p || (n && (!jobs || !qseq || !tseq || !x))) return err(FA_ERR_ARG, "null argument");
    if (n == 0) return FA_OK;
    for (uint32_t i = 0; i < n; ++i)
        if (jobs[i].qlen < 0 || jobs[i].tlen < 0 || jobs[i].q_off + (uint64_t)jobs[i].qlen > qseq_len ||
            jobs[i].t_off + (uint64_t)jobs[i].tlen > tseq_len)
            return err(FA_ERR_ARG, "job sequence range outside the buffers");
    int ms = 0;
    for (int i = 0; i < 25; ++i) if (p->mat[i] > ms) ms = p->mat[i];
    BA_CUDA(cudaSetDevice(fa_ctx_device(ctx)));
    DBuf dj(sizeof(fa_job) * (size_t)n), dq(qseq_len + kSeqPad), dt(tseq_len + kSeqPad),
        dh(hints ? sizeof(fa_band_hint) * (size_t)n : 0), dx(sizeof(float) * 16 * (size_t)n);
    if (!dj.ok() || !dq.ok() || !dt.ok() || !dx.ok() || (hints && !dh.ok()))
        return err(FA_ERR_CAPACITY, "device allocation failed");
    BA_CUDA(cudaMemcpy(dj.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dq.p, qseq, qseq_len, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dt.p, tseq, tseq_len, cudaMemcpyHostToDevice));
    if (hints) BA_CUDA(cudaMemcpy(dh.p, hints, sizeof(fa_band_hint) * (size_t)n, cudaMemcpyHostToDevice));
    BA_CUDA(launch_band_features(dj.as<fa_job>(), n, SeqBuf{dq.as<uint8_t>(), qseq_len, nullptr, 0, 0},
                                 SeqBuf{dt.as<uint8_t>(), tseq_len, nullptr, 0, 0},
                                 hints ? dh.as<fa_band_hint>() : nullptr, ms, dx.as<float>(), 0));
    BA_CUDA(cudaMemcpy(x, dx.p, sizeof(float) * 16 * (size_t)n, cudaMemcpyDeviceToHost));
    return FA_OK;
}

int fa_band_model_fit_norm(fa_band_model *m, const float *x, uint32_t n) {
    if (!m || (n && !x)) return err(FA_ERR_ARG, "null argument");
    for (int k = 0; k < 16; ++k) {
        double s = 0, s2 = 0;
        for (uint32_t i = 0; i < n; ++i) { s += x[(size_t)i * 16 + k]; s2 += (double)x[(size_t)i * 16 + k] * x[(size_t)i * 16 + k]; }
        const double mu = n ? s / n : 0, var = n ? s2 / n - mu * mu : 1;
        m->mean[k] = (float)mu;
        m->std_[k] = (float)std::sqrt(var > 1e-12 ? var : 1.0);
    }
    return FA_OK;
}

int fa_band_predict(fa_ctx *ctx, const fa_band_model *m, const float *x, const fa_job *jobs, uint32_t n, float margin,
                    int w_min, float *y_out, int32_t *w_out) {
    if (!ctx || !m || (n && !x)) return err(FA_ERR_ARG, "null argument");
    if (n == 0) return FA_OK;
    BA_CUDA(cudaSetDevice(fa_ctx_device(ctx)));
    const auto wb = to_bf16(m->w);
    DBuf dw(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS), dx(sizeof(float) * 16 * (size_t)n),
        dj(jobs ? sizeof(fa_job) * (size_t)n : 0), dy(sizeof(float) * (size_t)n), dwo(sizeof(int32_t) * (size_t)n);
    if (!dw.ok() || !dx.ok() || !dy.ok() || !dwo.ok() || (jobs && !dj.ok())) return err(FA_ERR_CAPACITY, "device allocation failed");
    BA_CUDA(cudaMemcpy(dw.p, wb.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * 16 * (size_t)n, cudaMemcpyHostToDevice));
    if (jobs) BA_CUDA(cudaMemcpy(dj.p, jobs, sizeof(fa_job) * (size_t)n, cudaMemcpyHostToDevice));
    BA_CUDA(launch_band_predict(dw.as<__nv_bfloat16>(), m->mean, m->std_, dx.as<float>(), jobs ? dj.as<fa_job>() : nullptr,
                                n, margin, w_min, dy.as<float>(), dwo.as<int32_t>(), 0));
    if (y_out) BA_CUDA(cudaMemcpy(y_out, dy.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    if (w_out) BA_CUDA(cudaMemcpy(w_out, dwo.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
    return FA_OK;
}

int fa_band_grad(fa_ctx *ctx, const fa_band_model *m, const float *x, const float *target, uint32_t n, float tau,
                 float *grad, float *loss) {
    if (!ctx || !m || !grad || (n && (!x || !target))) return err(FA_ERR_ARG, "null argument");
    BA_CUDA(cudaSetDevice(fa_ctx_device(ctx)));
    const auto wb = to_bf16(m->w);
    DBuf dw(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS), dx(sizeof(float) * 16 * (size_t)(n ? n : 1)),
        dt(sizeof(float) * (size_t)(n ? n : 1)), dg(sizeof(float) * FA_BAND_NPARAMS), dl(sizeof(float));
    if (!dw.ok() || !dx.ok() || !dt.ok() || !dg.ok() || !dl.ok()) return err(FA_ERR_CAPACITY, "device allocation failed");
    BA_CUDA(cudaMemcpy(dw.p, wb.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * 16 * (size_t)n, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dt.p, target, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemset(dg.p, 0, sizeof(float) * FA_BAND_NPARAMS));
    BA_CUDA(cudaMemset(dl.p, 0, sizeof(float)));
    BA_CUDA(launch_band_backward(dw.as<__nv_bfloat16>(), m->mean, m->std_, dx.as<float>(), dt.as<float>(), n, tau,
                                 n ? 1.f / (float)n : 0.f, dg.as<float>(), dl.as<float>(), 0));
    BA_CUDA(cudaMemcpy(grad, dg.p, sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyDeviceToHost));
    if (loss) {
        float l = 0.f;
        BA_CUDA(cudaMemcpy(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
        *loss = n ? l / (float)n : 0.f;
    }
    return FA_OK;
}

int fa_band_train(fa_ctx *ctx, fa_band_model *m, const float *x, const float *target, uint32_t n, int epochs,
                  uint32_t batch, float lr, float tau, uint64_t seed, float *epoch_loss) {
    if (!ctx || !m || (n && (!x || !target))) return err(FA_ERR_ARG, "null argument");
    if (n == 0 || epochs <= 0) return FA_OK;
    if (batch == 0) batch = 4096;
    BA_CUDA(cudaSetDevice(fa_ctx_device(ctx)));
    DBuf dx(sizeof(float) * 16 * (size_t)n), dt(sizeof(float) * (size_t)n), dw(sizeof(float) * FA_BAND_NPARAMS),
        dwb(sizeof(__nv_bfloat16) * FA_BAND_NPARAMS), dm(sizeof(float) * FA_BAND_NPARAMS),
        dv(sizeof(float) * FA_BAND_NPARAMS), dg(sizeof(float) * FA_BAND_NPARAMS), dl(sizeof(float));
    if (!dx.ok() || !dt.ok() || !dw.ok() || !dwb.ok() || !dm.ok() || !dv.ok() || !dg.ok() || !dl.ok())
        return err(FA_ERR_CAPACITY, "device allocation failed");
    // shuffle once on the host (seeded), upload
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    std::mt19937_64 rng(seed);
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[rng() % (i + 1)]);
    std::vector<float> xs((size_t)n * 16), ts(n);
    for (uint32_t i = 0; i < n; ++i) {
        memcpy(&xs[(size_t)i * 16], &x[(size_t)perm[i] * 16], 64);
        ts[i] = target[perm[i]];
    }
    BA_CUDA(cudaMemcpy(dx.p, xs.data(), xs.size() * 4, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dt.p, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice));
    const auto wb = to_bf16(m->w);
    BA_CUDA(cudaMemcpy(dw.p, m->w.data(), sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dwb.p, wb.data(), sizeof(__nv_bfloat16) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dm.p, m->m.data(), sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    BA_CUDA(cudaMemcpy(dv.p, m->v.data(), sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyHostToDevice));
    for (int ep = 0; ep < epochs; ++ep) {
        BA_CUDA(cudaMemset(dl.p, 0, sizeof(float)));
        for (uint32_t b0 = 0; b0 < n; b0 += batch) {
            const uint32_t nb = std::min(batch, n - b0);
            BA_CUDA(cudaMemset(dg.p, 0, sizeof(float) * FA_BAND_NPARAMS));
            BA_CUDA(launch_band_backward(dwb.as<__nv_bfloat16>(), m->mean, m->std_, dx.as<float>() + (size_t)b0 * 16,
                                         dt.as<float>() + b0, nb, tau, 1.f / (float)nb, dg.as<float>(), dl.as<float>(), 0));
            BA_CUDA(launch_band_adam(dw.as<float>(), dwb.as<__nv_bfloat16>(), dm.as<float>(), dv.as<float>(), dg.as<float>(),
                                     lr, ++m->step, 0));
        }
        if (epoch_loss) {
            float l = 0.f;
            BA_CUDA(cudaMemcpy(&l, dl.p, 4, cudaMemcpyDeviceToHost));
            epoch_loss[ep] = l / (float)n;
        }
    }
    BA_CUDA(cudaMemcpy(m->w.data(), dw.p, sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyDeviceToHost));
    BA_CUDA(cudaMemcpy(m->m.data(), dm.p, sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyDeviceToHost));
    BA_CUDA(cudaMemcpy(m->v.data(), dv.p, sizeof(float) * FA_BAND_NPARAMS, cudaMemcpyDeviceToHost));
    return FA_OK;
}

}  // extern "C"
