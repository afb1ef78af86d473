// C ABI: the learned search radius (features, MLP parameters, training,
// prediction, model files). Declarations are in include/shapex.h.

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.cuh"

using namespace shapex;
using namespace shapex::capi;

extern "C" {

// ---- learned search radius ---------------------------------------------------

namespace {

int mlp_alloc(se_ctx* c) {
    if (c->mlp) return SE_OK;
    SE_CUDA(c, regrow(c->mlp, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_m, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_v, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_g, kMlpParams), "alloc mlp");
    SE_CUDA(c, regrow(c->mlp_loss, 1), "alloc mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    c->mlp_step = 0;
    return SE_OK;
}

int mlp_work(se_ctx* c, int64_t n) {
    if (n <= c->mw_cap) return SE_OK;
    SE_CUDA(c, regrow(c->mw.yhat, n), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.h1, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.h2, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dy, n), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dh1, n * kMlpH), "alloc mlp work");
    SE_CUDA(c, regrow(c->mw.dh2, n * kMlpH), "alloc mlp work");
    c->mw_cap = n;
    return SE_OK;
}

// Device pointer for n floats given by the caller: host data goes through the
// context's staging buffer at float offset `off` (the buffer holds `total`).
int stage_in(se_ctx* c, const float* src, int64_t n, int mem, int64_t off, int64_t total, const float** out) {
    if (mem == SE_MEM_DEVICE || n == 0) {
        *out = src;
        return SE_OK;
    }
    if (c->xs_cap < total) {
        SE_CUDA(c, regrow(c->xs_buf, total), "alloc staging");
        c->xs_cap = total;
    }
    SE_CUDA(c, cudaMemcpyAsync(c->xs_buf + off, src, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "copy in");
    *out = c->xs_buf + off;
    return SE_OK;
}

uint64_t xorshift(uint64_t& s) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

}  // namespace

int se_features(se_ctx* c, int64_t start, int64_t count, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    const int64_t u = c->info.n_points;
    if (start < 0 || count < 0 || start + count > u) return fail(c, SE_ERR_INVALID_ARG, "range outside [0, u)");
    if (count == 0) return SE_OK;
    if (!out) return fail(c, SE_ERR_INVALID_ARG, "null output");
    float* dst = out;
    if (mem == SE_MEM_HOST) {
        if (c->xs_cap < count * kMlpF) {
            SE_CUDA(c, regrow(c->xs_buf, count * kMlpF), "alloc staging");
            c->xs_cap = count * kMlpF;
        }
        dst = c->xs_buf;
    }
    SE_CUDA(c, enqueue_features(c->b, u, c->opt.code_bits, start, count, dst, c->stream), "launch features");
    if (mem == SE_MEM_HOST)
        SE_CUDA(c, cudaMemcpyAsync(out, dst, sizeof(float) * count * kMlpF, cudaMemcpyDeviceToHost, c->stream),
                "copy features");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_init(se_ctx* c, uint64_t seed) {
    if (int rc = prologue(c)) return rc;
    if (int rc = mlp_alloc(c)) return rc;
    float h[kMlpParams] = {};
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull;
    if (!s) s = 1;
    auto uni = [&](float a) { return a * (2.0f * (float)((xorshift(s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0f); };
    const float a1 = sqrtf(6.0f / kMlpF), a2 = sqrtf(6.0f / kMlpH);
    for (int i = 0; i < kMlpF * kMlpH; ++i) h[MlpLayout::W1 + i] = uni(a1);
    for (int i = 0; i < kMlpH * kMlpH; ++i) h[MlpLayout::W2 + i] = uni(a2);
    for (int i = 0; i < kMlpH; ++i) h[MlpLayout::W3 + i] = uni(a2) * 0.1f;
    SE_CUDA(c, cudaMemcpyAsync(c->mlp, h, sizeof(h), cudaMemcpyHostToDevice, c->stream), "upload mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "init mlp");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    c->mlp_step = 0;
    c->mlp_ready = true;
    return SE_OK;
}

int se_mlp_params(se_ctx* c, float* params, int set, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!params) return fail(c, SE_ERR_INVALID_ARG, "null params");
    if (int rc = mlp_alloc(c)) return rc;
    const cudaMemcpyKind k = set ? (mem == SE_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice)
                                 : (mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
    if (set) {
        SE_CUDA(c, cudaMemcpyAsync(c->mlp, params, sizeof(float) * kMlpParams, k, c->stream), "set params");
        SE_CUDA(c, cudaMemsetAsync(c->mlp_m, 0, sizeof(float) * kMlpParams, c->stream), "reset adam");
        SE_CUDA(c, cudaMemsetAsync(c->mlp_v, 0, sizeof(float) * kMlpParams, c->stream), "reset adam");
        c->mlp_step = 0;
        c->mlp_ready = true;
    } else {
        SE_CUDA(c, cudaMemcpyAsync(params, c->mlp, sizeof(float) * kMlpParams, k, c->stream), "get params");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_enable(se_ctx* c, int learned, int skip_seed) {
    if (!c) return SE_ERR_INVALID_ARG;
    if (learned && !c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    c->opt.learned = learned ? 1 : 0;
    c->opt.learned_skip_seed = skip_seed ? 1 : 0;
    return SE_OK;
}

int se_mlp_set_loss(se_ctx* c, float quantile) {
    if (!c) return SE_ERR_INVALID_ARG;
    if (!(quantile == 0.0f || (quantile > 0.0f && quantile < 1.0f)))
        return fail(c, SE_ERR_INVALID_ARG, "quantile must be 0 (squared error) or in (0, 1)");
    c->mlp_tau = quantile;
    return SE_OK;
}

int se_mlp_set_margin(se_ctx* c, float margin_log2) {
    if (!c) return SE_ERR_INVALID_ARG;
    if (!(margin_log2 > -64.0f && margin_log2 < 64.0f)) return fail(c, SE_ERR_INVALID_ARG, "margin out of range");
    c->mlp_margin = margin_log2;
    return SE_OK;
}

int se_mlp_forward(se_ctx* c, const float* features, int64_t n, float* out, int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 0) return fail(c, SE_ERR_INVALID_ARG, "negative n");
    if (n == 0) return SE_OK;
    if (!features || !out) return fail(c, SE_ERR_INVALID_ARG, "null pointer");
    const float* X;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    float* Y = mem == SE_MEM_HOST ? c->xs_buf + n * kMlpF : out;
    SE_CUDA(c, enqueue_mlp_forward(c->mlp, X, n, Y, nullptr, nullptr, c->stream), "launch forward");
    if (mem == SE_MEM_HOST)
        SE_CUDA(c, cudaMemcpyAsync(out, Y, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream), "copy out");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_predict(se_ctx* c, int64_t start, int64_t count, float* yhat, float* r2, int mem) {
    if (int rc = prologue(c)) return rc;
    if (!c->built) return fail(c, SE_ERR_NOT_BUILT, "not built");
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    const int64_t u = c->info.n_points;
    if (start < 0 || count < 0 || start + count > u) return fail(c, SE_ERR_INVALID_ARG, "range outside [0, u)");
    if (count == 0) return SE_OK;
    float *dy = yhat, *dr = r2;
    if (mem == SE_MEM_HOST) {
        if (c->xs_cap < 2 * count) {
            SE_CUDA(c, regrow(c->xs_buf, 2 * count), "alloc staging");
            c->xs_cap = 2 * count;
        }
        dy = yhat ? c->xs_buf : nullptr;
        dr = r2 ? c->xs_buf + count : nullptr;
    }
    SE_CUDA(c, enqueue_predict_radius(c->b, c->mlp, c->mlp_margin, u, c->opt.code_bits, start, count, dr, dy,
                                      c->stream),
            "launch prediction");
    if (mem == SE_MEM_HOST) {
        if (yhat) SE_CUDA(c, cudaMemcpyAsync(yhat, dy, sizeof(float) * count, cudaMemcpyDeviceToHost, c->stream), "copy");
        if (r2) SE_CUDA(c, cudaMemcpyAsync(r2, dr, sizeof(float) * count, cudaMemcpyDeviceToHost, c->stream), "copy");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_grad(se_ctx* c, const float* features, const float* targets, int64_t n, float* grads, float* loss,
                int mem) {
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 1 || !features || !targets) return fail(c, SE_ERR_INVALID_ARG, "bad arguments");
    if (int rc = mlp_work(c, n)) return rc;
    const float *X, *Y;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    if (int rc = stage_in(c, targets, n, mem, n * kMlpF, n * kMlpF + n, &Y)) return rc;
    SE_CUDA(c, enqueue_mlp_grad(c->mlp, X, Y, n, c->mlp_tau, c->mw, c->mlp_g, c->mlp_loss, c->stream), "launch grad");
    const cudaMemcpyKind k = mem == SE_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (grads) SE_CUDA(c, cudaMemcpyAsync(grads, c->mlp_g, sizeof(float) * kMlpParams, k, c->stream), "copy grads");
    if (loss) SE_CUDA(c, cudaMemcpyAsync(loss, c->mlp_loss, sizeof(float), k, c->stream), "copy loss");
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_train(se_ctx* c, const float* features, const float* targets, int64_t n, int steps, int batch, float lr,
                 float* losses, int mem) {
    NvtxRange nvtx("shapex.se_mlp_train");
    if (int rc = prologue(c)) return rc;
    if (int rc = check_mem(c, mem)) return rc;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    if (n < 1 || steps < 0 || batch < 1 || !features || !targets || !(lr > 0.0f))
        return fail(c, SE_ERR_INVALID_ARG, "bad arguments");
    if (batch > n) batch = (int)n;
    if (int rc = mlp_work(c, batch)) return rc;
    const float *X, *Y;
    if (int rc = stage_in(c, features, n * kMlpF, mem, 0, n * kMlpF + n, &X)) return rc;
    if (int rc = stage_in(c, targets, n, mem, n * kMlpF, n * kMlpF + n, &Y)) return rc;
    float* dloss = nullptr;
    if (losses) {
        SE_CUDA(c, regrow(dloss, steps > 0 ? steps : 1), "alloc losses");
    }
    int64_t row = 0;
    for (int it = 0; it < steps; ++it) {
        if (row + batch > n) row = 0;
        SE_CUDA(c, enqueue_mlp_grad(c->mlp, X + row * kMlpF, Y + row, batch, c->mlp_tau, c->mw, c->mlp_g,
                                    dloss ? dloss + it : c->mlp_loss, c->stream),
                "launch grad");
        SE_CUDA(c, enqueue_adam(c->mlp, c->mlp_g, c->mlp_m, c->mlp_v, lr, ++c->mlp_step, c->stream), "launch adam");
        row += batch;
    }
    if (dloss) {
        cudaError_t e = cudaMemcpyAsync(losses, dloss, sizeof(float) * steps, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        cudaFree(dloss);
        if (e != cudaSuccess) return cuda_fail(c, e, "copy losses");
    }
    SE_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
    return SE_OK;
}

int se_mlp_save(se_ctx* c, const char* path) {
    if (!c || !path) return SE_ERR_INVALID_ARG;
    if (!c->mlp_ready) return fail(c, SE_ERR_NOT_BUILT, "model not initialised");
    float h[kMlpParams];
    if (int rc = se_mlp_params(c, h, 0, SE_MEM_HOST)) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(c, SE_ERR_INVALID_ARG, std::string("cannot write ") + path);
    const int32_t dims[2] = {kMlpF, kMlpH};
    bool ok = std::fwrite("SXMLP1\0\0", 1, 8, f) == 8 && std::fwrite(dims, 4, 2, f) == 2 &&
              std::fwrite(h, 4, kMlpParams, f) == (size_t)kMlpParams && std::fwrite(&c->mlp_margin, 4, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SE_OK : fail(c, SE_ERR_INVALID_ARG, std::string("write failed: ") + path);
}

int se_mlp_load(se_ctx* c, const char* path) {
    if (!c || !path) return SE_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(c, SE_ERR_INVALID_ARG, std::string("cannot read ") + path);
    char magic[8];
    int32_t dims[2];
    float h[kMlpParams];
    float margin = 0.0f;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SXMLP1", 6) == 0 &&
              std::fread(dims, 4, 2, f) == 2 && dims[0] == kMlpF && dims[1] == kMlpH &&
              std::fread(h, 4, kMlpParams, f) == (size_t)kMlpParams && std::fread(&margin, 4, 1, f) == 1;
    std::fclose(f);
    if (!ok) return fail(c, SE_ERR_INVALID_ARG, std::string("not a model file of this layout: ") + path);
    if (int rc = se_mlp_params(c, h, 1, SE_MEM_HOST)) return rc;
    c->mlp_margin = margin;
    return SE_OK;
}

}  // extern "C"
