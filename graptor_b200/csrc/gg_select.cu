// gg_select.cu -- the learned traversal-variant selector: network parameters,
// the hand-written inference / gradient / Adam kernels, the on-device timing
// collector, and the host side of the threshold fallback.
//
// Kernels
//   k_sel_forward : warp per sample, bfloat16 weights, float32 accumulation
//   k_sel_grad    : warp per sample; lane j accumulates, in registers, the
//                   gradient of everything hidden unit j owns (row j of W1
//                   and W2, column j of W3, b1[j], b2[j], b3[j<4]) over the
//                   warp's samples; each warp writes its partial gradient
//   k_sel_reduce  : sums the warps' partials in a fixed order (deterministic)
//                   and optionally applies an Adam step
#include <cuda_bf16.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <cub/cub.cuh>
#include <vector>

#include "gg_internal.cuh"
#include "gg_mlp.cuh"
#include "gg_select.h"

struct gg_selector {
    gg_ctx *ctx = nullptr;
    float *d_params = nullptr;        // float32 master parameters
    __nv_bfloat16 *d_wbf = nullptr;   // bfloat16 copy used for inference
    float *d_adam = nullptr;          // Adam first / second moments [2][NP]
    float h_params[GG_SEL_NPARAMS];
    int adam_t = 0;
};

namespace gg {

using namespace mlp;
constexpr int kSelWarps = 64;  // gradient partials (8 CTAs x 8 warps)

__global__ void k_sel_to_bf16(const float *p, __nv_bfloat16 *b, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(p[i]);
}

__global__ void __launch_bounds__(256) k_sel_forward(const __nv_bfloat16 *w, const float *X, int n, float *out) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int s = wid; s < n; s += nw) {
        float x[IN], o[OUT], z1, a1, z2, a2;
#pragma unroll
        for (int i = 0; i < IN; ++i) x[i] = X[s * IN + i];
        warp_forward(w, x, o, z1, a1, z2, a2);
        if (lane < OUT) out[s * OUT + lane] = o[lane];
    }
}

// Partial loss gradient of each warp over its samples (inv_cnt = 1/sum(mask)).
__global__ void __launch_bounds__(256) k_sel_grad(const float *w, const float *X, const float *Y, const float *M,
                                                  int n, float inv_cnt, float *partial, float *ploss) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int j = threadIdx.x & 31;
    float gW1[IN], gW2[H], gW3[OUT], gb1 = 0, gb2 = 0, gb3 = 0, loss = 0;
#pragma unroll
    for (int i = 0; i < IN; ++i) gW1[i] = 0;
#pragma unroll
    for (int k = 0; k < H; ++k) gW2[k] = 0;
#pragma unroll
    for (int v = 0; v < OUT; ++v) gW3[v] = 0;
    for (int s = wid; s < n; s += nw) {
        float x[IN], o[OUT], z1, a1, z2, a2;
#pragma unroll
        for (int i = 0; i < IN; ++i) x[i] = X[s * IN + i];
        warp_forward(w, x, o, z1, a1, z2, a2);
        float g_out[OUT];
#pragma unroll
        for (int v = 0; v < OUT; ++v) {
            const float r = (o[v] - Y[s * OUT + v]) * M[s * OUT + v];
            loss += r * r * inv_cnt;
            g_out[v] = 2.0f * r * inv_cnt;
        }
        float g_a2 = 0;
#pragma unroll
        for (int v = 0; v < OUT; ++v) {
            gW3[v] = fmaf(g_out[v], a2, gW3[v]);
            g_a2 = fmaf(w[OW3 + v * H + j], g_out[v], g_a2);
        }
        if (j < OUT) gb3 += g_out[j];
        const float g_z2 = z2 > 0.0f ? g_a2 : 0.0f;
        gb2 += g_z2;
        float g_a1 = 0;
#pragma unroll
        for (int k = 0; k < H; ++k) {
            gW2[k] = fmaf(g_z2, __shfl_sync(0xffffffffu, a1, k), gW2[k]);       // row j of W2
            g_a1 = fmaf(w[OW2 + k * H + j], __shfl_sync(0xffffffffu, g_z2, k), g_a1);  // column j
        }
        const float g_z1 = z1 > 0.0f ? g_a1 : 0.0f;
        gb1 += g_z1;
#pragma unroll
        for (int i = 0; i < IN; ++i) gW1[i] = fmaf(g_z1, x[i], gW1[i]);
    }
    float *P = partial + (size_t)wid * NP;
#pragma unroll
    for (int i = 0; i < IN; ++i) P[OW1 + j * IN + i] = gW1[i];
    P[OB1 + j] = gb1;
#pragma unroll
    for (int k = 0; k < H; ++k) P[OW2 + j * H + k] = gW2[k];
    P[OB2 + j] = gb2;
#pragma unroll
    for (int v = 0; v < OUT; ++v) P[OW3 + v * H + j] = gW3[v];
    if (j < OUT) P[OB3 + j] = gb3;
    if (j == 0) ploss[wid] = loss;
}

// Sum partials in warp order; adam_t > 0: Adam step with learning rate lr.
__global__ void k_sel_reduce(const float *partial, const float *ploss, int nwarps, float *grad_out,
                             float *loss_out, float *w, float *adam, int adam_t, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        float l = 0;
        for (int k = 0; k < nwarps; ++k) l += ploss[k];
        *loss_out = l;
    }
    if (p >= NP) return;
    float g = 0;
    for (int k = 0; k < nwarps; ++k) g += partial[(size_t)k * NP + p];
    if (grad_out) grad_out[p] = g;
    if (adam_t > 0) {
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        float m = adam[p] = b1 * adam[p] + (1 - b1) * g;
        float v = adam[NP + p] = b2 * adam[NP + p] + (1 - b2) * g * g;
        const float mh = m / (1 - powf(b1, (float)adam_t)), vh = v / (1 - powf(b2, (float)adam_t));
        w[p] -= lr * mh / (sqrtf(vh) + eps);
    }
}

static gg_status sel_sync_bf16(gg_selector *s) {
    k_sel_to_bf16<<<(NP + 255) / 256, 256, 0, s->ctx->stream>>>(s->d_params, s->d_wbf, NP);
    GG_LAUNCHED(s->ctx);
    return GG_OK;
}

// Device scratch for a dataset: X, Y, M, partials, losses, grad, loss.
struct SelBuf {
    gg_ctx *ctx;
    float *X = nullptr, *Y = nullptr, *M = nullptr, *part = nullptr, *pl = nullptr, *grad = nullptr, *loss = nullptr;
    ~SelBuf() {
        cudaFree(X); cudaFree(Y); cudaFree(M); cudaFree(part); cudaFree(pl); cudaFree(grad); cudaFree(loss);
    }
    gg_status load(const float *hX, const float *hY, const float *hM, int n) {
        GG_CUDA(ctx, cudaMalloc(&X, (size_t)std::max(n, 1) * IN * 4));
        GG_CUDA(ctx, cudaMalloc(&Y, (size_t)std::max(n, 1) * OUT * 4));
        GG_CUDA(ctx, cudaMalloc(&M, (size_t)std::max(n, 1) * OUT * 4));
        GG_CUDA(ctx, cudaMalloc(&part, (size_t)kSelWarps * NP * 4));
        GG_CUDA(ctx, cudaMalloc(&pl, kSelWarps * 4));
        GG_CUDA(ctx, cudaMalloc(&grad, NP * 4));
        GG_CUDA(ctx, cudaMalloc(&loss, 4));
        if (n) {
            GG_CUDA(ctx, cudaMemcpyAsync(X, hX, (size_t)n * IN * 4, cudaMemcpyHostToDevice, ctx->stream));
            GG_CUDA(ctx, cudaMemcpyAsync(Y, hY, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, ctx->stream));
            GG_CUDA(ctx, cudaMemcpyAsync(M, hM, (size_t)n * OUT * 4, cudaMemcpyHostToDevice, ctx->stream));
        }
        return GG_OK;
    }
};

static float mask_count(const float *M, int n) {
    double c = 0;
    for (int i = 0; i < n * OUT; ++i) c += M[i];
    return (float)std::max(1.0, c);
}

// Degree Gini coefficient of the graph (a selector feature), once per graph.
__global__ void k_gini_terms(const uint32_t *sorted, uint32_t n, double *num, double *den) {
    double a = 0, b = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a += (2.0 * (i + 1) - n - 1) * sorted[i];
        b += sorted[i];
    }
    a = dev::block_sum<double, 256>(a);
    b = dev::block_sum<double, 256>(b);
    if (threadIdx.x == 0) {
        atomicAdd(num, a);
        atomicAdd(den, b);
    }
}

__global__ void k_degrees(const uint64_t *off, uint32_t n, uint32_t *deg) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        deg[i] = (uint32_t)(off[i + 1] - off[i]);
}

gg_status graph_gini(gg_graph *g, float *out) {
    if (g->gini >= 0) {
        *out = g->gini;
        return GG_OK;
    }
    gg_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    uint32_t *d0 = nullptr, *d1 = nullptr;
    double *acc = nullptr;
    void *tmp = nullptr;
    size_t tb = 0;
    auto done = [&](gg_status s) { cudaFree(d0); cudaFree(d1); cudaFree(acc); cudaFree(tmp); return s; };
#define GK(e) do { cudaError_t _e = (e); if (_e != cudaSuccess) return done(cuda_error(ctx, _e, #e)); } while (0)
    GK(cudaMalloc(&d0, ((size_t)g->n + 1) * 4));
    GK(cudaMalloc(&d1, ((size_t)g->n + 1) * 4));
    GK(cudaMalloc(&acc, 16));
    GK(cudaMemsetAsync(acc, 0, 16, st));
    k_degrees<<<ctx->sm_count * 4, 256, 0, st>>>(g->off, g->n, d0);
    ctx->launches++;
    GK(cub::DeviceRadixSort::SortKeys(nullptr, tb, d0, d1, (int64_t)g->n, 0, 32, st));
    GK(cudaMalloc(&tmp, tb));
    GK(cub::DeviceRadixSort::SortKeys(tmp, tb, d0, d1, (int64_t)g->n, 0, 32, st));
    ctx->launches++;
    k_gini_terms<<<ctx->sm_count * 4, 256, 0, st>>>(d1, g->n, acc, acc + 1);
    ctx->launches++;
    double h[2] = {0, 0};
    GK(cudaMemcpyAsync(h, acc, 16, cudaMemcpyDeviceToHost, st));
    GK(cudaStreamSynchronize(st));
#undef GK
    g->gini = (h[1] > 0 && g->n) ? (float)(h[0] / ((double)g->n * h[1])) : 0.0f;
    *out = g->gini;
    return done(GG_OK);
}

}  // namespace gg

using namespace gg;

extern "C" {

gg_status gg_selector_create(gg_ctx *ctx, gg_selector **out) {
    if (!ctx || !out) return GG_ERR_ARG;
    gg_selector *s = new (std::nothrow) gg_selector;
    if (!s) return GG_ERR_OOM;
    s->ctx = ctx;
    cudaError_t e;
    if ((e = cudaMalloc(&s->d_params, NP * 4)) != cudaSuccess || (e = cudaMalloc(&s->d_wbf, NP * 2)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_adam, 2 * NP * 4)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->d_adam, 0, 2 * NP * 4, ctx->stream)) != cudaSuccess) {
        gg_selector_destroy(s);
        return cuda_error(ctx, e, "gg_selector_create");
    }
    // deterministic He-style initialisation (splitmix-based normal approx.)
    uint64_t z = 0x5EED5EEDull;
    auto u01 = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    for (int i = 0; i < NP; ++i) s->h_params[i] = 0.0f;
    auto fill = [&](int off, int rows, int cols) {
        const double sd = std::sqrt(2.0 / cols);
        for (int i = 0; i < rows * cols; ++i) {
            double g = std::sqrt(-2.0 * std::log(u01())) * std::cos(6.283185307179586 * u01());
            s->h_params[off + i] = (float)(g * sd);
        }
    };
    fill(OW1, H, IN);
    fill(OW2, H, H);
    fill(OW3, OUT, H);
    gg_status st = gg_selector_set_params(s, s->h_params, NP);
    if (st != GG_OK) {
        gg_selector_destroy(s);
        return st;
    }
    *out = s;
    return GG_OK;
}

gg_status gg_selector_destroy(gg_selector *s) {
    if (!s) return GG_ERR_ARG;
    cudaStreamSynchronize(s->ctx->stream);
    cudaFree(s->d_params);
    cudaFree(s->d_wbf);
    cudaFree(s->d_adam);
    delete s;
    return GG_OK;
}

gg_status gg_selector_set_params(gg_selector *s, const float *p, int n) {
    if (!s || !p || n != NP) return GG_ERR_ARG;
    if (p != s->h_params) std::memcpy(s->h_params, p, NP * 4);
    GG_CUDA(s->ctx, cudaMemcpyAsync(s->d_params, s->h_params, NP * 4, cudaMemcpyHostToDevice, s->ctx->stream));
    GG_CHECK(sel_sync_bf16(s));
    GG_CUDA(s->ctx, cudaMemsetAsync(s->d_adam, 0, 2 * NP * 4, s->ctx->stream));
    s->adam_t = 0;
    GG_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    return GG_OK;
}

gg_status gg_selector_get_params(gg_selector *s, float *p, int n) {
    if (!s || !p || n != NP) return GG_ERR_ARG;
    GG_CUDA(s->ctx, cudaMemcpyAsync(s->h_params, s->d_params, NP * 4, cudaMemcpyDeviceToHost, s->ctx->stream));
    GG_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    std::memcpy(p, s->h_params, NP * 4);
    return GG_OK;
}

gg_status gg_selector_forward(gg_selector *s, const float *X, int n, float *out) {
    if (!s || (n && (!X || !out)) || n < 0) return GG_ERR_ARG;
    if (n == 0) return GG_OK;
    gg_ctx *ctx = s->ctx;
    float *dX = nullptr, *dO = nullptr;
    cudaError_t e = cudaMalloc(&dX, (size_t)n * IN * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dO, (size_t)n * OUT * 4);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dX, X, (size_t)n * IN * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        k_sel_forward<<<std::min(1024, (n + 7) / 8), 256, 0, ctx->stream>>>(s->d_wbf, dX, n, dO);
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dO, (size_t)n * OUT * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dX);
    cudaFree(dO);
    return e == cudaSuccess ? GG_OK : cuda_error(ctx, e, "gg_selector_forward");
}

gg_status gg_selector_loss_grad(gg_selector *s, const float *X, const float *Y, const float *M, int n,
                                float *loss, float *grad) {
    if (!s || n < 0 || (n && (!X || !Y || !M)) || !loss) return GG_ERR_ARG;
    gg_ctx *ctx = s->ctx;
    SelBuf b{ctx};
    GG_CHECK(b.load(X, Y, M, n));
    k_sel_grad<<<kSelWarps / 8, 256, 0, ctx->stream>>>(s->d_params, b.X, b.Y, b.M, n, 1.0f / mask_count(M, n),
                                                        b.part, b.pl);
    GG_LAUNCHED(ctx);
    k_sel_reduce<<<(NP + 255) / 256, 256, 0, ctx->stream>>>(b.part, b.pl, kSelWarps, b.grad, b.loss, nullptr,
                                                            nullptr, 0, 0.0f);
    GG_LAUNCHED(ctx);
    GG_CUDA(ctx, cudaMemcpyAsync(loss, b.loss, 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (grad) GG_CUDA(ctx, cudaMemcpyAsync(grad, b.grad, NP * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GG_OK;
}

gg_status gg_selector_train(gg_selector *s, const float *X, const float *Y, const float *M, int n, int epochs,
                            float lr, float *final_loss) {
    if (!s || n <= 0 || !X || !Y || !M || epochs < 0 || !(lr > 0)) return GG_ERR_ARG;
    gg_ctx *ctx = s->ctx;
    SelBuf b{ctx};
    GG_CHECK(b.load(X, Y, M, n));
    const float inv = 1.0f / mask_count(M, n);
    for (int ep = 0; ep < epochs; ++ep) {
        k_sel_grad<<<kSelWarps / 8, 256, 0, ctx->stream>>>(s->d_params, b.X, b.Y, b.M, n, inv, b.part, b.pl);
        GG_LAUNCHED(ctx);
        k_sel_reduce<<<(NP + 255) / 256, 256, 0, ctx->stream>>>(b.part, b.pl, kSelWarps, nullptr, b.loss,
                                                                s->d_params, s->d_adam, ++s->adam_t, lr);
        GG_LAUNCHED(ctx);
    }
    GG_CHECK(sel_sync_bf16(s));
    // loss after the last step
    k_sel_grad<<<kSelWarps / 8, 256, 0, ctx->stream>>>(s->d_params, b.X, b.Y, b.M, n, inv, b.part, b.pl);
    GG_LAUNCHED(ctx);
    k_sel_reduce<<<(NP + 255) / 256, 256, 0, ctx->stream>>>(b.part, b.pl, kSelWarps, nullptr, b.loss, nullptr,
                                                            nullptr, 0, 0.0f);
    GG_LAUNCHED(ctx);
    if (final_loss) GG_CUDA(ctx, cudaMemcpyAsync(final_loss, b.loss, 4, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaMemcpyAsync(s->h_params, s->d_params, NP * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GG_OK;
}

gg_status gg_graph_set_selector(gg_graph *g, gg_selector *s) {
    if (!g) return GG_ERR_ARG;
    if (s && s->ctx != g->ctx) return set_error(g->ctx, GG_ERR_ARG, "selector of another context");
    g->sel_on = false;
    if (!s) return GG_OK;
    // the graph copies the weights as they are now: the selector may be
    // retrained or destroyed afterwards
    gg_ctx *ctx = g->ctx;
    if (!g->sel_h) {
        g->sel_h = new (std::nothrow) float[NP];
        if (!g->sel_h) return GG_ERR_OOM;
    }
    if (!g->sel_d) GG_CUDA(ctx, cudaMalloc(&g->sel_d, NP * sizeof(__nv_bfloat16)));
    GG_CUDA(ctx, cudaMemcpyAsync(g->sel_d, s->d_wbf, NP * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice,
                                 s->ctx->stream));
    GG_CUDA(ctx, cudaMemcpyAsync(s->h_params, s->d_params, NP * 4, cudaMemcpyDeviceToHost, s->ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(s->ctx->stream));
    std::memcpy(g->sel_h, s->h_params, NP * 4);
    g->sel_on = true;
    float gi;
    GG_CHECK(graph_gini(g, &gi));
    return GG_OK;
}

}  // extern "C"

namespace gg {

const void *selector_weights(gg_graph *g) { return g->sel_on ? (const void *)g->sel_d : nullptr; }

// The ten selector features of an iteration (see gg_select.h).
void selector_features(float *x, double nactv, double nacte, double unreached, int iter, double n, double m,
                       float gini) {
    x[0] = (float)(std::log2(1.0 + nactv) / 32);
    x[1] = (float)(std::log2(1.0 + nacte) / 40);
    x[2] = (float)(std::log2(1.0 + std::max(0.0, unreached)) / 32);
    x[3] = (float)(std::log2(1.0 + std::min(iter, 255)) / 8);
    x[4] = (float)(std::log2(1.0 + (n > 0 ? m / n : 0)) / 8);
    x[5] = gini;
    x[6] = (float)(n > 0 ? nactv / n : 0);
    x[7] = (float)(m > 0 ? nacte / m : 0);
    x[8] = (float)std::min(4.0, m > 0 ? (nactv + nacte) / m : 0.0);
    x[9] = (float)(std::log2(std::max(1.0, n)) / 32);
}

static float bf16r(float f) {  // round to bfloat16 like the device copy
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    std::memcpy(&f, &u, 4);
    return f;
}

// Host-driven edgemap calls with GG_THRESH_LEARNED: the same network on the
// host (bfloat16-rounded weights); the threshold when no selector is attached.
int learned_select(gg_graph *g, uint64_t nactv, uint64_t nacte, int iter, bool can_early_exit) {
    (void)can_early_exit;
    if (!g->sel_on) return (nactv + nacte) <= (g->m / 20) ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
    const float *p = g->sel_h;
    float x[IN], h1[H], h2[H], o[OUT];
    selector_features(x, (double)nactv, (double)nacte, 0.0, iter, g->n, (double)g->m, std::max(0.0f, g->gini));
    for (int j = 0; j < H; ++j) {
        float a = bf16r(p[OB1 + j]);
        for (int i = 0; i < IN; ++i) a += bf16r(p[OW1 + j * IN + i]) * x[i];
        h1[j] = std::max(a, 0.0f);
    }
    for (int j = 0; j < H; ++j) {
        float a = bf16r(p[OB2 + j]);
        for (int k = 0; k < H; ++k) a += bf16r(p[OW2 + j * H + k]) * h1[k];
        h2[j] = std::max(a, 0.0f);
    }
    int best = 0;
    for (int v = 0; v < OUT; ++v) {
        float a = bf16r(p[OB3 + v]);
        for (int k = 0; k < H; ++k) a += bf16r(p[OW3 + v * H + k]) * h2[k];
        o[v] = a;
        if (o[v] < o[best]) best = v;
    }
    // variant ids are the output order; the threshold's choice stands unless
    // the network predicts a clear gain over it
    const int tv = (nactv + nacte) <= (g->m / 20) ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
    return o[best] < o[tv] - mlp::kSelMargin ? best : tv;
}

}  // namespace gg

extern "C" gg_status gg_selector_collect(gg_graph *g, int analytic, uint32_t root, int max_samples, float *X,
                                         float *Y, int cap, int *nrec) {
    if (!g || !nrec || (analytic != 0 && analytic != 1) || max_samples < 1 || cap < 0 || (cap && (!X || !Y)))
        return GG_ERR_ARG;
    if (analytic == 0 && root >= g->n) return GG_ERR_ARG;
    *nrec = 0;
    float gini;
    GG_CHECK(graph_gini(g, &gini));
    gg_run_opts o;
    o.threshold = analytic == 0 ? GG_THRESH_DEFAULT : GG_THRESH_FRAC;
    o.threshold_k = analytic == 0 ? 0 : 5;
    o.variant = GG_VAR_AUTO;
    o.collect_stats = 1;
    auto run = [&](gg_run_stats *st) -> gg_status {
        return analytic == 0 ? gg_bfs_level(g, root, &o, nullptr, nullptr, st) : gg_cc(g, &o, nullptr, nullptr, st);
    };
    // reference run with the threshold's choices (device-driven, nothing forced)
    gg_run_stats rs;
    g->force_iter = INT_MAX;
    g->force_variant = 0;
    gg_status s = run(&rs);
    if (s != GG_OK) { g->force_iter = -1; return s; }
    const int T = rs.iterations;
    // CC's first step starts from the all-true frontier and is always a pull
    const int first = (analytic == 1 && T > 1) ? 1 : 0;
    // sampled iterations: even positions spaced evenly over the run, odd ones
    // geometrically (long runs spend many iterations on small frontiers
    // early on, which even spacing would barely see); duplicates dropped
    const int span = T - first;
    const int k = std::min(max_samples, span);
    std::vector<int> its;
    for (int si = 0; si < k; ++si) {
        int p = 0;
        if (k > 1 && (si & 1)) p = (int)std::lround(std::pow((double)span, (double)si / (k - 1))) - 1;
        else if (k > 1) p = (int)((long long)si * (span - 1) / (k - 1));
        its.push_back(first + std::min(std::max(p, 0), span - 1));
    }
    std::sort(its.begin(), its.end());
    its.erase(std::unique(its.begin(), its.end()), its.end());
    for (size_t si = 0; si < its.size() && *nrec < cap; ++si) {
        const int it = its[si];
        float *x = X + (size_t)*nrec * GG_SEL_FEATURES;
        float *y = Y + (size_t)*nrec * GG_SEL_VARIANTS;
        bool have_x = false;
        for (int v = 0; v < GG_SEL_VARIANTS; ++v) {
            g->force_iter = it;
            g->force_variant = v;
            double best = 1e30;
            for (int rep = 0; rep < 2; ++rep) {  // min of two runs: less timing noise
                s = run(&rs);
                if (s != GG_OK) { g->force_iter = -1; return s; }
                // CC's push steps race (a label can travel several hops in one
                // step), so a run may converge before iteration `it`: no sample
                const auto &fr = g->force_rec;
                if (!fr.seen) continue;
                if (!have_x) {
                    selector_features(x, fr.nactv, fr.nacte, (double)g->n - fr.reached, it, g->n, (double)g->m,
                                      gini);
                    have_x = true;
                }
                // BFS: every variant leaves the same next frontier, so the
                // iteration's own time decides; CC: a fused push finishes the
                // run, so the time until the run ends does
                const double t = analytic == 0 ? fr.iter_ms : fr.rest_ms;
                if (t > 0) best = std::min(best, t);
            }
            y[v] = best < 1e30 ? (float)std::log2(best * 1e3) : std::nanf("");
        }
        if (have_x) ++*nrec;
    }
    g->force_iter = -1;
    g->force_variant = -1;
    return GG_OK;
}
