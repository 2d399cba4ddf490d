// gg_mlp.cuh -- device code of the traversal-variant selector network
// (10 -> 32 -> 32 -> 4, ReLU).  One warp evaluates one sample: lane j owns
// hidden unit j of both hidden layers, activations move between lanes by
// shuffles, the four outputs are warp sums.
#pragma once
#include <cuda_bf16.h>

#include "gg_select.h"

namespace gg {
namespace mlp {

constexpr int IN = GG_SEL_FEATURES, H = 32, OUT = GG_SEL_VARIANTS;
// A learned choice replaces the threshold's only when its predicted time is
// lower by more than this (log2 units: 2^-0.2 = 13% faster).
constexpr float kSelMargin = 0.2f;
// CC's records time the rest of the run, whose variants differ by a few per
// cent at most on the training graphs: a CC step overrides the threshold
// only on a predicted gain of more than 2^0.5 (41 %).
constexpr float kSelMarginCC = 0.5f;
constexpr int OW1 = 0, OB1 = OW1 + H * IN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H,
              OB3 = OW3 + OUT * H, NP = OB3 + OUT;
static_assert(NP == GG_SEL_NPARAMS, "parameter layout");

template <typename W> __device__ __forceinline__ float wv(const W *w, int i);
template <> __device__ __forceinline__ float wv<float>(const float *w, int i) { return w[i]; }
template <> __device__ __forceinline__ float wv<__nv_bfloat16>(const __nv_bfloat16 *w, int i) {
    return __bfloat162float(w[i]);
}

// Forward pass of one sample by one full warp.  x: the 10 features (same in
// every lane).  Returns the outputs in out[0..3] (every lane), and the
// lane's pre-activations z1, z2 and activations a1, a2 for a backward pass.
template <typename W>
__device__ __forceinline__ void warp_forward(const W *w, const float *x, float *out, float &z1, float &a1,
                                             float &z2, float &a2) {
    const int j = threadIdx.x & 31;
    float acc = wv(w, OB1 + j);
#pragma unroll
    for (int i = 0; i < IN; ++i) acc = fmaf(wv(w, OW1 + j * IN + i), x[i], acc);
    z1 = acc;
    a1 = fmaxf(acc, 0.0f);
    acc = wv(w, OB2 + j);
#pragma unroll
    for (int k = 0; k < H; ++k) acc = fmaf(wv(w, OW2 + j * H + k), __shfl_sync(0xffffffffu, a1, k), acc);
    z2 = acc;
    a2 = fmaxf(acc, 0.0f);
#pragma unroll
    for (int v = 0; v < OUT; ++v) {
        float p = wv(w, OW3 + v * H + j) * a2;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        out[v] = p + wv(w, OB3 + v);
    }
}

// One lane's share of the network (hidden unit j = lane: its rows of the
// two hidden layers, its column of the output layer, the output biases),
// loaded into registers ahead of use so that the loads overlap other work.
struct LaneWeights {
    float w1[IN], b1, w2[H], b2, w3[OUT], b3[OUT];
};

template <typename W>
__device__ __forceinline__ void load_lane(const W *w, LaneWeights &L) {
    const int j = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < IN; ++i) L.w1[i] = wv(w, OW1 + j * IN + i);
    L.b1 = wv(w, OB1 + j);
#pragma unroll
    for (int k = 0; k < H; ++k) L.w2[k] = wv(w, OW2 + j * H + k);
    L.b2 = wv(w, OB2 + j);
#pragma unroll
    for (int v = 0; v < OUT; ++v) {
        L.w3[v] = wv(w, OW3 + v * H + j);
        L.b3[v] = wv(w, OB3 + v);
    }
}

// warp_forward on weights already in registers (same arithmetic, same order)
__device__ __forceinline__ void warp_forward_regs(const LaneWeights &L, const float *x, float *out) {
    float acc = L.b1;
#pragma unroll
    for (int i = 0; i < IN; ++i) acc = fmaf(L.w1[i], x[i], acc);
    const float a1 = fmaxf(acc, 0.0f);
    acc = L.b2;
#pragma unroll
    for (int k = 0; k < H; ++k) acc = fmaf(L.w2[k], __shfl_sync(0xffffffffu, a1, k), acc);
    const float a2 = fmaxf(acc, 0.0f);
#pragma unroll
    for (int v = 0; v < OUT; ++v) {
        float p = L.w3[v] * a2;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        out[v] = p + L.b3[v];
    }
}

}  // namespace mlp
}  // namespace gg
