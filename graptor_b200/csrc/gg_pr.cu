// gg_pr.cu -- PageRank power iteration (PRv / PR_vary) and the ADD_GATHER
// edgemap.
//
// Reference loop (bench/PRv.C:115-290, bench/PR_vary.C:247-447), per
// iteration:
//   y[d]  = sum_{s->d} contrib[s]                  dense pull, PRv.C:202-212
//   s     = sum y                                   (double)   PRv.C:227-231
//   y    += (1-s)/n                                 dangling + teleport mass
//   s     = sum y ; y *= 1/s                        renormalise
//   delta = sum |x-y| (double); x = y; y = 0; contrib = d*x/outdeg
// until iter == maxiter or delta <= tol.
//
// B200 design: two kernels per iteration plus a one-thread bookkeeping
// kernel, all enqueued up front; a device-resident state block carries the
// sums and a "done" flag that makes later iterations return immediately once
// the residual test passes, so the host never synchronises inside the loop.
//   k_pr_gather : warp owns 32 destinations; short rows summed per lane, long
//                 rows by the whole warp with 4 independent coalesced loads in
//                 flight per lane; contributions decoded from the storage
//                 format (FP32, BF16, FP16, FP8-E4M3 with scale, customfp<6,10>,
//                 BF16-by-truncation); accumulation in float or double; the
//                 block sums of y (double) are folded in with one atomic per CTA.
//   k_pr_update : y += w, y *= 1/s, delta, x = y, contrib = d*x/deg encoded,
//                 one pass.  The second sum of the reference (sum of the
//                 rounded y+w) is taken as s + n*w in double: equal in exact
//                 arithmetic, different by at most n/2 float ulps of 1/n.
//   k_pr_finish : residual test, iteration count, FP8 scale for the next
//                 encode (from this iteration's max with 2x headroom); FP16
//                 is scaled the same way, since contributions of order 1/n
//                 fall below its normal range.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <cmath>
#include <cstring>

#include <cstdio>
#include <cstdlib>

#include <algorithm>
#include "gg_internal.cuh"

namespace gg {

// ---------------------------------------------------------------------------
// Storage formats
// ---------------------------------------------------------------------------
template <int DT> struct Store;
// Rank / accumulator type of the vertex passes: double for the FP64 variant
// (PR_vary's FP64 run_prec instantiation), float otherwise.
template <int DT> using XT = typename std::conditional<DT == GG_F64, double, float>::type;
template <> struct Store<GG_F64> {
    using T = double;
    __device__ static double dec(T v) { return v; }
    __device__ static T enc(double f) { return f; }
};
template <> struct Store<GG_F32> {
    using T = float;
    __device__ static float dec(T v) { return v; }
    __device__ static T enc(float f) { return f; }
};
// bfloat16 / float16 stored as raw 16-bit words: plain integer loads and
// stores (the class types' assignment made the bfloat16 update kernel several
// times slower than the float16 one).
template <> struct Store<GG_BF16> {
    using T = uint16_t;
    __device__ static float dec(T v) { return __uint_as_float((uint32_t)v << 16); }
    __device__ static T enc(float f) { return dev::bf16_rne(f); }
};
template <> struct Store<GG_F16> {
    using T = uint16_t;
    __device__ static float dec(T v) { return __half2float(__ushort_as_half(v)); }
    __device__ static T enc(float f) { return __half_as_ushort(__float2half_rn(f)); }
};
template <> struct Store<GG_FP8E4M3> {
    using T = __nv_fp8_storage_t;
    __device__ static float dec(T v) {
        __half_raw h = __nv_cvt_fp8_to_halfraw(v, __NV_E4M3);
        return __half2float(__half(h));
    }
    __device__ static T enc(float f) { return __nv_cvt_float_to_fp8(f, __NV_SATFINITE, __NV_E4M3); }
};
// Graptor customfp<6,10> (include/graptor/customfp.h:97-166): low 6 exponent
// bits + top 10 mantissa bits, truncated; decoding restores exponent bit 6.
template <> struct Store<GG_CFP_6_10> {
    using T = uint16_t;
    __device__ static float dec(T v) { return __uint_as_float(((uint32_t)v | (1u << 16)) << 13); }
    __device__ static T enc(float f) { return (T)((__float_as_uint(f) >> 13) & 0xFFFFu); }
};
// Graptor scustomfp<true,8,7>: bfloat16 by truncation.
template <> struct Store<GG_BF16_TRUNC> {
    using T = uint16_t;
    __device__ static float dec(T v) { return __uint_as_float((uint32_t)v << 16); }
    __device__ static T enc(float f) { return (T)(__float_as_uint(f) >> 16); }
};

struct PrState {
    double s1;        // sum of y after the gather
    double delta;     // L1 residual of this iteration
    float cmax;       // max contribution written by the update (for FP8 scaling)
    float scale;      // encode multiplier of the stored contributions
    float scale_inv;  // decode multiplier
    int done;
    int iters;
    int maxiter;
    double tol;
    double deltas[GG_MAX_ITERS];
    // staged runs (PR_vary's run_prec_X then run_prec_Y): the active stage,
    // each stage's dtype and residual bound, and a re-encode request raised
    // when the stage changes
    int stage, nstages, reencode;
    int stage_dt[4];
    double stage_tol[4];
    // BF16 stochastic rounding; tail averaging from iteration avg_from on
    int sr;
    int avg_from, avg_n;
};

// MurmurHash3's fmix32 finaliser: 16 random bits per (vertex, iteration)
__device__ __forceinline__ uint32_t sr_bits(uint32_t v, uint32_t it) {
    uint32_t h = v * 0x9E3779B1u + it * 0x85EBCA77u + 0x165667B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h & 0xFFFFu;
}
// bfloat16 of a non-negative float rounded up with probability (f - down) /
// (up - down): the low 16 bits of the pattern plus 16 random bits carry into
// bit 16 exactly that often (inf stays inf)
__device__ __forceinline__ uint16_t bf16_stochastic(float f, uint32_t v, uint32_t it) {
    const uint32_t u = __float_as_uint(f);
    if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);
    return (uint16_t)((u + sr_bits(v, it)) >> 16);
}

// true when a kernel of stage `stage` (-1: unstaged) has nothing to do
__device__ __forceinline__ bool pr_idle(const PrState *st, int stage) {
    return st && (st->done || (stage >= 0 && st->stage != stage));
}

constexpr unsigned FULL = 0xffffffffu;

// Scaled formats: FP8-E4M3 (max 448) and FP16 (max 65504, min normal 2^-14)
// store contrib * scale with scale a power of two chosen so that the
// largest contribution lands at half the format's range (2x headroom).
__device__ __host__ inline bool scaled_format(int dt) { return dt == GG_FP8E4M3 || dt == GG_F16; }
__device__ __host__ inline float scale_for(int dt, float cmax) {
    if (!scaled_format(dt) || !(cmax > 0.0f)) return 1.0f;
    const float half_range = dt == GG_FP8E4M3 ? 224.0f : 32768.0f;
    int e;
    frexpf(half_range / cmax, &e);
    return ldexpf(1.0f, e - 1);
}

template <int DT, bool ACC64, bool ADD_OLD, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_pr_gather(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_adj,
            const typename Store<DT>::T *__restrict__ contrib, uint32_t n, float *y_f32,
            double *y_f64, PrState *st, float scale_inv_arg, int K, uint32_t T, int stream,
            const uint64_t *__restrict__ word_prefix, int stage) {
    using S = Store<DT>;
    using Acc = typename std::conditional<ACC64, double, float>::type;
    constexpr int U = 4;  // 32-edge chunks in flight per warp iteration
    __shared__ Acc sm[BLOCK / 32][33];
    if (pr_idle(st, stage)) return;
    const float sinv = st ? st->scale_inv : scale_inv_arg;
    const uint32_t lane = threadIdx.x & 31u;
    Acc *row = sm[threadIdx.x >> 5];
    const uint32_t nwords = (n + 31u) >> 5;
    const uint32_t nw = (gridDim.x * BLOCK) >> 5;
    const uint64_t oend = in_off[n];
    double ysum = 0;
    // a contiguous range of words of equal light-edge work per warp
    uint32_t wlo, whi;
    dev::balanced_range(word_prefix, nwords, (blockIdx.x * BLOCK + threadIdx.x) >> 5, nw, wlo, whi);
    for (uint32_t w = wlo; w < whi; ++w) {
        const uint32_t d = (w << 5) + lane;
        const bool valid = d < n;
        const uint64_t beg = valid ? in_off[d] : oend;
        const uint64_t end = valid ? in_off[d + 1] : oend;
        // heavy rows are summed by k_pr_heavy_chunks / k_pr_heavy_finalize
        const bool heavy = end - beg > (uint64_t)T;
        const bool mine = valid && !heavy;
        Acc acc = 0;
        if (stream && __ballot_sync(FULL, heavy) == 0) {
            // Streaming: the word's 32 rows are contiguous in in_adj; lanes
            // take consecutive edges, find their row by a 5-step search over
            // the lanes' row starts, and sum per row with a segmented scan.
            const uint64_t o0 = __shfl_sync(FULL, beg, 0);
            const uint64_t o1 = __shfl_sync(FULL, end, 31);
            row[lane] = 0;
            __syncwarp();
            for (uint64_t base = o0; base < o1; base += 32 * U) {
                uint32_t sidx[U];
                Acc val[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t e = base + u * 32 + lane;
                    sidx[u] = e < o1 ? __ldg(in_adj + e) : 0u;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t e = base + u * 32 + lane;
                    val[u] = e < o1 ? (Acc)S::dec(contrib[sidx[u]]) : (Acc)0;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t e = base + u * 32 + lane;
                    if (base + u * 32 >= o1) break;  // warp-uniform
                    const bool ok = e < o1;
                    uint32_t r = 0;
#pragma unroll
                    for (uint32_t step = 16; step >= 1; step >>= 1) {
                        const uint64_t bc = __shfl_sync(FULL, beg, r + step);
                        if (bc <= e) r += step;
                    }
                    if (!ok) r = 32;
                    Acc v = val[u];
#pragma unroll
                    for (int dd = 1; dd < 32; dd <<= 1) {
                        const Acc t = __shfl_up_sync(FULL, v, dd);
                        const uint32_t rr = __shfl_up_sync(FULL, r, dd);
                        if (lane >= (uint32_t)dd && rr == r) v += t;
                    }
                    const uint32_t rn = __shfl_down_sync(FULL, r, 1);
                    const bool tail = lane == 31 || rn != r;
                    if (ok && tail) row[r] += v;
                    __syncwarp();
                }
            }
            acc = row[lane];
            __syncwarp();
        } else {
            // words holding a heavy row: per-row sums for the light rows
            const bool shortrow = end - beg <= (uint64_t)K;
            if (mine && shortrow)
                for (uint64_t e = beg; e < end; ++e) acc += (Acc)S::dec(contrib[__ldg(in_adj + e)]);
            unsigned pend = __ballot_sync(FULL, mine && !shortrow);
            while (pend) {
                const int j = __ffs(pend) - 1;
                pend &= pend - 1;
                const uint64_t bj = __shfl_sync(FULL, beg, j);
                const uint64_t ej = __shfl_sync(FULL, end, j);
                Acc part = 0;
                for (uint64_t b2 = bj; b2 < ej; b2 += 32) {
                    const uint64_t e = b2 + lane;
                    if (e < ej) part += (Acc)S::dec(contrib[__ldg(in_adj + e)]);
                }
                part = dev::warp_sum(part);
                if ((int)lane == j) acc = part;
            }
        }
        if (mine) {
            if (DT == GG_FP8E4M3 || DT == GG_F16) acc *= (Acc)sinv;
            if (y_f64) {
                double v = ADD_OLD ? y_f64[d] + (double)acc : (double)acc;
                y_f64[d] = v;
                ysum += v;
            } else {
                float v = ADD_OLD ? (float)((double)y_f32[d] + (double)acc) : (float)acc;
                y_f32[d] = v;
                ysum += (double)v;
            }
        }
    }
    if (st) {
        ysum = dev::block_sum<double, BLOCK>(ysum);
        if (threadIdx.x == 0) atomicAdd(&st->s1, ysum);
    }
}

// One warp per chunk of a heavy row: partial[c] = sum of the chunk's
// decoded contributions (4 independent coalesced loads per lane in flight).
template <int DT, bool ACC64>
__global__ void __launch_bounds__(256)
k_pr_heavy_chunks(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_adj,
                  const typename Store<DT>::T *__restrict__ contrib, HeavyRows H,
                  typename std::conditional<ACC64, double, float>::type *partial, const PrState *st,
                  int stage) {
    using S = Store<DT>;
    using Acc = typename std::conditional<ACC64, double, float>::type;
    if (pr_idle(st, stage)) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < H.nchunks; c += nw) {
        const uint32_t lo = H.crow[c];  // heavy row owning chunk c
        const uint32_t v = H.v[lo];
        const uint64_t rb = in_off[v], re = in_off[v + 1];
        const uint64_t e0 = rb + (c - H.first[lo]) * H.CH;
        const uint64_t e1 = min(e0 + H.CH, re);
        Acc part = 0;
        uint64_t base = e0;
        for (; base + 256 <= e1; base += 256) {  // two 128-edge blocks of loads in flight
            uint32_t s8[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) s8[u] = __ldg(in_adj + base + 32 * u + lane);
            Acc c8[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) c8[u] = (Acc)S::dec(contrib[s8[u]]);
            part += c8[0] + c8[1] + c8[2] + c8[3];
            part += c8[4] + c8[5] + c8[6] + c8[7];
        }
        for (; base + 128 <= e1; base += 128) {
            uint32_t s0 = __ldg(in_adj + base + lane);
            uint32_t s1 = __ldg(in_adj + base + 32 + lane);
            uint32_t s2 = __ldg(in_adj + base + 64 + lane);
            uint32_t s3 = __ldg(in_adj + base + 96 + lane);
            part += (Acc)S::dec(contrib[s0]) + (Acc)S::dec(contrib[s1]) +
                    (Acc)S::dec(contrib[s2]) + (Acc)S::dec(contrib[s3]);
        }
        for (; base < e1; base += 32) {
            uint64_t e = base + lane;
            if (e < e1) part += (Acc)S::dec(contrib[__ldg(in_adj + e)]);
        }
        part = dev::warp_sum(part);
        if (lane == 0) partial[c] = part;
    }
}

// Heavy row totals, partials summed in chunk order (deterministic).
template <int DT, bool ACC64, bool ADD_OLD, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_pr_heavy_finalize(HeavyRows H, const typename std::conditional<ACC64, double, float>::type *partial,
                    float *y_f32, double *y_f64, PrState *st, float scale_inv_arg, int stage) {
    using Acc = typename std::conditional<ACC64, double, float>::type;
    if (pr_idle(st, stage)) return;
    const float sinv = st ? st->scale_inv : scale_inv_arg;
    double ysum = 0;
    for (uint32_t h = blockIdx.x * BLOCK + threadIdx.x; h < H.nheavy; h += gridDim.x * BLOCK) {
        Acc acc = 0;
        for (uint64_t c = H.first[h]; c < H.first[h + 1]; ++c) acc += partial[c];
        if (DT == GG_FP8E4M3 || DT == GG_F16) acc *= (Acc)sinv;
        const uint32_t d = H.v[h];
        if (y_f64) {
            double v = ADD_OLD ? y_f64[d] + (double)acc : (double)acc;
            y_f64[d] = v;
            ysum += v;
        } else {
            float v = ADD_OLD ? (float)((double)y_f32[d] + (double)acc) : (float)acc;
            y_f32[d] = v;
            ysum += (double)v;
        }
    }
    if (st) {
        ysum = dev::block_sum<double, BLOCK>(ysum);
        if (threadIdx.x == 0) atomicAdd(&st->s1, ysum);
    }
}

template <int DT, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_pr_update(const XT<DT> *__restrict__ y, XT<DT> *__restrict__ x, typename Store<DT>::T *contrib,
            const uint64_t *__restrict__ off, uint32_t n, float damp, double damp64, int renorm_f32, PrState *st,
            int stage, float *acc = nullptr) {
    using S = Store<DT>;
    if (pr_idle(st, stage)) return;
    const int it = st->iters;
    const bool sr = DT == GG_BF16 && st->sr;
    const bool accum = acc && it >= st->avg_from;
    const double s1 = st->s1;
    const double w = (1.0 - s1) / (double)n;
    const double s2 = s1 + (double)n * w;
    const float wf32 = 1.0f / (float)s2;
    const double wf64 = 1.0 / s2;
    const float enc_scale = st->scale;
    double dl = 0;
    float cm = 0.0f;
    const uint32_t stride = gridDim.x * BLOCK;
    if constexpr (DT == GG_F64) {
        // all double: y += w, renormalise by 1/s, contrib = d * x / deg
        for (uint32_t v = blockIdx.x * BLOCK + threadIdx.x; v < n; v += stride) {
            const double yv = (y[v] + w) * wf64;
            dl += fabs(x[v] - yv);
            x[v] = yv;
            const uint64_t deg = off[v + 1] - off[v];
            contrib[v] = damp64 * yv / (double)deg;
        }
        (void)wf32;
        (void)enc_scale;
    } else
    for (uint32_t v = blockIdx.x * BLOCK + threadIdx.x; v < n; v += stride) {
        float yv = (float)((double)y[v] + w);
        yv = renorm_f32 ? yv * wf32 : (float)((double)yv * wf64);
        const float xv = x[v];
        dl += (double)fabsf(xv - yv);
        x[v] = yv;
        const uint64_t deg = off[v + 1] - off[v];
        const float c = damp * yv / (float)deg;
        if constexpr (DT == GG_BF16) {
            contrib[v] = sr ? bf16_stochastic(c, v, (uint32_t)it) : S::enc(c);
            if (accum) acc[v] += yv;
        } else {
            contrib[v] = S::enc(scaled_format(DT) ? c * enc_scale : c);
        }
        if (deg && c > cm) cm = c;
    }
    dl = dev::block_sum<double, BLOCK>(dl);
    // max of non-negative floats: integer order of the bit patterns
    __shared__ float sh[BLOCK / 32];
    for (int o = 16; o > 0; o >>= 1) cm = fmaxf(cm, __shfl_xor_sync(FULL, cm, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = cm;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (int i = 0; i < BLOCK / 32; ++i) b = fmaxf(b, sh[i]);
        atomicAdd(&st->delta, dl);
        atomicMax((int *)&st->cmax, __float_as_int(b));
    }
}

__global__ void k_pr_finish(PrState *st, int dt) {
    st->reencode = 0;
    if (st->done) return;
    const int it = st->iters;
    if (st->avg_from >= 0 && it >= st->avg_from) st->avg_n++;
    if (it < GG_MAX_ITERS) st->deltas[it] = st->delta;
    st->iters = it + 1;
    if (st->nstages > 1) dt = st->stage_dt[st->stage];
    if (st->stage + 1 < st->nstages && !(st->delta > st->stage_tol[st->stage])) {
        // next stage: its re-encode kernels rewrite the contributions from x
        st->stage++;
        st->reencode = 1;
        if (st->iters >= st->maxiter) st->done = 1;
    } else {
        if (st->iters >= st->maxiter || !(st->delta > st->tol)) st->done = 1;
        st->scale_inv = 1.0f / st->scale;     // decode of what the update just wrote
        st->scale = scale_for(dt, st->cmax);  // next encode
    }
    st->s1 = 0;
    st->delta = 0;
    st->cmax = 0.0f;
}

// Tail averaging: the ranks become the mean of the accumulated iterations.
__global__ void k_pr_average(float *x, const float *acc, uint32_t n, const PrState *st) {
    const int k = st->avg_n;
    if (k <= 0) return;
    const float inv = 1.0f / (float)k;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) x[v] = acc[v] * inv;
}

// Scale of the contributions about to be encoded, from the max found by the
// pass-0 kernel (one thread, between the two passes: every CTA of pass 1
// then reads the same value).  stage >= 0: only when that stage re-encodes.
__global__ void k_pr_setscale(PrState *st, int dt, int stage) {
    if (stage >= 0 && (st->done || !st->reencode || st->stage != stage)) return;
    const float sc = scale_for(dt, st->cmax);
    st->scale = sc;
    st->scale_inv = 1.0f / sc;
    st->cmax = 0.0f;
}

// A new stage's contributions from the current ranks: pass 0 finds the
// max, pass 1 encodes with st->scale.
template <int DT, int BLOCK>
__global__ void k_pr_reencode(const float *x, typename Store<DT>::T *contrib, const uint64_t *off, uint32_t n,
                              float damp, PrState *st, int stage, int pass) {
    using S = Store<DT>;
    if (st->done || !st->reencode || st->stage != stage) return;
    float cm = 0.0f;
    const float scale = st->scale;
    const uint32_t stride = gridDim.x * BLOCK;
    for (uint32_t v = blockIdx.x * BLOCK + threadIdx.x; v < n; v += stride) {
        const uint64_t deg = off[v + 1] - off[v];
        const float c = damp * x[v] / (float)deg;
        if (pass == 0) {
            if (deg && c > cm) cm = c;
        } else {
            contrib[v] = S::enc(scaled_format(DT) ? c * scale : c);
        }
    }
    if (pass == 0) {
        for (int o = 16; o > 0; o >>= 1) cm = fmaxf(cm, __shfl_xor_sync(FULL, cm, o));
        if ((threadIdx.x & 31) == 0) atomicMax((int *)&st->cmax, __float_as_int(cm));
    }
}

// Initial x = 1/n, contrib = d*x/deg (PRv.C:155-182); first pass finds the max.
template <int DT, int BLOCK>
__global__ void k_pr_init(XT<DT> *x, typename Store<DT>::T *contrib, const uint64_t *off, uint32_t n,
                          float damp, double damp64, PrState *st, int pass) {
    using S = Store<DT>;
    const float x0 = 1.0f / (float)n;
    float cm = 0.0f;
    const uint32_t stride = gridDim.x * BLOCK;
    if constexpr (DT == GG_F64) {
        if (pass == 1)
            for (uint32_t v = blockIdx.x * BLOCK + threadIdx.x; v < n; v += stride) {
                const double xd = 1.0 / (double)n;
                x[v] = xd;
                contrib[v] = damp64 * xd / (double)(off[v + 1] - off[v]);
            }
        if (pass == 1 && blockIdx.x == 0 && threadIdx.x == 0) {
            st->scale = 1.0f;
            st->scale_inv = 1.0f;
            st->cmax = 0.0f;
        }
        return;
    }
    const float scale = pass == 1 ? st->scale : 1.0f;  // set by k_pr_setscale between the passes
    for (uint32_t v = blockIdx.x * BLOCK + threadIdx.x; v < n; v += stride) {
        const uint64_t deg = off[v + 1] - off[v];
        const float c = damp * x0 / (float)deg;
        if (pass == 0) {
            if (deg && c > cm) cm = c;
        } else {
            x[v] = x0;
            contrib[v] = S::enc(scaled_format(DT) ? c * scale : c);
        }
    }
    if (pass == 0) {
        for (int o = 16; o > 0; o >>= 1) cm = fmaxf(cm, __shfl_xor_sync(FULL, cm, o));
        if ((threadIdx.x & 31) == 0) atomicMax((int *)&st->cmax, __float_as_int(cm));
    }
}

constexpr int kBlock = 256;

static unsigned pr_grid(gg_ctx *ctx, uint64_t work) {
    uint64_t b = (work + kBlock - 1) / kBlock;
    uint64_t cap = (uint64_t)ctx->sm_count * tuning().pr_blocks_per_sm;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

// gather of one iteration / one API call: light rows, heavy chunks, heavy totals
template <int DT, bool ACC64, bool ADD_OLD>
static gg_status gather_launch(gg_graph *g, const typename Store<DT>::T *contrib, float *yf,
                               double *yd, PrState *st, float sinv, void *partial, int stage = -1) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    using Acc = typename std::conditional<ACC64, double, float>::type;
    const HeavyRows &H = g->heavy;
    const uint64_t warps = (uint64_t)((g->n + 31) / 32);
    uint64_t blocks = (warps * 32 + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->sm_count * tuning().pr_blocks_per_sm;
    if (blocks > cap) blocks = cap;
    k_pr_gather<DT, ACC64, ADD_OLD, 256><<<(unsigned)(blocks ? blocks : 1), 256, 0, s>>>(
        g->in_off, g->in_adj, contrib, g->n, yf, yd, st, sinv, tuning().pull_k, H.T, tuning().pr_stream,
        H.light_prefix, stage);
    GG_LAUNCHED(ctx);
    if (H.nchunks) {
        uint64_t cb = (H.nchunks * 32 + 255) / 256;
        if (cb > cap) cb = cap;
        k_pr_heavy_chunks<DT, ACC64><<<(unsigned)cb, 256, 0, s>>>(g->in_off, g->in_adj, contrib, H,
                                                                  (Acc *)partial, st, stage);
        GG_LAUNCHED(ctx);
        uint64_t fb = (H.nheavy + 255) / 256;
        if (fb > cap) fb = cap;
        k_pr_heavy_finalize<DT, ACC64, ADD_OLD, 256><<<(unsigned)fb, 256, 0, s>>>(H, (const Acc *)partial, yf, yd,
                                                                                 st, sinv, stage);
        GG_LAUNCHED(ctx);
    }
    return GG_OK;
}

// Damping of the FP64 variant: the shortest decimal that rounds to the float
// parameter (0.85f -> 0.85), as the double-precision reference uses it.
static double damping_f64(float d) {
    char buf[32];
    for (int prec = 1; prec <= 9; ++prec) {
        std::snprintf(buf, sizeof(buf), "%.*g", prec, (double)d);
        const double v = std::strtod(buf, nullptr);
        if ((float)v == d) return v;
    }
    return (double)d;
}

template <int DT>
static gg_status pr_run(gg_graph *g, const gg_pr_params *p, XT<DT> *x, XT<DT> *y, void *contrib,
                        PrState *st, void *partial, float *acc = nullptr) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    using T = typename Store<DT>::T;
    const uint32_t n = g->n;
    const unsigned gv = pr_grid(ctx, n);
    const double d64 = damping_f64(p->damping);
    k_pr_init<DT, kBlock><<<gv, kBlock, 0, s>>>(x, (T *)contrib, g->off, n, p->damping, d64, st, 0);
    GG_LAUNCHED(ctx);
    k_pr_setscale<<<1, 1, 0, s>>>(st, DT, -1);
    GG_LAUNCHED(ctx);
    k_pr_init<DT, kBlock><<<gv, kBlock, 0, s>>>(x, (T *)contrib, g->off, n, p->damping, d64, st, 1);
    GG_LAUNCHED(ctx);
    float *yf = DT == GG_F64 ? nullptr : (float *)y;
    double *yd = DT == GG_F64 ? (double *)y : nullptr;
    for (int it = 0; it < p->maxiter; ++it) {
        if (p->accum_f64 || DT == GG_F64)
            GG_CHECK((gather_launch<DT, true, false>(g, (const T *)contrib, yf, yd, st, 1.0f, partial)));
        else
            GG_CHECK((gather_launch<DT, false, false>(g, (const T *)contrib, yf, yd, st, 1.0f, partial)));
        k_pr_update<DT, kBlock><<<gv, kBlock, 0, s>>>(y, x, (T *)contrib, g->off, n, p->damping, d64,
                                                      p->renorm_f32, st, -1, acc);
        GG_LAUNCHED(ctx);
        k_pr_finish<<<1, 1, 0, s>>>(st, DT);
        GG_LAUNCHED(ctx);
    }
    if constexpr (DT == GG_BF16) {
        if (acc) {
            k_pr_average<<<gv, kBlock, 0, s>>>(x, acc, n, st);
            GG_LAUNCHED(ctx);
        }
    }
    return GG_OK;
}

// Staged runs (PR_vary.C:652-757, e.g. VARIANT 4620 = run_prec_46 with
// customfp<6,10> contributions until the residual is below 1e-3, then
// run_prec_20 with FP32 contributions and double sums until 1e-7): every
// iteration launches each stage's kernels and those of inactive stages return
// at once, so the switch is taken on the device without a host round trip.
enum { OP_GATHER, OP_UPDATE, OP_REENC0, OP_SETSCALE, OP_REENC1, OP_INIT0, OP_INIT1 };

template <int DT>
static gg_status stage_op(gg_graph *g, int op, int stage, bool acc64, const gg_pr_params *p, float *x, float *y,
                          void *contrib, PrState *st, void *partial) {
    using T = typename Store<DT>::T;
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    const unsigned gv = pr_grid(ctx, g->n);
    switch (op) {
    case OP_GATHER:
        if (acc64) return gather_launch<DT, true, false>(g, (const T *)contrib, y, nullptr, st, 1.0f, partial, stage);
        return gather_launch<DT, false, false>(g, (const T *)contrib, y, nullptr, st, 1.0f, partial, stage);
    case OP_UPDATE:
        k_pr_update<DT, kBlock><<<gv, kBlock, 0, s>>>(y, x, (T *)contrib, g->off, g->n, p->damping, 0.0,
                                                      p->renorm_f32, st, stage);
        break;
    case OP_REENC0:
    case OP_REENC1:
        k_pr_reencode<DT, kBlock><<<gv, kBlock, 0, s>>>(x, (T *)contrib, g->off, g->n, p->damping, st, stage,
                                                        op == OP_REENC1);
        break;
    case OP_SETSCALE: k_pr_setscale<<<1, 1, 0, s>>>(st, DT, stage); break;
    default:
        k_pr_init<DT, kBlock><<<gv, kBlock, 0, s>>>(x, (T *)contrib, g->off, g->n, p->damping, 0.0, st,
                                                    op == OP_INIT1);
        break;
    }
    GG_LAUNCHED(ctx);
    return GG_OK;
}

static gg_status stage_dispatch(int dt, gg_graph *g, int op, int stage, bool acc64, const gg_pr_params *p,
                                float *x, float *y, void *contrib, PrState *st, void *partial) {
    switch (dt) {
    case GG_F32: return stage_op<GG_F32>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    case GG_BF16: return stage_op<GG_BF16>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    case GG_F16: return stage_op<GG_F16>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    case GG_FP8E4M3: return stage_op<GG_FP8E4M3>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    case GG_CFP_6_10: return stage_op<GG_CFP_6_10>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    default: return stage_op<GG_BF16_TRUNC>(g, op, stage, acc64, p, x, y, contrib, st, partial);
    }
}

static gg_status pr_run_staged(gg_graph *g, const gg_pr_params *p, float *x, float *y, void *contrib,
                               PrState *st, void *partial) {
    const int ns = p->nstages;
    const int *dt = p->stage_dtype;
    const int *acc = p->stage_accum_f64;
    GG_CHECK(stage_dispatch(dt[0], g, OP_INIT0, -1, false, p, x, y, contrib, st, partial));
    GG_CHECK(stage_dispatch(dt[0], g, OP_SETSCALE, -1, false, p, x, y, contrib, st, partial));
    GG_CHECK(stage_dispatch(dt[0], g, OP_INIT1, -1, false, p, x, y, contrib, st, partial));
    for (int it = 0; it < p->maxiter; ++it) {
        for (int k = 0; k < ns; ++k)
            GG_CHECK(stage_dispatch(dt[k], g, OP_GATHER, k, acc[k] != 0, p, x, y, contrib, st, partial));
        for (int k = 0; k < ns; ++k)
            GG_CHECK(stage_dispatch(dt[k], g, OP_UPDATE, k, false, p, x, y, contrib, st, partial));
        k_pr_finish<<<1, 1, 0, g->ctx->stream>>>(st, dt[0]);
        GG_LAUNCHED(g->ctx);
        for (int k = 1; k < ns; ++k) {
            GG_CHECK(stage_dispatch(dt[k], g, OP_REENC0, k, false, p, x, y, contrib, st, partial));
            GG_CHECK(stage_dispatch(dt[k], g, OP_SETSCALE, k, false, p, x, y, contrib, st, partial));
            GG_CHECK(stage_dispatch(dt[k], g, OP_REENC1, k, false, p, x, y, contrib, st, partial));
        }
    }
    return GG_OK;
}

// ADD_GATHER edgemap: y[d] += sum_{s in in(d), s active} dec(contrib[s]) * scale.
template <int DT>
static gg_status gather_api(gg_graph *g, const gg_emap_desc *d) {
    using T = typename Store<DT>::T;
    float *yf = d->a->t == GG_F32 ? (float *)d->a->d : nullptr;
    double *yd = d->a->t == GG_F64 ? (double *)d->a->d : nullptr;
    const float sc = d->src_scale != 0.0f ? d->src_scale : 1.0f;
    void *partial = nullptr;
    GG_CHECK(graph_scratch(g, (g->heavy.nchunks + 1) * 8, &partial));
    if (d->accum_f64)
        return gather_launch<DT, true, true>(g, (const T *)d->src->d, yf, yd, nullptr, sc, partial);
    return gather_launch<DT, false, true>(g, (const T *)d->src->d, yf, yd, nullptr, sc, partial);
}

// ADD_GATHER with a source frontier (APRv.C:477-487, api::filter(F, strong,
// src)): y[d] += sum over in-edges (s, d) with s in F of contrib[s].  The
// contributions of the vertices outside F are masked to zero in a scratch
// copy (one pass over n values), which the regular gather then sums: its
// light-row streaming and heavy-row chunks keep every warp busy whatever
// the degree mix.
template <typename T>
__global__ void k_mask_contrib(const T *__restrict__ contrib, const uint32_t *__restrict__ bits, uint32_t n,
                               T *__restrict__ out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[v] = dev::bit_test(bits, v) ? contrib[v] : (T)0;
}

static gg_status gather_src_filtered(gg_graph *g, const gg_emap_desc *d, gg_frontier *in) {
    gg_ctx *ctx = g->ctx;
    const bool f64 = d->src->t == GG_F64;
    if (!(d->src->t == GG_F32 || (f64 && d->accum_f64)))
        return set_error(ctx, GG_ERR_UNSUPPORTED, "a source-filtered ADD_GATHER takes F32 or F64 contributions");
    GG_CHECK(frontier_ensure_bitmap(in));
    float *yf = d->a->t == GG_F32 ? (float *)d->a->d : nullptr;
    double *yd = d->a->t == GG_F64 ? (double *)d->a->d : nullptr;
    // scratch: the masked contributions, then the heavy rows' partial sums
    const size_t esz = f64 ? 8 : 4;
    const size_t cb = (((size_t)g->n + 1) * esz + 255) / 256 * 256;
    void *base = nullptr;
    GG_CHECK(graph_scratch(g, cb + (g->heavy.nchunks + 1) * 8, &base));
    void *partial = (char *)base + cb;
    const unsigned grid = pr_grid(ctx, g->n);
    if (f64) {
        k_mask_contrib<double><<<grid, 256, 0, ctx->stream>>>((const double *)d->src->d, in->bitmap, g->n,
                                                              (double *)base);
        GG_LAUNCHED(ctx);
        return gather_launch<GG_F64, true, true>(g, (const double *)base, yf, yd, nullptr, 1.0f, partial);
    }
    k_mask_contrib<float><<<grid, 256, 0, ctx->stream>>>((const float *)d->src->d, in->bitmap, g->n, (float *)base);
    GG_LAUNCHED(ctx);
    if (d->accum_f64) return gather_launch<GG_F32, true, true>(g, (const float *)base, yf, yd, nullptr, 1.0f, partial);
    return gather_launch<GG_F32, false, true>(g, (const float *)base, yf, yd, nullptr, 1.0f, partial);
}

gg_status pr_edgemap_gather(gg_graph *g, const gg_emap_desc *d, gg_frontier *in) {
    gg_ctx *ctx = g->ctx;
    if (!d->src || d->src->g != g) return set_error(ctx, GG_ERR_ARG, "ADD_GATHER needs a contribution property of g");
    if (d->a->t != GG_F32 && d->a->t != GG_F64) return set_error(ctx, GG_ERR_ARG, "ADD_GATHER accumulator must be F32 or F64");
    if (d->dst_filter != GG_FILTER_NONE) return set_error(ctx, GG_ERR_UNSUPPORTED, "ADD_GATHER takes no dst filter");
    if (d->src_scale != 0.0f && d->src->t != GG_FP8E4M3)
        return set_error(ctx, GG_ERR_UNSUPPORTED, "src_scale applies to FP8 contributions only");
    if (in && !in->all) return gather_src_filtered(g, d, in);
    switch (d->src->t) {
    case GG_F32: return gather_api<GG_F32>(g, d);
    case GG_BF16: return gather_api<GG_BF16>(g, d);
    case GG_F16: return gather_api<GG_F16>(g, d);
    case GG_FP8E4M3: return gather_api<GG_FP8E4M3>(g, d);
    case GG_CFP_6_10: return gather_api<GG_CFP_6_10>(g, d);
    case GG_BF16_TRUNC: return gather_api<GG_BF16_TRUNC>(g, d);
    case GG_F64:  // PR_vary VARIANT 11: double contributions, double sums
        if (!d->accum_f64) return set_error(ctx, GG_ERR_UNSUPPORTED, "double contributions take double sums");
        return gather_api<GG_F64>(g, d);
    default: return set_error(ctx, GG_ERR_UNSUPPORTED, "contribution dtype");
    }
}

}  // namespace gg

using namespace gg;

extern "C" gg_status gg_pagerank(gg_graph *g, const gg_pr_params *p, gg_prop *x, float *host_x,
                                 gg_run_stats *stats) {
    if (!g || !p) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    if (p->maxiter < 0 || p->maxiter > GG_MAX_ITERS) return set_error(ctx, GG_ERR_ARG, "maxiter out of range");
    const bool staged = p->nstages > 1;
    const int dt = staged ? p->stage_dtype[0] : p->contrib_dtype;
    auto known = [](int t) {
        return t == GG_F32 || t == GG_BF16 || t == GG_F16 || t == GG_FP8E4M3 || t == GG_CFP_6_10 || t == GG_BF16_TRUNC;
    };
    if (p->nstages < 0 || p->nstages > 4) return set_error(ctx, GG_ERR_ARG, "nstages must be 0..4");
    if (staged)
        for (int k = 0; k < p->nstages; ++k)
            if (!known(p->stage_dtype[k])) return set_error(ctx, GG_ERR_UNSUPPORTED, "stage contribution dtype");
    if (!staged && !known(dt) && dt != GG_F64) return set_error(ctx, GG_ERR_UNSUPPORTED, "contribution dtype");
    if ((p->stochastic || p->average_last) && (staged || dt != GG_BF16))
        return set_error(ctx, GG_ERR_UNSUPPORTED, "stochastic rounding / tail averaging apply to BF16 runs only");
    if (p->average_last < 0) return set_error(ctx, GG_ERR_ARG, "average_last must be >= 0");
    const gg_dtype xt = dt == GG_F64 ? GG_F64 : GG_F32;
    if (x && (x->g != g || x->t != xt))
        return set_error(ctx, GG_ERR_ARG, "x must be an F32 property of g (F64 for the FP64 variant)");
    if (g->n == 0) return GG_OK;
    gg_prop *xp = x, *tmpx = nullptr;
    if (!xp) {
        GG_CHECK(gg_prop_create(g, xt, &tmpx));
        xp = tmpx;
    }
    // scratch: y (f32 / f64), contrib (up to 8 B), state
    const size_t esz = dt == GG_F64 ? 8 : 4;
    const size_t nb = (((size_t)g->n + 1) * esz + 255) / 256 * 256;
    const size_t sb = (sizeof(PrState) + 255) / 256 * 256;
    void *base = nullptr;
    const size_t ab = p->average_last > 0 ? (((size_t)g->n + 1) * 4 + 255) / 256 * 256 : 0;
    gg_status s = graph_scratch(g, 2 * nb + sb + ab + (g->heavy.nchunks + 1) * 8, &base);
    if (s != GG_OK) { if (tmpx) gg_prop_destroy(tmpx); return s; }
    float *y = (float *)base;
    void *contrib = (char *)base + nb;
    PrState *st = (PrState *)((char *)base + 2 * nb);
    float *acc = ab ? (float *)((char *)base + 2 * nb + sb) : nullptr;
    void *partial = (char *)base + 2 * nb + sb + ab;
    PrState init;
    memset(&init, 0, sizeof(init));
    init.maxiter = p->maxiter;
    init.tol = p->tol;
    init.scale = 1.0f;
    init.scale_inv = 1.0f;
    init.done = p->maxiter == 0;
    init.nstages = staged ? p->nstages : 1;
    for (int k = 0; k < 4; ++k) {
        init.stage_dt[k] = staged && k < p->nstages ? p->stage_dtype[k] : dt;
        init.stage_tol[k] = staged && k + 1 < p->nstages ? p->stage_tol[k] : p->tol;
    }
    init.sr = p->stochastic ? 1 : 0;
    init.avg_from = p->average_last > 0 ? std::max(0, p->maxiter - p->average_last) : -1;
    uint64_t k0 = ctx->launches;
    cudaEventRecord(ctx->ev0, ctx->stream);
    cudaError_t e = cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && acc) e = cudaMemsetAsync(acc, 0, (size_t)g->n * 4, ctx->stream);
    if (e == cudaSuccess) {
        if (staged) {
            s = pr_run_staged(g, p, (float *)xp->d, y, contrib, st, partial);
        } else switch (dt) {
        case GG_F64: s = pr_run<GG_F64>(g, p, (double *)xp->d, (double *)base, contrib, st, partial); break;
        case GG_F32: s = pr_run<GG_F32>(g, p, (float *)xp->d, y, contrib, st, partial); break;
        case GG_BF16: s = pr_run<GG_BF16>(g, p, (float *)xp->d, y, contrib, st, partial, acc); break;
        case GG_F16: s = pr_run<GG_F16>(g, p, (float *)xp->d, y, contrib, st, partial); break;
        case GG_FP8E4M3: s = pr_run<GG_FP8E4M3>(g, p, (float *)xp->d, y, contrib, st, partial); break;
        case GG_CFP_6_10: s = pr_run<GG_CFP_6_10>(g, p, (float *)xp->d, y, contrib, st, partial); break;
        default: s = pr_run<GG_BF16_TRUNC>(g, p, (float *)xp->d, y, contrib, st, partial); break;
        }
    } else {
        s = cuda_error(ctx, e, "gg_pagerank state upload");
    }
    cudaEventRecord(ctx->ev1, ctx->stream);
    PrState fin;
    if (s == GG_OK) {
        e = cudaMemcpyAsync(&fin, st, sizeof(fin), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) s = cuda_error(ctx, e, "gg_pagerank");
    }
    if (s == GG_OK && stats) {
        memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->total_ms = ms;
        stats->iterations = fin.iters;
        stats->kernels = ctx->launches - k0;
        for (int i = 0; i < fin.iters && i < GG_MAX_ITERS; ++i) {
            stats->delta[i] = fin.deltas[i];
            stats->variant[i] = GG_VAR_PULL_DENSE;
            stats->scanned[i] = g->m;
            stats->nactv[i] = g->n;
            stats->nacte[i] = g->m;
        }
        stats->scanned_edges = (uint64_t)fin.iters * g->m;
    }
    if (s == GG_OK && host_x) {
        if (xt == GG_F64) {  // the float copy of the double ranks
            std::vector<double> hx(g->n);
            s = gg_prop_download(xp, hx.data());
            for (uint32_t v = 0; s == GG_OK && v < g->n; ++v) host_x[v] = (float)hx[v];
        } else {
            s = gg_prop_download(xp, host_x);
        }
    }
    if (tmpx) gg_prop_destroy(tmpx);
    return s;
}
