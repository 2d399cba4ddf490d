// gg_batch.cu -- batched traversals.
//
//  * Multi-source BFS (up to 64 roots at once): one uint64 word per vertex
//    holds a bit per root for the frontier, the next frontier and the visited
//    set; an iteration is a push (OR frontier bits into out-neighbours' next
//    words, 64-bit atomicOr) or a pull (OR in-neighbours' frontier words, exit
//    early once every still-unvisited root has reached the vertex), chosen by
//    the m/20 rule on the frontier's vertex and edge counts.  The whole run is
//    one cooperative launch with the bounded grid barrier of gg_grid.cuh.
//    Levels are written per (vertex, root): level[v*64 + i].
//  * Personalized PageRank for up to 128 seeds: x_s <- alpha*e_s +
//    (1-alpha)*A^T D^-1 x_s.  The contribution matrix c[v][s] = x_s[v]/deg(v)
//    is stored in bfloat16, one 256-byte row per vertex, so every gathered
//    edge is one coalesced row read by a warp (lane = 4 seeds); sums are
//    float32.  Hub rows are cut into chunks (HeavyRows) summed by separate
//    warps into float32 partials.  The iteration loop is captured once into a
//    CUDA graph and launched as one graph.
//  * Disjoint union of many graphs on the device (gg_graph_union), so BFS
//    from every part's root and CC of every part run as one traversal.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "gg_batch.h"
#include "gg_grid.cuh"
#include "gg_internal.cuh"

namespace gg {

constexpr unsigned FULLB = 0xffffffffu;
constexpr int kBB = 256;
constexpr unsigned long long kMsPushDiv = 4;  // push while |F| + outdeg(F) <= m / 4

// ---------------------------------------------------------------------------
// Multi-source BFS
// ---------------------------------------------------------------------------
struct MsState {
    grid::Barrier bar;
    int iterations;
    unsigned long long nfront, efront;        // current frontier: vertices, edges
    unsigned long long nnext, enext;          // being accumulated
    unsigned long long reached_e;             // sum over roots of the out-degrees reached
    unsigned long long t_ns[GG_MAX_ITERS + 1];
    int variant[GG_MAX_ITERS];
};

struct MsArgs {
    const uint64_t *off, *in_off;
    const uint32_t *adj, *in_adj;
    uint32_t n;
    uint64_t m;
    unsigned long long *visited, *front, *next;
    int32_t *level;  // [n][64]
    unsigned long long all;  // mask of the roots in use
    MsState *st;
    unsigned long long timeout_ns;
    int max_iters;
    int K;
    HeavyRows H;     // CSC rows longer than H.T edges, cut into H.CH-edge chunks
    int symmetric;   // the chunks also cut the CSR rows (push)
};

template <typename T> __device__ __forceinline__ T ldcgb(const T *p) { return __ldcg(p); }

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long x) {
    const unsigned lo = __reduce_or_sync(FULLB, (unsigned)x);
    const unsigned hi = __reduce_or_sync(FULLB, (unsigned)(x >> 32));
    return ((unsigned long long)hi << 32) | lo;
}

// Push: out-edges of frontier vertices OR their frontier bits (minus the
// target's visited bits) into the target's next word.  Light rows: a warp
// per 32 vertices (lanes alone up to K edges, then the warp per long row);
// heavy rows of a symmetric graph: a warp per chunk.
__device__ void ms_push(const MsArgs &A, uint64_t gw, uint64_t nw, uint32_t lane) {
    const uint32_t T = A.symmetric ? A.H.T : 0xFFFFFFFFu;
    for (uint64_t w = gw; w * 32 < A.n; w += nw) {
        const uint32_t v = (uint32_t)(w * 32 + lane);
        const unsigned long long f = v < A.n ? ldcgb(A.front + v) : 0ull;
        uint64_t beg = 0, end = 0;
        if (f) {
            beg = A.off[v];
            end = A.off[v + 1];
            if (end - beg > T) end = beg;  // chunked below
        }
        const uint32_t k1 = (uint32_t)min(end - beg, (uint64_t)A.K);
        for (uint32_t k = 0; k < k1; ++k) {
            const uint32_t u = __ldg(A.adj + beg + k);
            const unsigned long long nv = f & ~ldcgb(A.visited + u);
            if (nv) atomicOr(A.next + u, nv);
        }
        unsigned pend = __ballot_sync(FULLB, f && beg + k1 < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULLB, beg + k1, j), endj = __shfl_sync(FULLB, end, j);
            const unsigned long long fj = __shfl_sync(FULLB, f, j);
            for (uint64_t e = ej + lane; e < endj; e += 32) {
                const uint32_t u = __ldg(A.adj + e);
                const unsigned long long nv = fj & ~ldcgb(A.visited + u);
                if (nv) atomicOr(A.next + u, nv);
            }
        }
    }
    if (!A.symmetric) return;
    for (uint64_t c = gw; c < A.H.nchunks; c += nw) {
        const uint32_t h = A.H.crow[c];
        const uint32_t v = A.H.v[h];
        const unsigned long long f = ldcgb(A.front + v);
        if (!f) continue;
        const uint64_t e0 = A.off[v] + (c - A.H.first[h]) * A.H.CH;
        const uint64_t e1 = min(e0 + A.H.CH, A.off[v + 1]);
        for (uint64_t e = e0 + lane; e < e1; e += 32) {
            const uint32_t u = __ldg(A.adj + e);
            const unsigned long long nv = f & ~ldcgb(A.visited + u);
            if (nv) atomicOr(A.next + u, nv);
        }
    }
}

// Pull: a vertex ORs its in-neighbours' frontier words until every root it
// has not been reached from is present.  Light rows: each warp a contiguous
// range of 32-vertex words of equal light-edge work; heavy rows: a warp per
// chunk, atomicOr of the chunk's new bits.
__device__ void ms_pull(const MsArgs &A, uint64_t gw, uint64_t nw, uint32_t lane) {
    const uint32_t nwords = (A.n + 31) / 32;
    uint32_t wlo, whi;
    dev::balanced_range(A.H.light_prefix, nwords, gw, nw, wlo, whi);
    for (uint32_t w = wlo; w < whi; ++w) {
        const uint32_t v = w * 32 + lane;
        const bool valid = v < A.n;
        const unsigned long long vis = valid ? ldcgb(A.visited + v) : A.all;
        uint64_t e = 0, end = 0;
        if (valid && vis != A.all) {
            e = A.in_off[v];
            end = A.in_off[v + 1];
            if (end - e > A.H.T) end = e;  // heavy: chunked below
        }
        bool act = e < end;
        unsigned long long acc = 0;
        const uint64_t lim = min(end, e + (uint64_t)A.K);
        for (; act && e < lim; ++e) {
            acc |= ldcgb(A.front + __ldg(A.in_adj + e));
            if ((acc | vis) == A.all) act = false;
        }
        unsigned pend = __ballot_sync(FULLB, act && e < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULLB, e, j), endj = __shfl_sync(FULLB, end, j);
            const unsigned long long visj = __shfl_sync(FULLB, vis, j);
            unsigned long long accj = __shfl_sync(FULLB, acc, j);
            for (uint64_t base = ej; base < endj; base += 32) {
                const uint64_t ed = base + lane;
                accj |= warp_or64(ed < endj ? ldcgb(A.front + __ldg(A.in_adj + ed)) : 0ull);
                if ((accj | visj) == A.all) break;
            }
            if ((int)lane == j) acc = accj;
        }
        const unsigned long long nx = acc & ~vis;
        if (valid && nx) A.next[v] = nx;
    }
    for (uint64_t c = gw; c < A.H.nchunks; c += nw) {
        const uint32_t h = A.H.crow[c];
        const uint32_t v = A.H.v[h];
        const unsigned long long vis = ldcgb(A.visited + v);
        if (vis == A.all) continue;
        const uint64_t e0 = A.in_off[v] + (c - A.H.first[h]) * A.H.CH;
        const uint64_t e1 = min(e0 + A.H.CH, A.in_off[v + 1]);
        unsigned long long acc = 0;
        for (uint64_t base = e0; base < e1; base += 32) {
            const uint64_t ed = base + lane;
            acc |= warp_or64(ed < e1 ? ldcgb(A.front + __ldg(A.in_adj + ed)) : 0ull);
            if ((acc | vis) == A.all) break;
        }
        const unsigned long long nx = acc & ~vis;
        if (lane == 0 && nx) atomicOr(A.next + v, nx);
    }
}

__global__ void __launch_bounds__(kBB) k_msbfs(MsArgs A) {
    MsState *st = A.st;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * kBB) >> 5;
    const uint64_t gw = ((uint64_t)blockIdx.x * kBB + threadIdx.x) >> 5;
    const uint64_t tid = (uint64_t)blockIdx.x * kBB + threadIdx.x, nth = (uint64_t)gridDim.x * kBB;
    if (blockIdx.x == 0 && threadIdx.x == 0) st->t_ns[0] = grid::globaltimer();
    int iter = 0;
    for (; iter < A.max_iters; ++iter) {
        const unsigned long long nf = ldcgb(&st->nfront), ef = ldcgb(&st->efront);
        if (nf == 0) break;
        // a pull scans most in-edges (it stops early only once every root
        // has reached the vertex), a push only the frontier's out-edges
        const bool push = (nf + ef) <= A.m / kMsPushDiv;
        if (blockIdx.x == 0 && threadIdx.x == 0 && iter < GG_MAX_ITERS)
            st->variant[iter] = push ? GG_VAR_PUSH_DENSE : GG_VAR_PULL_DENSE;
        if (push) ms_push(A, gw, nw, lane);
        else ms_pull(A, gw, nw, lane);
        if (!grid::sync(&st->bar, A.timeout_ns)) return;
        // update: visited, levels, next frontier, counts
        unsigned long long cnt = 0, edg = 0, red = 0;
        for (uint64_t v = tid; v < A.n; v += nth) {
            const unsigned long long nx = ldcgb(A.next + v);
            A.front[v] = nx;
            if (nx) {
                A.next[v] = 0ull;
                A.visited[v] = ldcgb(A.visited + v) | nx;
                const uint64_t deg = A.off[v + 1] - A.off[v];
                cnt++;
                edg += deg;
                red += deg * (unsigned long long)__popcll(nx);
                for (unsigned long long b = nx; b; b &= b - 1) A.level[v * 64 + (__ffsll((long long)b) - 1)] = iter + 1;
            }
        }
        cnt = dev::block_sum<unsigned long long, kBB>(cnt);
        edg = dev::block_sum<unsigned long long, kBB>(edg);
        red = dev::block_sum<unsigned long long, kBB>(red);
        if (threadIdx.x == 0) {
            if (cnt) atomicAdd(&st->nnext, cnt);
            if (edg) atomicAdd(&st->enext, edg);
            if (red) atomicAdd(&st->reached_e, red);
        }
        if (!grid::sync(&st->bar, A.timeout_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->nfront = st->nnext;
            st->efront = st->enext;
            st->nnext = 0;
            st->enext = 0;
            if (iter < GG_MAX_ITERS) st->t_ns[iter + 1] = grid::globaltimer();
        }
        if (!grid::sync(&st->bar, A.timeout_ns)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->iterations = iter;
}

__global__ void k_ms_init(MsArgs A) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    const int32_t inf = (int32_t)(A.n + 1);
    for (uint64_t i = tid; i < (uint64_t)A.n * 64; i += nth) A.level[i] = inf;
    for (uint64_t v = tid; v < A.n; v += nth) {
        A.visited[v] = 0;
        A.front[v] = 0;
        A.next[v] = 0;
    }
}

__global__ void k_ms_roots(MsArgs A, const uint32_t *roots, int k) {
    // one thread: roots may repeat
    if (blockIdx.x || threadIdx.x) return;
    unsigned long long nf = 0, ef = 0;
    for (int i = 0; i < k; ++i) {
        const uint32_t r = roots[i];
        if (A.front[r] == 0) {
            nf++;
            ef += A.off[r + 1] - A.off[r];
        }
        A.front[r] |= 1ull << i;
        A.visited[r] |= 1ull << i;
        A.level[(uint64_t)r * 64 + i] = 0;
        A.st->reached_e += A.off[r + 1] - A.off[r];
    }
    A.st->nfront = nf;
    A.st->efront = ef;
}

// ---------------------------------------------------------------------------
// Personalized PageRank, 128 seeds, bfloat16 rows
// ---------------------------------------------------------------------------
constexpr int kPprSeeds = 128;  // 4 per lane

struct PprArgs {
    const uint64_t *in_off, *off;
    const uint32_t *in_adj;
    uint32_t n;
    const uint2 *cin;   // [n] rows of 128 bf16 (uint2 = 4 bf16 per lane)
    uint2 *cout;        // next contributions
    uint2 *xout;        // ranks (bf16), written by the last iteration only (else null)
    const uint32_t *seeds;  // [128]
    float alpha;
    HeavyRows H;
    float4 *partial;    // [nchunks][32] float4 per lane
};

__device__ __forceinline__ void bf4_acc(uint2 v, float4 &a) {
    a.x += __uint_as_float(v.x << 16);
    a.y += __uint_as_float(v.x & 0xFFFF0000u);
    a.z += __uint_as_float(v.y << 16);
    a.w += __uint_as_float(v.y & 0xFFFF0000u);
}

__device__ __forceinline__ uint2 f4_to_bf4(float4 f) {
    uint2 r;
    r.x = (uint32_t)dev::bf16_rne(f.x) | ((uint32_t)dev::bf16_rne(f.y) << 16);
    r.y = (uint32_t)dev::bf16_rne(f.z) | ((uint32_t)dev::bf16_rne(f.w) << 16);
    return r;
}

// x = alpha*e_seed + (1-alpha)*acc; c = x/deg; written as bf16 rows
__device__ __forceinline__ void ppr_finish(const PprArgs &A, uint32_t d, float4 acc, uint32_t lane) {
    const float b = 1.0f - A.alpha;
    float4 x = make_float4(b * acc.x, b * acc.y, b * acc.z, b * acc.w);
    const uint32_t s0 = lane * 4;
    if (A.seeds[s0] == d) x.x += A.alpha;
    if (A.seeds[s0 + 1] == d) x.y += A.alpha;
    if (A.seeds[s0 + 2] == d) x.z += A.alpha;
    if (A.seeds[s0 + 3] == d) x.w += A.alpha;
    const uint64_t deg = A.off[d + 1] - A.off[d];
    const float inv = deg ? 1.0f / (float)deg : 0.0f;
    if (A.xout) A.xout[(uint64_t)d * 32 + lane] = f4_to_bf4(x);
    A.cout[(uint64_t)d * 32 + lane] = f4_to_bf4(make_float4(x.x * inv, x.y * inv, x.z * inv, x.w * inv));
}

// light rows: a warp per row
__global__ void __launch_bounds__(kBB) k_ppr_light(PprArgs A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * kBB) >> 5;
    for (uint64_t d = ((uint64_t)blockIdx.x * kBB + threadIdx.x) >> 5; d < A.n; d += nw) {
        const uint64_t beg = A.in_off[d], end = A.in_off[d + 1];
        if (end - beg > A.H.T) continue;  // heavy: chunked kernels
        float4 acc = make_float4(0, 0, 0, 0);
        uint64_t e = beg;
        for (; e + 4 <= end; e += 4) {  // four rows in flight
            const uint32_t u0 = __ldg(A.in_adj + e), u1 = __ldg(A.in_adj + e + 1), u2 = __ldg(A.in_adj + e + 2),
                           u3 = __ldg(A.in_adj + e + 3);
            const uint2 r0 = A.cin[(uint64_t)u0 * 32 + lane], r1 = A.cin[(uint64_t)u1 * 32 + lane],
                        r2 = A.cin[(uint64_t)u2 * 32 + lane], r3 = A.cin[(uint64_t)u3 * 32 + lane];
            bf4_acc(r0, acc);
            bf4_acc(r1, acc);
            bf4_acc(r2, acc);
            bf4_acc(r3, acc);
        }
        for (; e < end; ++e) bf4_acc(A.cin[(uint64_t)__ldg(A.in_adj + e) * 32 + lane], acc);
        ppr_finish(A, (uint32_t)d, acc, lane);
    }
}

// heavy rows: a warp per chunk, float partials
__global__ void __launch_bounds__(kBB) k_ppr_heavy(PprArgs A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * kBB) >> 5;
    for (uint64_t c = ((uint64_t)blockIdx.x * kBB + threadIdx.x) >> 5; c < A.H.nchunks; c += nw) {
        const uint32_t h = A.H.crow[c];
        const uint32_t v = A.H.v[h];
        const uint64_t e0 = A.in_off[v] + (c - A.H.first[h]) * A.H.CH;
        const uint64_t e1 = min(e0 + A.H.CH, A.in_off[v + 1]);
        float4 acc = make_float4(0, 0, 0, 0);
        for (uint64_t e = e0; e < e1; ++e) bf4_acc(A.cin[(uint64_t)__ldg(A.in_adj + e) * 32 + lane], acc);
        A.partial[c * 32 + lane] = acc;
    }
}

__global__ void __launch_bounds__(kBB) k_ppr_heavy_finish(PprArgs A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * kBB) >> 5;
    for (uint64_t h = ((uint64_t)blockIdx.x * kBB + threadIdx.x) >> 5; h < A.H.nheavy; h += nw) {
        float4 acc = make_float4(0, 0, 0, 0);
        for (uint64_t c = A.H.first[h]; c < A.H.first[h + 1]; ++c) {
            const float4 p = A.partial[c * 32 + lane];
            acc.x += p.x;
            acc.y += p.y;
            acc.z += p.z;
            acc.w += p.w;
        }
        ppr_finish(A, A.H.v[h], acc, lane);
    }
}

__global__ void k_ppr_init(uint2 *c, uint2 *x, const uint64_t *off, uint32_t n, const uint32_t *seeds) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < (uint64_t)n * 32; i += nth) {
        const uint32_t d = (uint32_t)(i / 32), lane = (uint32_t)(i % 32);
        float4 xv = make_float4(seeds[lane * 4] == d, seeds[lane * 4 + 1] == d, seeds[lane * 4 + 2] == d,
                                seeds[lane * 4 + 3] == d);
        const uint64_t deg = off[d + 1] - off[d];
        const float inv = deg ? 1.0f / (float)deg : 0.0f;
        x[i] = f4_to_bf4(xv);
        c[i] = f4_to_bf4(make_float4(xv.x * inv, xv.y * inv, xv.z * inv, xv.w * inv));
    }
}

__global__ void k_ppr_unpack(const uint2 *x, uint32_t n, int k, float *out) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < (uint64_t)n * k; i += nth) {
        const uint64_t d = i / k;
        const uint32_t s = (uint32_t)(i % k);
        const uint2 r = x[d * 32 + s / 4];
        const uint32_t word = (s & 2) ? r.y : r.x;
        out[i] = __uint_as_float((s & 1) ? (word & 0xFFFF0000u) : (word << 16));
    }
}

// ---------------------------------------------------------------------------
// Disjoint union
// ---------------------------------------------------------------------------
__global__ void k_union_part(const uint64_t *off, const uint32_t *adj, uint32_t n, uint64_t m, uint64_t ebase,
                             uint32_t vbase, uint64_t *uoff, uint32_t *uadj) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < n; v += nth) uoff[vbase + v] = off[v] + ebase;
    for (uint64_t e = tid; e < m; e += nth) uadj[ebase + e] = adj[e] + vbase;
}

__global__ void k_set_u64(uint64_t *p, uint64_t v) { *p = v; }

static unsigned bgrid(gg_ctx *ctx, uint64_t work) {
    uint64_t b = (work + kBB - 1) / kBB, cap = (uint64_t)ctx->sm_count * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace gg

using namespace gg;

extern "C" {

gg_status gg_msbfs(gg_graph *g, const uint32_t *roots, int k, int32_t *host_levels, gg_run_stats *stats) {
    if (!g || !roots || k < 1 || k > 64) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    for (int i = 0; i < k; ++i)
        if (roots[i] >= g->n) return set_error(ctx, GG_ERR_ARG, "gg_msbfs: root out of range");
    cudaStream_t s = ctx->stream;
    const uint64_t n = g->n;
    // scratch: visited, front, next (8n each), levels (256n), roots, state
    const size_t words = (3 * n + 1) * 8, lev = n * 64 * 4;
    void *base;
    GG_CHECK(graph_scratch(g, words + lev + 64 * 4 + sizeof(MsState) + 512, &base));
    char *p = (char *)base;
    MsArgs A;
    std::memset(&A, 0, sizeof(A));
    A.visited = (unsigned long long *)p;
    A.front = A.visited + n;
    A.next = A.front + n;
    A.level = (int32_t *)(p + words);
    uint32_t *droots = (uint32_t *)(p + words + lev);
    MsState *st = (MsState *)(((uintptr_t)(p + words + lev + 64 * 4) + 255) & ~(uintptr_t)255);
    A.off = g->off;
    A.adj = g->adj;
    A.in_off = g->in_off;
    A.in_adj = g->in_adj;
    A.n = g->n;
    A.m = g->m;
    A.all = k == 64 ? ~0ull : ((1ull << k) - 1);
    A.st = st;
    A.timeout_ns = tuning().barrier_timeout_ns;
    A.max_iters = (int)std::min<uint64_t>(n + 2, 1u << 30);
    A.K = tuning().pull_k;
    A.H = g->heavy;
    A.symmetric = g->symmetric;
    GG_CUDA(ctx, cudaMemcpyAsync(droots, roots, k * 4, cudaMemcpyHostToDevice, s));
    GG_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(MsState), s));
    cudaEventRecord(ctx->ev0, s);
    k_ms_init<<<bgrid(ctx, n * 64), kBB, 0, s>>>(A);
    GG_LAUNCHED(ctx);
    k_ms_roots<<<1, 32, 0, s>>>(A, droots, k);
    GG_LAUNCHED(ctx);
    const int per_sm = resident_ctas((const void *)k_msbfs, kBB);
    void *args[] = {&A};
    GG_CUDA(ctx, cudaLaunchCooperativeKernel((const void *)k_msbfs, dim3(ctx->sm_count * per_sm), dim3(kBB), args, 0, s));
    ctx->launches++;
    cudaEventRecord(ctx->ev1, s);
    MsState hs;
    GG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
    GG_CUDA(ctx, cudaStreamSynchronize(s));
    if (hs.bar.err & DEV_ERR_TIMEOUT) return set_error(ctx, GG_ERR_TIMEOUT, "gg_msbfs: grid barrier timed out");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->total_ms = ms;
        stats->iterations = hs.iterations;
        stats->edges_reached = hs.reached_e;
        for (int i = 0; i < std::min(hs.iterations, GG_MAX_ITERS); ++i) {
            stats->variant[i] = hs.variant[i];
            stats->iter_ms[i] = (hs.t_ns[i + 1] - hs.t_ns[i]) * 1e-6;
            stats->kernel_ms[i] = stats->iter_ms[i];
        }
    }
    if (host_levels) {
        // [n][64] on the device -> [n][k] on the host
        std::vector<int32_t> tmp(n * 64);
        GG_CUDA(ctx, cudaMemcpy(tmp.data(), A.level, n * 64 * 4, cudaMemcpyDeviceToHost));
        for (uint64_t v = 0; v < n; ++v)
            std::memcpy(host_levels + v * k, tmp.data() + v * 64, k * 4);
    }
    return GG_OK;
}

gg_status gg_ppr(gg_graph *g, const uint32_t *seeds, int k, float alpha, int iters, float *host_x,
                 gg_run_stats *stats) {
    if (!g || !seeds || k < 1 || k > kPprSeeds || !(alpha > 0 && alpha < 1) || iters < 0) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    for (int i = 0; i < k; ++i)
        if (seeds[i] >= g->n) return set_error(ctx, GG_ERR_ARG, "gg_ppr: seed out of range");
    cudaStream_t s = ctx->stream;
    const uint64_t n = g->n;
    const size_t row = 256;  // 128 bf16
    const size_t part = (g->heavy.nchunks + 1) * 32 * sizeof(float4);
    void *base;
    GG_CHECK(graph_scratch(g, 3 * n * row + part + 512 + 1024, &base));
    char *p = (char *)base;
    uint2 *c0 = (uint2 *)p, *c1 = (uint2 *)(p + n * row), *x = (uint2 *)(p + 2 * n * row);
    float4 *partial = (float4 *)(p + 3 * n * row);
    uint32_t *dseeds = (uint32_t *)(p + 3 * n * row + part);
    std::vector<uint32_t> sd(kPprSeeds, 0xFFFFFFFFu);  // unused slots match no vertex
    std::memcpy(sd.data(), seeds, k * 4);
    GG_CUDA(ctx, cudaMemcpyAsync(dseeds, sd.data(), kPprSeeds * 4, cudaMemcpyHostToDevice, s));
    GG_CUDA(ctx, cudaStreamSynchronize(s));
    PprArgs A;
    std::memset(&A, 0, sizeof(A));
    A.in_off = g->in_off;
    A.off = g->off;
    A.in_adj = g->in_adj;
    A.n = g->n;
    A.seeds = dseeds;
    A.alpha = alpha;
    A.H = g->heavy;
    A.partial = partial;
    const unsigned gl = (unsigned)(ctx->sm_count * resident_ctas((const void *)k_ppr_light, kBB));
    const unsigned gh = (unsigned)(ctx->sm_count * resident_ctas((const void *)k_ppr_heavy, kBB));
    // capture the iteration loop once (on a private stream), then run
    // init + the graph on the context stream between the timing events
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs;
    GG_CUDA(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    for (int it = 0; it < iters && e == cudaSuccess; ++it) {
        A.cin = (it & 1) ? c1 : c0;
        A.cout = (it & 1) ? c0 : c1;
        A.xout = it + 1 == iters ? x : nullptr;  // only the ranks of the last iteration are kept
        k_ppr_light<<<gl, kBB, 0, cs>>>(A);
        if (A.H.nchunks) {
            k_ppr_heavy<<<gh, kBB, 0, cs>>>(A);
            k_ppr_heavy_finish<<<bgrid(ctx, (uint64_t)A.H.nheavy * 32), kBB, 0, cs>>>(A);
        }
        ctx->launches += A.H.nchunks ? 3 : 1;
    }
    if (e == cudaSuccess) {
        e = cudaStreamEndCapture(cs, &graph);
    } else {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(cs, &junk);
        if (junk) cudaGraphDestroy(junk);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, s);
    if (e == cudaSuccess) {
        k_ppr_init<<<bgrid(ctx, n * 32), kBB, 0, s>>>(c0, x, g->off, g->n, dseeds);
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && iters) e = cudaGraphLaunch(exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return cuda_error(ctx, e, "gg_ppr");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->total_ms = ms;
        stats->iterations = iters;
        stats->scanned_edges = (uint64_t)iters * g->m;
    }
    if (host_x) {
        float *dx = nullptr;
        GG_CUDA(ctx, cudaMalloc(&dx, n * k * 4));
        k_ppr_unpack<<<bgrid(ctx, n * k), kBB, 0, s>>>(x, g->n, k, dx);
        ctx->launches++;
        cudaError_t ee = cudaMemcpyAsync(host_x, dx, n * k * 4, cudaMemcpyDeviceToHost, s);
        if (ee == cudaSuccess) ee = cudaStreamSynchronize(s);
        cudaFree(dx);
        if (ee != cudaSuccess) return cuda_error(ctx, ee, "gg_ppr download");
    }
    return GG_OK;
}

gg_status gg_graph_union(gg_ctx *ctx, gg_graph *const *parts, int k, gg_graph **out, uint32_t *vertex_base) {
    if (!ctx || !parts || k < 1 || !out) return GG_ERR_ARG;
    uint64_t n = 0, m = 0;
    int sym = 1;
    bool sorted = true;  // a part's rows keep their order, shifted by its vertex base
    for (int i = 0; i < k; ++i) {
        if (!parts[i] || parts[i]->ctx != ctx) return set_error(ctx, GG_ERR_ARG, "gg_graph_union: bad part");
        sorted &= parts[i]->rows_sorted;
        if (vertex_base) vertex_base[i] = (uint32_t)n;
        n += parts[i]->n;
        m += parts[i]->m;
        sym &= parts[i]->symmetric;
    }
    if (vertex_base) vertex_base[k] = (uint32_t)n;
    if (n >= 0xFFFFFFFFull) return set_error(ctx, GG_ERR_ARG, "gg_graph_union: more than 2^32-1 vertices");
    uint64_t *uoff = nullptr;
    uint32_t *uadj = nullptr;
    cudaStream_t s = ctx->stream;
    GG_CUDA(ctx, cudaMalloc(&uoff, (n + 1) * 8));
    cudaError_t e = cudaMalloc(&uadj, (m ? m : 1) * 4);
    if (e != cudaSuccess) { cudaFree(uoff); return cuda_error(ctx, e, "gg_graph_union"); }
    uint64_t eb = 0, vb = 0;
    for (int i = 0; i < k; ++i) {
        gg_graph *q = parts[i];
        k_union_part<<<bgrid(ctx, std::max<uint64_t>(q->n, q->m)), kBB, 0, s>>>(q->off, q->adj, q->n, q->m, eb,
                                                                                  (uint32_t)vb, uoff, uadj);
        ctx->launches++;
        eb += q->m;
        vb += q->n;
    }
    k_set_u64<<<1, 1, 0, s>>>(uoff + n, m);
    ctx->launches++;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { cudaFree(uoff); cudaFree(uadj); return cuda_error(ctx, e, "gg_graph_union"); }
    return graph_adopt_device_csr(ctx, (uint32_t)n, m, uoff, uadj, sym, sorted, out);
}

}  // extern "C"
