// gg_core.cu -- contexts, graphs, vertex properties and frontiers of libgg.so.
//
// Graph storage replaces Graptor's GraphCSx + VEBO/Graptor SIMD layout
// (include/graptor/graph/GraphCSx.h:293-2262, graph/CGraphVEBOGraptor.h:60-496)
// with a plain device CSR (out-edges, used by push) and CSC (in-edges, used by
// pull): uint64 offsets, uint32 vertex ids; rows are sorted when the graph is
// built on the device, and uploaded rows are checked (gg_graph::rows_sorted)
// but kept in the caller's order.  For symmetric graphs
// the CSC aliases the CSR.  Graph construction (generation, symmetrising,
// self-loop removal, de-duplication, transposition) runs on the device with a
// radix sort of packed (row, col) keys.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "gg_internal.cuh"

namespace gg {

gg_status set_error(gg_ctx *ctx, gg_status s, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return s;
}

gg_status cuda_error(gg_ctx *ctx, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return set_error(ctx, GG_ERR_OOM, m);
    return set_error(ctx, GG_ERR_CUDA, m);
}

size_t dtype_size(gg_dtype t) {
    switch (t) {
    case GG_I32: case GG_U32: case GG_F32: return 4;
    case GG_F64: return 8;
    case GG_BF16: case GG_F16: case GG_CFP_6_10: case GG_BF16_TRUNC: return 2;
    case GG_FP8E4M3: case GG_U8: return 1;
    }
    return 0;
}

Tuning &tuning() {
    static Tuning t;
    return t;
}

int resident_ctas(const void *kernel, int block) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(kernel, block);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    cache[key] = nb;
    return nb;
}

unsigned occ_grid(gg_ctx *ctx, const void *kernel, int block, uint64_t work_threads) {
    const uint64_t cap = (uint64_t)ctx->sm_count * resident_ctas(kernel, block);
    uint64_t b = (work_threads + block - 1) / block;
    if (b > cap) b = cap;
    return (unsigned)(b ? b : 1);
}

uint32_t bin_of_degree(uint64_t deg) {
    const Tuning &t = tuning();
    return deg <= t.bin_small_max ? 0u : (deg <= t.bin_medium_max ? 1u : 2u);
}

gg_status graph_scratch(gg_graph *g, size_t bytes, void **p) {
    if (bytes > g->scratch_bytes) {
        if (g->scratch) cudaFree(g->scratch);
        g->scratch = nullptr;
        g->scratch_bytes = 0;
        size_t want = bytes + bytes / 4;
        GG_CUDA(g->ctx, cudaMalloc(&g->scratch, want));
        g->scratch_bytes = want;
    }
    *p = g->scratch;
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Kernels: graph construction
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    // SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014).
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t mix64_h(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t stream_base(uint64_t seed, uint64_t stream) {
    return mix64_h(seed ^ mix64_h(stream + 0x51ED270B27A8C3F1ull));
}
static uint64_t prob_u32(double p) {
    double t = p * 4294967296.0;
    if (t < 0) t = 0;
    if (t > 4294967296.0) t = 4294967296.0;
    return (uint64_t)(t + 0.5);
}

// R-MAT: edge i, level l draws u = hi32(mix64(base + 64 i + l)); quadrant
// a/b/c/d by the cumulative thresholds; level 0 is the most significant bit.
__global__ void k_gen_rmat(uint64_t *keys, uint64_t nedges, int scale, int lg, uint64_t base,
                           uint64_t ta, uint64_t tb, uint64_t tc, int symmetric) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < nedges; i += stride) {
        uint32_t s = 0, d = 0;
        for (int l = 0; l < scale; ++l) {
            uint64_t u = mix64(base + i * 64 + (uint64_t)l) >> 32;
            uint32_t sb = u >= tb ? 1u : 0u;
            uint32_t db = ((u >= ta && u < tb) || u >= tc) ? 1u : 0u;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        keys[i] = ((uint64_t)s << lg) | d;
        if (symmetric) keys[nedges + i] = ((uint64_t)d << lg) | s;
    }
}

__global__ void k_gen_er(uint64_t *keys, uint64_t M, uint32_t n, int lg, uint64_t base,
                         uint64_t dbase, uint32_t dangling_bp, int symmetric) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < M; i += stride) {
        uint64_t h1 = mix64(base + 2 * i), h2 = mix64(base + 2 * i + 1);
        uint32_t s = (uint32_t)(((h1 >> 32) * (uint64_t)n) >> 32);
        uint32_t d = (uint32_t)(((h2 >> 32) * (uint64_t)n) >> 32);
        if (!symmetric && dangling_bp && (mix64(dbase + s) % 10000ull) < dangling_bp) d = s;
        keys[i] = ((uint64_t)s << lg) | d;
        if (symmetric) keys[M + i] = ((uint64_t)d << lg) | s;
    }
}

// Grid: each vertex u emits its right and down edges (both directions) unless
// deleted; absent edges become self-loops (dropped by the CSR build).
__global__ void k_gen_grid(uint64_t *keys, uint32_t rows, uint32_t cols, int lg, uint64_t base,
                           uint32_t del_bp) {
    uint64_t n = (uint64_t)rows * cols;
    uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; u < n; u += stride) {
        uint32_t r = (uint32_t)(u / cols), c = (uint32_t)(u % cols);
        uint64_t self = (u << lg) | u;
        bool h = c + 1 < cols && (mix64(base + 2 * u) % 10000ull) >= del_bp;
        bool v = r + 1 < rows && (mix64(base + 2 * u + 1) % 10000ull) >= del_bp;
        keys[4 * u + 0] = h ? ((u << lg) | (u + 1)) : self;
        keys[4 * u + 1] = h ? (((u + 1) << lg) | u) : self;
        keys[4 * u + 2] = v ? ((u << lg) | (u + cols)) : self;
        keys[4 * u + 3] = v ? (((u + cols) << lg) | u) : self;
    }
}

// keep[i] = not a self-loop and not a duplicate of key[i-1] (keys sorted)
__global__ void k_mark_unique(const uint64_t *keys, uint64_t nk, int lg, uint8_t *keep) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t mask = (lg >= 64) ? ~0ull : ((1ull << lg) - 1);
    for (; i < nk; i += stride) {
        uint64_t k = keys[i];
        bool self = (k >> lg) == (k & mask);
        bool dup = i > 0 && keys[i - 1] == k;
        keep[i] = (!self && !dup) ? 1 : 0;
    }
}

// adj[i] = column of key i; off[r] = first index of row r (rows sorted).
__global__ void k_keys_to_csr(const uint64_t *keys, uint64_t m, int lg, uint32_t n, uint64_t *off,
                              uint32_t *adj) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t mask = (1ull << lg) - 1;
    for (; i < m; i += stride) {
        uint64_t k = keys[i];
        uint32_t r = (uint32_t)(k >> lg);
        adj[i] = (uint32_t)(k & mask);
        uint64_t rp = (i == 0) ? 0 : (keys[i - 1] >> lg) + 1;
        if (i == 0) rp = 0;
        for (uint64_t v = rp; v <= r; ++v) off[v] = i;
        if (i == m - 1)
            for (uint64_t v = (uint64_t)r + 1; v <= n; ++v) off[v] = m;
    }
}

__global__ void k_fill_u64(uint64_t *p, uint64_t k, uint64_t val) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < k) p[i] = val;
}

// CSR -> transposed keys (col << lg | row), one warp per row.
__global__ void k_csr_to_tkeys(const uint64_t *off, const uint32_t *adj, uint32_t n, int lg,
                               uint64_t *keys) {
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t lane = threadIdx.x & 31;
    uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = warp; v < n; v += nw) {
        for (uint64_t e = off[v] + lane; e < off[v + 1]; e += 32)
            keys[e] = ((uint64_t)adj[e] << lg) | v;
    }
}

// Edge list -> sort keys (src << lg | dst), and the reverse edge when
// symmetrising; ids out of range raise *bad and become self-loops (dropped).
__global__ void k_edges_to_keys(const uint32_t *src, const uint32_t *dst, uint64_t ne, uint32_t n, int lg,
                                int sym, uint64_t *keys, uint32_t *bad) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ne; i += stride) {
        uint32_t s = src[i], d = dst[i];
        if (s >= n || d >= n) {
            atomicOr(bad, 1u);
            s = d = 0;
        }
        keys[i] = ((uint64_t)s << lg) | d;
        if (sym) keys[ne + i] = ((uint64_t)d << lg) | s;
    }
}

// CSR -> sort keys (src << lg | dst), plus the reverse edges when symmetrising
__global__ void k_csr_to_keys(const uint64_t *off, const uint32_t *adj, uint32_t n, int lg, int sym, uint64_t m,
                              uint64_t *keys) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = warp; v < n; v += nw)
        for (uint64_t e = off[v] + lane; e < off[v + 1]; e += 32) {
            const uint32_t d = adj[e];
            keys[e] = ((uint64_t)v << lg) | d;
            if (sym) keys[m + e] = ((uint64_t)d << lg) | v;
        }
}

__global__ void k_max_degree(const uint64_t *off, uint32_t n, unsigned long long *best) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    unsigned long long b = 0;
    for (; i < n; i += stride) {
        uint64_t d = off[i + 1] - off[i];
        // max degree, ties to the smallest id
        unsigned long long key = (d << 32) | (0xFFFFFFFFull - i);
        if (key > b) b = key;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        b = x > b ? x : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(best, b);
}

// chunks per CSC row (0 for light rows)
__global__ void k_heavy_count(const uint64_t *in_off, uint32_t n, uint32_t T, uint32_t CH,
                              uint8_t *flag, uint64_t *nch) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        uint64_t d = in_off[i + 1] - in_off[i];
        bool h = d > T;
        flag[i] = h ? 1 : 0;
        nch[i] = h ? (d + CH - 1) / CH : 0;
    }
}

__global__ void k_heavy_gather(const uint32_t *hv, uint32_t nh, const uint64_t *nch, uint64_t *cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nh) cnt[i] = nch[hv[i]];
    if (i == nh) cnt[i] = 0;
}

__global__ void k_nonzero_flags(const uint64_t *in_off, uint32_t n, uint8_t *flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (; i < n; i += stride) flag[i] = in_off[i + 1] > in_off[i] ? 1 : 0;
}

// per-word work estimates (see HeavyRows)
__global__ void k_word_costs(const uint64_t *in_off, uint32_t n, uint32_t T, uint64_t *light,
                             uint64_t *pull) {
    const uint32_t nwords = (n + 31) / 32;
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (; w < nwords; w += stride) {
        uint64_t cl = 0, cp = 0;
        for (uint32_t v = w * 32; v < min(n, w * 32 + 32); ++v) {
            const uint64_t d = in_off[v + 1] - in_off[v];
            cl += 4 + (d <= T ? d : 0);
            cp += 2 + (d < 16 ? d : 16);
        }
        light[w] = cl;
        pull[w] = cp;
    }
}

// crow[c] = heavy index owning chunk c
__global__ void k_heavy_crow(const uint64_t *first, uint32_t nh, uint32_t *crow) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    for (; h < nh; h += stride)
        for (uint64_t c = first[h]; c < first[h + 1]; ++c) crow[c] = h;
}

static int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l < 1 ? 1 : l;
}

static unsigned grid_for(gg_ctx *ctx, uint64_t work, int block = 256) {
    uint64_t b = (work + block - 1) / block;
    uint64_t cap = (uint64_t)ctx->sm_count * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// Sort keys (2*lg significant bits), drop self-loops and duplicates, build
// off[n+1] / adj[m].  keys is consumed (its buffer is reused).
static gg_status build_from_keys(gg_ctx *ctx, uint32_t n, uint64_t *keys, uint64_t nk, int lg,
                                 uint64_t **off_out, uint32_t **adj_out, uint64_t *m_out) {
    cudaStream_t st = ctx->stream;
    uint64_t *sorted = nullptr, *d_m = nullptr;
    uint8_t *keep = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    uint64_t *off = nullptr;
    uint32_t *adj = nullptr;
    uint64_t m = 0;
    gg_status rc = GG_OK;
    auto fail = [&](gg_status s) {
        cudaFree(sorted); cudaFree(keep); cudaFree(tmp); cudaFree(d_m);
        cudaFree(off); cudaFree(adj);
        return s;
    };
#define BK(expr) do { cudaError_t _e = (expr); if (_e != cudaSuccess) return fail(cuda_error(ctx, _e, #expr)); } while (0)
    if (nk > 0) {
        BK(cudaMalloc(&sorted, nk * sizeof(uint64_t)));
        BK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, sorted, (int64_t)nk, 0, 2 * lg, st));
        BK(cub::DeviceSelect::Flagged(nullptr, tb2, sorted, keep, keys, d_m, (int64_t)nk, st));
        if (tb2 > tmp_bytes) tmp_bytes = tb2;
        BK(cudaMalloc(&tmp, tmp_bytes));
        BK(cudaMalloc(&keep, nk));
        BK(cudaMalloc(&d_m, sizeof(uint64_t)));
        BK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, sorted, (int64_t)nk, 0, 2 * lg, st));
        ctx->launches++;
        k_mark_unique<<<grid_for(ctx, nk), 256, 0, st>>>(sorted, nk, lg, keep);
        ctx->launches++;
        BK(cub::DeviceSelect::Flagged(tmp, tmp_bytes, sorted, keep, keys, d_m, (int64_t)nk, st));
        ctx->launches++;
        BK(cudaMemcpyAsync(&m, d_m, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
    }
    BK(cudaMalloc(&off, ((size_t)n + 1) * sizeof(uint64_t)));
    BK(cudaMalloc(&adj, (m ? m : 1) * sizeof(uint32_t)));
    if (m > 0) {
        k_keys_to_csr<<<grid_for(ctx, m), 256, 0, st>>>(keys, m, lg, n, off, adj);
        ctx->launches++;
    } else {
        k_fill_u64<<<(n + 256) / 256, 256, 0, st>>>(off, (uint64_t)n + 1, 0);
        ctx->launches++;
    }
    BK(cudaGetLastError());
    BK(cudaStreamSynchronize(st));
    cudaFree(sorted); cudaFree(keep); cudaFree(tmp); cudaFree(d_m);
#undef BK
    *off_out = off;
    *adj_out = adj;
    *m_out = m;
    return rc;
}

gg_status build_heavy_rows(gg_graph *g) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    HeavyRows &H = g->heavy;
    H.T = tuning().heavy_deg;
    H.CH = tuning().heavy_chunk;
    const uint32_t n = g->n;
    uint8_t *flag = nullptr;
    uint64_t *nch = nullptr, *d_num = nullptr;
    void *tmp = nullptr;
    size_t tb = 0, tb2 = 0;
    gg_status rc = GG_OK;
    auto done = [&](gg_status s) { cudaFree(flag); cudaFree(nch); cudaFree(d_num); cudaFree(tmp); return s; };
#define HK(expr) do { cudaError_t _e = (expr); if (_e != cudaSuccess) return done(cuda_error(ctx, _e, #expr)); } while (0)
    HK(cudaMalloc(&flag, n + 1));
    HK(cudaMalloc(&nch, ((size_t)n + 1) * 8));
    HK(cudaMalloc(&d_num, 8));
    HK(cudaMalloc(&H.v, ((size_t)n + 1) * 4));
    k_heavy_count<<<grid_for(ctx, n), 256, 0, st>>>(g->in_off, n, H.T, H.CH, flag, nch);
    ctx->launches++;
    thrust::counting_iterator<uint32_t> it(0);
    HK(cub::DeviceSelect::Flagged(nullptr, tb, it, flag, H.v, d_num, (int64_t)n, st));
    HK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, nch, nch, (int64_t)n + 1, st));
    HK(cudaMalloc(&tmp, std::max(tb, tb2)));
    tb = std::max(tb, tb2);
    HK(cub::DeviceSelect::Flagged(tmp, tb, it, flag, H.v, d_num, (int64_t)n, st));
    ctx->launches++;
    uint64_t nh = 0;
    HK(cudaMemcpyAsync(&nh, d_num, 8, cudaMemcpyDeviceToHost, st));
    HK(cudaStreamSynchronize(st));
    H.nheavy = (uint32_t)nh;
    HK(cudaMalloc(&H.first, (nh + 1) * 8));
    k_heavy_gather<<<(unsigned)((nh + 256) / 256), 256, 0, st>>>(H.v, (uint32_t)nh, nch, H.first);
    ctx->launches++;
    HK(cub::DeviceScan::ExclusiveSum(tmp, tb, H.first, H.first, (int64_t)nh + 1, st));
    ctx->launches++;
    HK(cudaMemcpyAsync(&H.nchunks, H.first + nh, 8, cudaMemcpyDeviceToHost, st));
    HK(cudaStreamSynchronize(st));
    {
        const uint32_t nwords = (n + 31) / 32;
        HK(cudaMalloc(&H.light_prefix, ((size_t)nwords + 1) * 8));
        HK(cudaMalloc(&H.pull_prefix, ((size_t)nwords + 1) * 8));
        k_word_costs<<<grid_for(ctx, nwords), 256, 0, st>>>(g->in_off, n, H.T, H.light_prefix, H.pull_prefix);
        ctx->launches++;
        size_t tb3 = 0;
        HK(cub::DeviceScan::InclusiveSum(nullptr, tb3, H.light_prefix, H.light_prefix, (int64_t)nwords, st));
        if (tb3 > tb) {
            cudaFree(tmp);
            tmp = nullptr;
            HK(cudaMalloc(&tmp, tb3));
            tb = tb3;
        }
        if (nwords) {
            HK(cub::DeviceScan::InclusiveSum(tmp, tb, H.light_prefix, H.light_prefix, (int64_t)nwords, st));
            HK(cub::DeviceScan::InclusiveSum(tmp, tb, H.pull_prefix, H.pull_prefix, (int64_t)nwords, st));
            ctx->launches += 2;
        }
    }
    {
        // vertices with in-edges (the first pull's candidates)
        uint8_t *nz = flag;  // reuse: flag[v] = in-degree > 0
        k_nonzero_flags<<<grid_for(ctx, n), 256, 0, st>>>(g->in_off, n, nz);
        ctx->launches++;
        HK(cudaMalloc(&g->nonisolated, ((size_t)n + 1) * 4));
        HK(cudaMalloc(&g->nonisolated_n, 8));
        size_t tb4 = 0;
        HK(cub::DeviceSelect::Flagged(nullptr, tb4, it, nz, g->nonisolated, g->nonisolated_n, (int64_t)n, st));
        if (tb4 > tb) {
            cudaFree(tmp);
            tmp = nullptr;
            HK(cudaMalloc(&tmp, tb4));
            tb = tb4;
        }
        HK(cub::DeviceSelect::Flagged(tmp, tb, it, nz, g->nonisolated, g->nonisolated_n, (int64_t)n, st));
        ctx->launches++;
        HK(cudaStreamSynchronize(st));
    }
    HK(cudaMalloc(&H.crow, (H.nchunks + 1) * 4));
    if (nh) {
        k_heavy_crow<<<grid_for(ctx, nh), 256, 0, st>>>(H.first, (uint32_t)nh, H.crow);
        ctx->launches++;
        HK(cudaStreamSynchronize(st));
    }
#undef HK
    return done(rc);
}

__global__ void k_first_in(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_adj, uint32_t n,
                           uint4 *first_in) {
    for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < n; d += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = in_off[d], e = in_off[d + 1];
        const uint64_t deg = e - b;
        first_in[d] = make_uint4(b < e ? in_adj[b] : 0xFFFFFFFFu, b + 1 < e ? in_adj[b + 1] : 0xFFFFFFFFu,
                                 deg > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)deg,
                                 b + 2 < e ? in_adj[b + 2] : 0xFFFFFFFFu);
    }
}

__global__ void k_first1(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_adj, uint32_t n,
                         uint2 *first1) {
    for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < n; d += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = in_off[d], e = in_off[d + 1];
        const uint64_t deg = e - b;
        first1[d] = make_uint2(b < e ? in_adj[b] : 0xFFFFFFFFu, deg > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)deg);
    }
}

gg_status graph_ensure_first1(gg_graph *g) {
    if (g->first1) return GG_OK;
    gg_ctx *ctx = g->ctx;
    GG_CUDA(ctx, cudaMalloc(&g->first1, ((size_t)g->n + 1) * sizeof(uint2)));
    if (g->n) {
        k_first1<<<grid_for(ctx, g->n), 256, 0, ctx->stream>>>(g->in_off, g->in_adj, g->n, g->first1);
        GG_LAUNCHED(ctx);
    }
    return GG_OK;
}

static gg_status graph_finish(gg_graph *g) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    if (g->symmetric) {
        g->in_off = g->off;
        g->in_adj = g->adj;
    } else {
        int lg = ceil_log2(g->n);
        uint64_t *keys = nullptr;
        GG_CUDA(ctx, cudaMalloc(&keys, (g->m ? g->m : 1) * sizeof(uint64_t)));
        if (g->m) {
            k_csr_to_tkeys<<<grid_for(ctx, (uint64_t)g->n * 32), 256, 0, st>>>(g->off, g->adj, g->n, lg, keys);
            GG_LAUNCHED(ctx);
        }
        uint64_t mt = 0;
        gg_status s = build_from_keys(ctx, g->n, keys, g->m, lg, &g->in_off, &g->in_adj, &mt);
        cudaFree(keys);
        if (s != GG_OK) return s;
        if (mt != g->m) return set_error(ctx, GG_ERR_ARG, "graph has self-loops or duplicate edges");
    }
    // max-degree vertex (the BFS root of the small configuration)
    unsigned long long *d_best = nullptr, h_best = 0;
    GG_CUDA(ctx, cudaMalloc(&d_best, sizeof(unsigned long long)));
    GG_CUDA(ctx, cudaMemsetAsync(d_best, 0, sizeof(unsigned long long), st));
    if (g->n) {
        k_max_degree<<<grid_for(ctx, g->n), 256, 0, st>>>(g->off, g->n, d_best);
        GG_LAUNCHED(ctx);
    }
    GG_CUDA(ctx, cudaMemcpyAsync(&h_best, d_best, sizeof(h_best), cudaMemcpyDeviceToHost, st));
    GG_CUDA(ctx, cudaStreamSynchronize(st));
    cudaFree(d_best);
    g->maxdeg = (uint32_t)(h_best >> 32);
    g->maxdeg_v = g->n ? (uint32_t)(0xFFFFFFFFull - (h_best & 0xFFFFFFFFull)) : 0;
    GG_CUDA(ctx, cudaMalloc(&g->first_in, ((size_t)g->n + 1) * sizeof(uint4)));
    if (g->n) {
        k_first_in<<<grid_for(ctx, g->n), 256, 0, st>>>(g->in_off, g->in_adj, g->n, g->first_in);
        GG_LAUNCHED(ctx);
    }
    return build_heavy_rows(g);
}

static void graph_free(gg_graph *g) {
    if (!g) return;
    delete[] g->sel_h;
    cudaFree(g->sel_d);
    if (g->in_off && g->in_off != g->off) cudaFree(g->in_off);
    if (g->in_adj && g->in_adj != g->adj) cudaFree(g->in_adj);
    cudaFree(g->off);
    cudaFree(g->adj);
    cudaFree(g->scratch);
    cudaFree(g->aux_cnt);
    cudaFree(g->heavy.v);
    cudaFree(g->heavy.first);
    cudaFree(g->heavy.crow);
    cudaFree(g->nonisolated);
    cudaFree(g->nonisolated_n);
    cudaFree(g->first_in);
    cudaFree(g->first1);
    cudaFree(g->kc_alive[0]);
    cudaFree(g->kc_alive[1]);
    cudaFree(g->kc_cnt);
    cudaFree(g->pstate2);
    for (int i = 0; i < 2; ++i) {
        if (g->copy_done[i]) {
            cudaEventSynchronize(g->copy_done[i]);
            cudaEventDestroy(g->copy_done[i]);
        }
        if (g->async_level[i]) gg_prop_destroy(g->async_level[i]);
    }
    if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
    cudaFree(g->pstate);
    cudaFree(g->wq);
    graph_bfs_free(g);
    cudaFree(g->heavy.light_prefix);
    cudaFree(g->heavy.pull_prefix);
    cudaFree(g->cand.list[0]);
    cudaFree(g->cand.list[1]);
    cudaFree(g->cand.cnt);
    for (auto *f : g->tmp_front)
        if (f) gg_frontier_destroy(f);
    for (auto *p : g->tmp_prop)
        if (p) gg_prop_destroy(p);
    for (auto *b : g->pool_bins) cudaFree(b);
    for (auto *b : g->pool_bitmaps) cudaFree(b);
    for (auto *c : g->pool_cnt) cudaFree(c);
    delete g;
}

// ---------------------------------------------------------------------------
// Kernels: properties and frontiers
// ---------------------------------------------------------------------------
__global__ void k_fill_bytes(void *p, uint64_t n, uint64_t val, int esz) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        switch (esz) {
        case 1: ((uint8_t *)p)[i] = (uint8_t)val; break;
        case 2: ((uint16_t *)p)[i] = (uint16_t)val; break;
        case 4: ((uint32_t *)p)[i] = (uint32_t)val; break;
        default: ((uint64_t *)p)[i] = val; break;
        }
    }
}

// Single-vertex frontier: bins + counts (frontier::create(n, v, deg)).
__global__ void k_front_single(uint32_t v, const uint64_t *off, uint32_t *b0, uint32_t *b1,
                               uint32_t *b2, uint64_t *cnt, uint32_t smax, uint32_t mmax) {
    uint64_t deg = off[v + 1] - off[v];
    for (int i = 0; i < FC_WORDS; ++i) cnt[i] = 0;
    cnt[FC_NACTV] = 1;
    cnt[FC_NACTE] = deg;
    int b = deg <= smax ? 0 : (deg <= mmax ? 1 : 2);
    (b == 0 ? b0 : b == 1 ? b1 : b2)[0] = v;
    cnt[FC_BIN0 + b] = 1;
}

__global__ void k_front_set_counts(uint64_t *cnt, uint64_t nactv, uint64_t nacte) {
    for (int i = 0; i < FC_WORDS; ++i) cnt[i] = 0;
    cnt[FC_NACTV] = nactv;
    cnt[FC_NACTE] = nacte;
}

// Warp-aggregated append of v (when act) into its degree bin.
__device__ __forceinline__ void emit_binned(bool act, uint32_t v, uint32_t bin, uint32_t *b0,
                                            uint32_t *b1, uint32_t *b2,
                                            unsigned long long *cnt) {
    const unsigned am = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t b = 0; b < NBINS; ++b) {
        unsigned mk = __ballot_sync(am, act && bin == b);
        if (mk == 0) continue;
        int leader = __ffs(mk) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(cnt + FC_BIN0 + b, (unsigned long long)__popc(mk));
        base = __shfl_sync(am, base, leader);
        if (act && bin == b) {
            uint32_t *dst = b == 0 ? b0 : (b == 1 ? b1 : b2);
            dst[base + __popc(mk & ((1u << lane) - 1u))] = v;
        }
    }
}

// Bitmap (or all vertices when bm == nullptr) -> binned list + counts, the
// appends staged per warp in shared memory.
__global__ void __launch_bounds__(256) k_bitmap_to_list(const uint32_t *bm, uint32_t n, const uint64_t *off,
                                                        uint32_t *b0, uint32_t *b1, uint32_t *b2,
                                                        unsigned long long *cnt, uint32_t smax, uint32_t mmax) {
    __shared__ uint32_t sb[3][8][256];
    const uint32_t wib = threadIdx.x >> 5;
    gg::dev::WarpAppender<256> ap0{sb[0][wib], 0, b0, cnt + FC_BIN0};
    gg::dev::WarpAppender<256> ap1{sb[1][wib], 0, b1, cnt + FC_BIN1};
    gg::dev::WarpAppender<256> ap2{sb[2][wib], 0, b2, cnt + FC_BIN2};
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long nv = 0, ne = 0;
    gg::dev::bitmap_to_bins(bm, n, off, smax, mmax, ap0, ap1, ap2, nv, ne);
    ap0.flush();
    ap1.flush();
    ap2.flush();
    nv = gg::dev::warp_sum(nv);
    ne = gg::dev::warp_sum(ne);
    if (lane == 0 && nv) {
        atomicAdd(cnt + FC_NACTV, nv);
        atomicAdd(cnt + FC_NACTE, ne);
    }
}

// List (bins) -> bitmap (bitmap pre-cleared).
__global__ void k_list_to_bitmap(const uint32_t *b0, const uint32_t *b1, const uint32_t *b2,
                                 const uint64_t *cnt, uint32_t *bm) {
    uint64_t c0 = cnt[FC_BIN0], c1 = cnt[FC_BIN1], c2 = cnt[FC_BIN2];
    uint64_t tot = c0 + c1 + c2;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < tot; i += stride) {
        uint32_t v = i < c0 ? b0[i] : (i < c0 + c1 ? b1[i - c0] : b2[i - c0 - c1]);
        atomicOr(bm + (v >> 5), 1u << (v & 31));
    }
}

}  // namespace gg

using namespace gg;

// ---------------------------------------------------------------------------
// C ABI: status, context
// ---------------------------------------------------------------------------
extern "C" {

const char *gg_status_string(gg_status s) {
    switch (s) {
    case GG_OK: return "GG_OK";
    case GG_ERR_ARG: return "GG_ERR_ARG";
    case GG_ERR_OOM: return "GG_ERR_OOM";
    case GG_ERR_CUDA: return "GG_ERR_CUDA";
    case GG_ERR_TIMEOUT: return "GG_ERR_TIMEOUT";
    case GG_ERR_UNSUPPORTED: return "GG_ERR_UNSUPPORTED";
    case GG_ERR_IO: return "GG_ERR_IO";
    case GG_ERR_STATE: return "GG_ERR_STATE";
    case GG_ERR_NOT_FOUND: return "GG_ERR_NOT_FOUND";
    }
    return "GG_ERR_UNKNOWN";
}

size_t gg_dtype_size(gg_dtype t) { return dtype_size(t); }

gg_status gg_ctx_create(int device, gg_ctx **out) {
    if (!out) return GG_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return GG_ERR_NOT_FOUND;
    }
    if (device < 0 || device >= ndev) return GG_ERR_ARG;
    gg_ctx *c = new (std::nothrow) gg_ctx;
    if (!c) return GG_ERR_OOM;
    c->device = device;
    auto bail = [&](cudaError_t e) {
        gg_status s = e == cudaErrorMemoryAllocation ? GG_ERR_OOM : GG_ERR_CUDA;
        gg_ctx_destroy(c);
        return s;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e);
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return bail(e);
    c->sm_count = prop.multiProcessorCount;
    c->l2_bytes = prop.l2CacheSize;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
    c->own_stream = true;
    if ((e = cudaMalloc(&c->d_err, sizeof(uint32_t))) != cudaSuccess) return bail(e);
    if ((e = cudaMemset(c->d_err, 0, sizeof(uint32_t))) != cudaSuccess) return bail(e);
    if ((e = cudaMallocHost(&c->h_pinned, 64 * sizeof(uint64_t))) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreate(&c->evk0)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreate(&c->evk1)) != cudaSuccess) return bail(e);
    *out = c;
    return GG_OK;
}

gg_status gg_ctx_destroy(gg_ctx *ctx) {
    if (!ctx) return GG_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->evk0) cudaEventDestroy(ctx->evk0);
    if (ctx->evk1) cudaEventDestroy(ctx->evk1);
    delete ctx;
    return GG_OK;
}

gg_status gg_ctx_set_stream(gg_ctx *ctx, void *stream) {
    if (!ctx) return GG_ERR_ARG;
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        GG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return GG_OK;
}

gg_status gg_ctx_get_stream(gg_ctx *ctx, void **stream) {
    if (!ctx || !stream) return GG_ERR_ARG;
    *stream = (void *)ctx->stream;
    return GG_OK;
}

gg_status gg_ctx_sync(gg_ctx *ctx) {
    if (!ctx) return GG_ERR_ARG;
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t flag = 0;
    GG_CUDA(ctx, cudaMemcpy(&flag, ctx->d_err, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(ctx->d_err, 0, sizeof(uint32_t));
        if (flag & DEV_ERR_TIMEOUT) return set_error(ctx, GG_ERR_TIMEOUT, "device wait timed out");
        return set_error(ctx, GG_ERR_STATE, "device error flag " + std::to_string(flag));
    }
    return GG_OK;
}

const char *gg_last_error(gg_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

uint64_t gg_ctx_launch_count(gg_ctx *ctx) { return ctx ? ctx->launches : 0; }

gg_status gg_tuning_set(const char *name, int64_t v) {
    if (!name || v < 0) return GG_ERR_ARG;
    Tuning &t = tuning();
    std::string k(name);
    if (k == "barrier_timeout_ns") {
        if (v < 1) return GG_ERR_ARG;
        t.barrier_timeout_ns = (unsigned long long)v;
        return GG_OK;
    }
    if (v > (int64_t)1 << 31) return GG_ERR_ARG;
    const Tuning saved = t;  // an invalid combination leaves every knob as it was
    if (k == "bin_small_max") t.bin_small_max = (uint32_t)v;
    else if (k == "bin_medium_max") t.bin_medium_max = (uint32_t)v;
    else if (k == "pull_k" && v >= 1 && v <= 1024) t.pull_k = (int)v;
    else if (k == "pull_split" && (v == 0 || v == 1)) t.pull_split = (int)v;
    else if (k == "graph_flat" && (v == 0 || v == 1)) t.graph_flat = (int)v;
    else if (k == "graph_pdl" && (v == 0 || v == 1)) t.graph_pdl = (int)v;
    else if (k == "graph_unroll" && v >= 1 && v <= 4) t.graph_unroll = (int)v;
    else if (k == "pull_first" && v <= 4) t.pull_first = (int)v;
    else if (k == "pull_stage" && (v == 0 || v == 4 || v == 8 || v == 16 || v == 32)) t.pull_stage = (int)v;
    else if (k == "pull_fresh" && v <= 1) t.pull_fresh = (int)v;
    else if (k == "pull_ctas" && v >= 4 && v <= 8) t.pull_ctas = (int)v;
    else if (k == "push_ctas" && v >= 4 && v <= 8) t.push_ctas = (int)v;
    else if (k == "push_k" && v >= 1 && v <= 1024) t.push_k = (int)v;
    else if (k == "heavy_deg" && v >= 32) t.heavy_deg = (uint32_t)v;
    else if (k == "heavy_chunk" && v >= 32) t.heavy_chunk = (uint32_t)v;
    else if (k == "large_chunk" && v >= 256) t.large_chunk = (uint32_t)v;
    else if (k == "pr_stream" && v <= 1) t.pr_stream = (int)v;
    else if (k == "blocks_per_sm" && v >= 1 && v <= 32) t.blocks_per_sm = (int)v;
    else if (k == "pr_blocks_per_sm" && v >= 1 && v <= 32) t.pr_blocks_per_sm = (int)v;
    else if (k == "persistent" && v <= 7) t.persistent = (int)v;
    else if (k == "fusion" && (v == 0 || v == 4)) t.fusion = (int)v;
    else if (k == "fusion_queue" && (v == 0 || v >= 32)) t.fusion_queue = (uint32_t)v;
    else if (k == "cc_hook" && v <= 2) t.cc_hook = (int)v;
    else if (k == "graph" && v <= 1) t.graph = (int)v;
    else if (k == "graph_handoff" && v <= (1 << 20)) t.graph_handoff = (int)v;
    else if (k == "handoff_ctas" && v <= (1 << 16)) t.handoff_ctas = (int)v;
    else if (k == "small_frontier" && v <= 1) t.small_frontier = (int)v;
    else if (k == "barrier_timeout_ns" && v >= 1) t.barrier_timeout_ns = (unsigned long long)v;
    else return GG_ERR_ARG;
    if (t.bin_small_max > t.bin_medium_max) {
        t = saved;
        return GG_ERR_ARG;
    }
    return GG_OK;
}

gg_status gg_tuning_get(const char *name, int64_t *v) {
    if (!name || !v) return GG_ERR_ARG;
    const Tuning &t = tuning();
    std::string k(name);
    if (k == "bin_small_max") *v = t.bin_small_max;
    else if (k == "bin_medium_max") *v = t.bin_medium_max;
    else if (k == "pull_k") *v = t.pull_k;
    else if (k == "pull_split") *v = t.pull_split;
    else if (k == "graph_flat") *v = t.graph_flat;
    else if (k == "graph_pdl") *v = t.graph_pdl;
    else if (k == "graph_unroll") *v = t.graph_unroll;
    else if (k == "pull_first") *v = t.pull_first;
    else if (k == "pull_stage") *v = t.pull_stage;
    else if (k == "pull_fresh") *v = t.pull_fresh;
    else if (k == "pull_ctas") *v = t.pull_ctas;
    else if (k == "push_ctas") *v = t.push_ctas;
    else if (k == "push_k") *v = t.push_k;
    else if (k == "heavy_deg") *v = t.heavy_deg;
    else if (k == "heavy_chunk") *v = t.heavy_chunk;
    else if (k == "large_chunk") *v = t.large_chunk;
    else if (k == "pr_stream") *v = t.pr_stream;
    else if (k == "blocks_per_sm") *v = t.blocks_per_sm;
    else if (k == "pr_blocks_per_sm") *v = t.pr_blocks_per_sm;
    else if (k == "persistent") *v = t.persistent;
    else if (k == "fusion") *v = t.fusion;
    else if (k == "fusion_queue") *v = t.fusion_queue;
    else if (k == "cc_hook") *v = t.cc_hook;
    else if (k == "graph") *v = t.graph;
    else if (k == "graph_handoff") *v = t.graph_handoff;
    else if (k == "handoff_ctas") *v = t.handoff_ctas;
    else if (k == "small_frontier") *v = t.small_frontier;
    else if (k == "barrier_timeout_ns") *v = (int64_t)t.barrier_timeout_ns;
    else return GG_ERR_ARG;
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Graphs
// ---------------------------------------------------------------------------
gg_status gg_graph_upload(gg_ctx *ctx, uint32_t n, uint64_t m, const uint64_t *off,
                          const uint32_t *adj, int symmetric, gg_graph **out) {
    if (!ctx || !out || !off || (m && !adj) || n == 0xFFFFFFFFu) return set_error(ctx, GG_ERR_ARG, "gg_graph_upload: bad arguments");
    *out = nullptr;
    if (off[0] != 0 || off[n] != m) return set_error(ctx, GG_ERR_ARG, "gg_graph_upload: off[0] != 0 or off[n] != m");
    for (uint32_t v = 0; v < n; ++v)
        if (off[v] > off[v + 1]) return set_error(ctx, GG_ERR_ARG, "gg_graph_upload: offsets not monotone");
    bool sorted = true;  // min-id hooking stops a row at its first larger id when rows are sorted
    for (uint32_t v = 0; v < n; ++v)
        for (uint64_t e = off[v]; e < off[v + 1]; ++e) {
            if (adj[e] >= n) return set_error(ctx, GG_ERR_ARG, "gg_graph_upload: vertex id out of range");
            if (e > off[v] && adj[e] < adj[e - 1]) sorted = false;
        }
    GG_CUDA(ctx, cudaSetDevice(ctx->device));
    gg_graph *g = new (std::nothrow) gg_graph;
    if (!g) return GG_ERR_OOM;
    g->ctx = ctx;
    g->n = n;
    g->m = m;
    g->symmetric = symmetric ? 1 : 0;
    g->rows_sorted = sorted;
    cudaError_t e;
    if ((e = cudaMalloc(&g->off, ((size_t)n + 1) * 8)) != cudaSuccess ||
        (e = cudaMalloc(&g->adj, (m ? m : 1) * 4)) != cudaSuccess ||
        (e = cudaMemcpy(g->off, off, ((size_t)n + 1) * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (m && (e = cudaMemcpy(g->adj, adj, m * 4, cudaMemcpyHostToDevice)) != cudaSuccess)) {
        graph_free(g);
        return cuda_error(ctx, e, "gg_graph_upload");
    }
    gg_status s = graph_finish(g);
    if (s != GG_OK) { graph_free(g); return s; }
    *out = g;
    return GG_OK;
}

}  // extern "C"

namespace gg {
// Takes ownership of a CSR already in device memory (off: n+1, adj: m).
gg_status graph_adopt_device_csr(gg_ctx *ctx, uint32_t n, uint64_t m, uint64_t *off, uint32_t *adj, int symmetric,
                                 bool rows_sorted, gg_graph **out) {
    *out = nullptr;
    gg_graph *g = new (std::nothrow) gg_graph;
    if (!g) {
        cudaFree(off);
        cudaFree(adj);
        return GG_ERR_OOM;
    }
    g->ctx = ctx;
    g->n = n;
    g->m = m;
    g->symmetric = symmetric ? 1 : 0;
    g->rows_sorted = rows_sorted;
    g->off = off;
    g->adj = adj;
    gg_status s = graph_finish(g);
    if (s != GG_OK) { graph_free(g); return s; }
    *out = g;
    return GG_OK;
}
}  // namespace gg

extern "C" {

gg_status gg_graph_read_bin(gg_ctx *ctx, const char *path, int symmetric, gg_graph **out) {
    if (!ctx || !path || !out) return GG_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return set_error(ctx, GG_ERR_IO, std::string("cannot open ") + path);
    uint64_t hdr[8];
    if (fread(hdr, sizeof(hdr), 1, f) != 1) { fclose(f); return set_error(ctx, GG_ERR_IO, "short header"); }
    if ((hdr[0] != 2 && hdr[0] != 3) || hdr[4] != 4 || hdr[5] != 8 || hdr[2] >= 0xFFFFFFFFull) {
        fclose(f);
        return set_error(ctx, GG_ERR_IO, "not a Graptor v2/v3 file with 4-byte VID / 8-byte EID");
    }
    uint32_t n = (uint32_t)hdr[2];
    uint64_t m = hdr[3];
    std::vector<uint64_t> off;
    std::vector<uint32_t> adj;
    try {
        off.resize((size_t)n + 1);
        adj.resize(m);
    } catch (...) {
        fclose(f);
        return set_error(ctx, GG_ERR_OOM, "host allocation");
    }
    bool ok = n == 0 || fread(off.data(), 8, n, f) == n;
    if (ok && hdr[0] == 3) {
        uint64_t last = 0;
        ok = fread(&last, 8, 1, f) == 1 && last == m;
    }
    ok = ok && (m == 0 || fread(adj.data(), 4, m, f) == m);
    fclose(f);
    if (!ok) return set_error(ctx, GG_ERR_IO, "truncated graph file");
    off[n] = m;
    gg_status s = gg_graph_upload(ctx, n, m, off.data(), adj.data(), symmetric, out);
    if (s == GG_ERR_ARG) return set_error(ctx, GG_ERR_IO, "corrupt graph file: " + ctx->err);
    return s;
}

// Ingest with cleaning on the device: sort + dedup drop duplicate edges
// (tools/RmDupEdges.C) and self-loops (tools/RmSelfEdges.C); SYMMETRISE adds
// every edge's reverse first (tools/CvtToUndir.C).
static gg_status graph_from_keys(gg_ctx *ctx, uint32_t n, uint64_t *keys, uint64_t nk, int sym, gg_graph **out) {
    const int lg = ceil_log2(n);
    uint64_t *off = nullptr;
    uint32_t *adj = nullptr;
    uint64_t m = 0;
    gg_status s = build_from_keys(ctx, n, keys, nk, lg, &off, &adj, &m);
    cudaFree(keys);
    if (s != GG_OK) return s;
    return graph_adopt_device_csr(ctx, n, m, off, adj, sym, true, out);  // keys sorted: rows ascending
}

gg_status gg_graph_from_edges(gg_ctx *ctx, uint32_t n, uint64_t nedges, const uint32_t *src, const uint32_t *dst,
                              int flags, gg_graph **out) {
    if (!ctx || !out || (nedges && (!src || !dst)) || n == 0xFFFFFFFFu || (flags & ~3)) return GG_ERR_ARG;
    *out = nullptr;
    const bool dev = flags & GG_INGEST_DEVICE, sym = flags & GG_INGEST_SYMMETRISE;
    if (!dev)
        for (uint64_t i = 0; i < nedges; ++i)
            if (src[i] >= n || dst[i] >= n) return set_error(ctx, GG_ERR_ARG, "gg_graph_from_edges: vertex id out of range");
    GG_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const uint64_t nk = sym ? 2 * nedges : nedges;
    uint64_t *keys = nullptr;
    uint32_t *tmp = nullptr, *bad = nullptr;
    auto fail = [&](cudaError_t e) {
        cudaFree(keys); cudaFree(tmp); cudaFree(bad);
        return cuda_error(ctx, e, "gg_graph_from_edges");
    };
    cudaError_t e;
    if ((e = cudaMalloc(&keys, (nk ? nk : 1) * 8)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&bad, 4)) != cudaSuccess || (e = cudaMemsetAsync(bad, 0, 4, st)) != cudaSuccess) return fail(e);
    const uint32_t *ds = src, *dd = dst;
    if (!dev && nedges) {
        if ((e = cudaMalloc(&tmp, nedges * 8)) != cudaSuccess ||
            (e = cudaMemcpyAsync(tmp, src, nedges * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(tmp + nedges, dst, nedges * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return fail(e);
        ds = tmp;
        dd = tmp + nedges;
    }
    if (nedges) {
        k_edges_to_keys<<<grid_for(ctx, nedges), 256, 0, st>>>(ds, dd, nedges, n, ceil_log2(n), sym, keys, bad);
        ctx->launches++;
    }
    uint32_t hbad = 0;
    if ((e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return fail(e);
    cudaFree(tmp);
    cudaFree(bad);
    if (hbad) {
        cudaFree(keys);
        return set_error(ctx, GG_ERR_ARG, "gg_graph_from_edges: vertex id out of range");
    }
    return graph_from_keys(ctx, n, keys, nk, sym, out);
}

gg_status gg_graph_read_bin_clean(gg_ctx *ctx, const char *path, int flags, gg_graph **out) {
    if (!ctx || !path || !out || (flags & ~GG_INGEST_SYMMETRISE)) return GG_ERR_ARG;
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return set_error(ctx, GG_ERR_IO, std::string("cannot open ") + path);
    uint64_t hdr[8];
    if (fread(hdr, sizeof(hdr), 1, f) != 1) { fclose(f); return set_error(ctx, GG_ERR_IO, "short header"); }
    if ((hdr[0] != 2 && hdr[0] != 3) || hdr[4] != 4 || hdr[5] != 8 || hdr[2] >= 0xFFFFFFFFull) {
        fclose(f);
        return set_error(ctx, GG_ERR_IO, "not a Graptor v2/v3 file with 4-byte VID / 8-byte EID");
    }
    const uint32_t n = (uint32_t)hdr[2];
    const uint64_t m = hdr[3];
    std::vector<uint64_t> off;
    std::vector<uint32_t> adj;
    try {
        off.resize((size_t)n + 1);
        adj.resize(m);
    } catch (...) {
        fclose(f);
        return set_error(ctx, GG_ERR_OOM, "host allocation");
    }
    bool ok = n == 0 || fread(off.data(), 8, n, f) == n;
    if (ok && hdr[0] == 3) {
        uint64_t last = 0;
        ok = fread(&last, 8, 1, f) == 1 && last == m;
    }
    ok = ok && (m == 0 || fread(adj.data(), 4, m, f) == m);
    fclose(f);
    if (!ok) return set_error(ctx, GG_ERR_IO, "truncated graph file");
    off[n] = m;
    if (off[0] != 0) return set_error(ctx, GG_ERR_IO, "corrupt graph file: first offset");
    for (uint32_t v = 0; v < n; ++v)
        if (off[v] > off[v + 1]) return set_error(ctx, GG_ERR_IO, "corrupt graph file: offsets not monotone");
    for (uint64_t e = 0; e < m; ++e)
        if (adj[e] >= n) return set_error(ctx, GG_ERR_IO, "corrupt graph file: vertex id out of range");
    GG_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool sym = flags & GG_INGEST_SYMMETRISE;
    const uint64_t nk = sym ? 2 * m : m;
    uint64_t *doff = nullptr, *keys = nullptr;
    uint32_t *dadj = nullptr;
    auto fail = [&](cudaError_t e) {
        cudaFree(doff); cudaFree(dadj); cudaFree(keys);
        return cuda_error(ctx, e, "gg_graph_read_bin_clean");
    };
    cudaError_t e;
    if ((e = cudaMalloc(&doff, ((size_t)n + 1) * 8)) != cudaSuccess || (e = cudaMalloc(&dadj, (m ? m : 1) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&keys, (nk ? nk : 1) * 8)) != cudaSuccess ||
        (e = cudaMemcpyAsync(doff, off.data(), ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (m && (e = cudaMemcpyAsync(dadj, adj.data(), m * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess))
        return fail(e);
    if (m) {
        k_csr_to_keys<<<grid_for(ctx, (uint64_t)n * 32), 256, 0, st>>>(doff, dadj, n, ceil_log2(n), sym, m, keys);
        ctx->launches++;
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
    cudaFree(doff);
    cudaFree(dadj);
    return graph_from_keys(ctx, n, keys, nk, sym, out);
}

gg_status gg_graph_write_bin(gg_graph *g, const char *path) {
    if (!g || !path) return GG_ERR_ARG;
    std::vector<uint64_t> off((size_t)g->n + 1);
    std::vector<uint32_t> adj(g->m);
    GG_CHECK(gg_graph_download(g, off.data(), adj.data()));
    FILE *f = fopen(path, "wb");
    if (!f) return set_error(g->ctx, GG_ERR_IO, std::string("cannot create ") + path);
    uint64_t hdr[8] = {2, 1, g->n, g->m, 4, 8, 0, 0};
    bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
              (g->n == 0 || fwrite(off.data(), 8, g->n, f) == g->n) &&
              (g->m == 0 || fwrite(adj.data(), 4, g->m, f) == g->m);
    ok = (fclose(f) == 0) && ok;
    return ok ? GG_OK : set_error(g->ctx, GG_ERR_IO, "write failed");
}

gg_status gg_graph_generate(gg_ctx *ctx, const gg_gen_params *p, gg_graph **out) {
    if (!ctx || !p || !out) return GG_ERR_ARG;
    *out = nullptr;
    GG_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    uint32_t n = 0;
    uint64_t nk = 0;
    int lg = 1;
    uint64_t *keys = nullptr;
    int symmetric = p->symmetric ? 1 : 0;
    if (p->kind == GG_GEN_RMAT) {
        if (p->scale < 1 || p->scale > 31) return set_error(ctx, GG_ERR_ARG, "rmat scale out of range");
        double a = p->a, b = p->b, c = p->c;
        if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return set_error(ctx, GG_ERR_ARG, "rmat probabilities");
        n = 1u << p->scale;
        lg = p->scale;
        nk = symmetric ? 2 * p->nedges : p->nedges;
        GG_CUDA(ctx, cudaMalloc(&keys, (nk ? nk : 1) * 8));
        if (p->nedges) {
            k_gen_rmat<<<grid_for(ctx, p->nedges), 256, 0, st>>>(
                keys, p->nedges, p->scale, lg, stream_base(p->seed, 1), prob_u32(a), prob_u32(a + b),
                prob_u32(a + b + c), symmetric);
            ctx->launches++;
        }
    } else if (p->kind == GG_GEN_ER) {
        if (p->n == 0 || p->avgdeg < 0) return set_error(ctx, GG_ERR_ARG, "er parameters");
        n = p->n;
        lg = ceil_log2(n);
        uint64_t M = (uint64_t)((double)n * p->avgdeg / (symmetric ? 2.0 : 1.0) + 0.5);
        nk = symmetric ? 2 * M : M;
        GG_CUDA(ctx, cudaMalloc(&keys, (nk ? nk : 1) * 8));
        if (M) {
            k_gen_er<<<grid_for(ctx, M), 256, 0, st>>>(keys, M, n, lg, stream_base(p->seed, 2),
                                                      stream_base(p->seed, 3), p->bp, symmetric);
            ctx->launches++;
        }
    } else if (p->kind == GG_GEN_GRID) {
        uint64_t n64 = (uint64_t)p->rows * p->cols;
        if (n64 == 0 || n64 >= 0xFFFFFFFFull) return set_error(ctx, GG_ERR_ARG, "grid size");
        n = (uint32_t)n64;
        lg = ceil_log2(n);
        symmetric = 1;
        nk = 4 * n64;
        GG_CUDA(ctx, cudaMalloc(&keys, nk * 8));
        k_gen_grid<<<grid_for(ctx, n64), 256, 0, st>>>(keys, p->rows, p->cols, lg, stream_base(p->seed, 4), p->bp);
        ctx->launches++;
    } else {
        return set_error(ctx, GG_ERR_ARG, "unknown generator kind");
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { cudaFree(keys); return cuda_error(ctx, e, "generator launch"); }
    gg_graph *g = new (std::nothrow) gg_graph;
    if (!g) { cudaFree(keys); return GG_ERR_OOM; }
    g->ctx = ctx;
    g->n = n;
    g->symmetric = symmetric;
    g->rows_sorted = true;  // built from sorted (row, col) keys
    gg_status s = build_from_keys(ctx, n, keys, nk, lg, &g->off, &g->adj, &g->m);
    cudaFree(keys);
    if (s != GG_OK) { graph_free(g); return s; }
    s = graph_finish(g);
    if (s != GG_OK) { graph_free(g); return s; }
    *out = g;
    return GG_OK;
}

gg_status gg_graph_info(gg_graph *g, uint32_t *n, uint64_t *m, int *symmetric) {
    if (!g) return GG_ERR_ARG;
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (symmetric) *symmetric = g->symmetric;
    return GG_OK;
}

gg_status gg_graph_download(gg_graph *g, uint64_t *off, uint32_t *adj) {
    if (!g) return GG_ERR_ARG;
    GG_CUDA(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    if (off) GG_CUDA(g->ctx, cudaMemcpy(off, g->off, ((size_t)g->n + 1) * 8, cudaMemcpyDeviceToHost));
    if (adj && g->m) GG_CUDA(g->ctx, cudaMemcpy(adj, g->adj, g->m * 4, cudaMemcpyDeviceToHost));
    return GG_OK;
}

gg_status gg_graph_device_ptrs(gg_graph *g, const uint64_t **off, const uint32_t **adj,
                               const uint64_t **in_off, const uint32_t **in_adj) {
    if (!g) return GG_ERR_ARG;
    if (off) *off = g->off;
    if (adj) *adj = g->adj;
    if (in_off) *in_off = g->in_off;
    if (in_adj) *in_adj = g->in_adj;
    return GG_OK;
}

gg_status gg_graph_max_degree_vertex(gg_graph *g, uint32_t *v, uint32_t *deg) {
    if (!g) return GG_ERR_ARG;
    if (v) *v = g->maxdeg_v;
    if (deg) *deg = g->maxdeg;
    return GG_OK;
}

gg_status gg_graph_destroy(gg_graph *g) {
    if (!g) return GG_ERR_ARG;
    cudaStreamSynchronize(g->ctx->stream);
    graph_free(g);
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Properties
// ---------------------------------------------------------------------------
gg_status gg_prop_create(gg_graph *g, gg_dtype t, gg_prop **out) {
    if (!g || !out) return GG_ERR_ARG;
    size_t esz = dtype_size(t);
    if (!esz) return set_error(g->ctx, GG_ERR_ARG, "bad dtype");
    gg_prop *p = new (std::nothrow) gg_prop;
    if (!p) return GG_ERR_OOM;
    p->g = g;
    p->t = t;
    p->esz = esz;
    cudaError_t e = cudaMalloc(&p->d, ((size_t)g->n + 1) * esz);
    if (e != cudaSuccess) { delete p; return cuda_error(g->ctx, e, "gg_prop_create"); }
    *out = p;
    return GG_OK;
}

gg_status gg_prop_create_managed(gg_graph *g, gg_dtype t, gg_prop **out) {
    if (!g || !out) return GG_ERR_ARG;
    size_t esz = dtype_size(t);
    if (!esz) return set_error(g->ctx, GG_ERR_ARG, "bad dtype");
    gg_prop *p = new (std::nothrow) gg_prop;
    if (!p) return GG_ERR_OOM;
    p->g = g;
    p->t = t;
    p->esz = esz;
    // host code writes the initial values in place; kernels then migrate the pages
    cudaError_t e = cudaMallocManaged(&p->d, ((size_t)g->n + 1) * esz, cudaMemAttachGlobal);
    if (e != cudaSuccess) { delete p; return cuda_error(g->ctx, e, "gg_prop_create_managed"); }
    p->managed = true;
    *out = p;
    return GG_OK;
}

gg_status gg_prop_prefetch(gg_prop *p, int to_device) {
    if (!p) return GG_ERR_ARG;
    if (!p->managed) return GG_OK;
    gg_ctx *ctx = p->g->ctx;
    const size_t bytes = ((size_t)p->g->n + 1) * p->esz;
    if (to_device == 2) GG_CUDA(ctx, cudaMemAdvise(p->d, bytes, cudaMemAdviseSetReadMostly, ctx->device));
    GG_CUDA(ctx, cudaMemPrefetchAsync(p->d, bytes, to_device ? ctx->device : cudaCpuDeviceId, ctx->stream));
    return GG_OK;
}

gg_status gg_prop_fill(gg_prop *p, const void *value) {
    if (!p || !value) return GG_ERR_ARG;
    uint64_t v = 0;
    memcpy(&v, value, p->esz);
    gg_ctx *ctx = p->g->ctx;
    k_fill_bytes<<<grid_for(ctx, p->g->n + 1), 256, 0, ctx->stream>>>(p->d, (uint64_t)p->g->n, v, (int)p->esz);
    GG_LAUNCHED(ctx);
    return GG_OK;
}

gg_status gg_prop_set(gg_prop *p, uint32_t v, const void *value) {
    if (!p || !value || v >= p->g->n) return GG_ERR_ARG;
    gg_ctx *ctx = p->g->ctx;
    uint64_t val = 0;
    memcpy(&val, value, p->esz);
    k_fill_bytes<<<1, 1, 0, ctx->stream>>>((char *)p->d + (size_t)v * p->esz, 1, val, (int)p->esz);
    GG_LAUNCHED(ctx);
    return GG_OK;
}

gg_status gg_prop_get(gg_prop *p, uint32_t v, void *value) {
    if (!p || !value || v >= p->g->n) return GG_ERR_ARG;
    gg_ctx *ctx = p->g->ctx;
    GG_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, (char *)p->d + (size_t)v * p->esz, p->esz,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(value, ctx->h_pinned, p->esz);
    return GG_OK;
}

gg_status gg_prop_download(gg_prop *p, void *host) {
    if (!p || !host) return GG_ERR_ARG;
    gg_ctx *ctx = p->g->ctx;
    GG_CUDA(ctx, cudaMemcpyAsync(host, p->d, (size_t)p->g->n * p->esz, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GG_OK;
}

gg_status gg_prop_upload(gg_prop *p, const void *host) {
    if (!p || !host) return GG_ERR_ARG;
    gg_ctx *ctx = p->g->ctx;
    GG_CUDA(ctx, cudaMemcpyAsync(p->d, host, (size_t)p->g->n * p->esz, cudaMemcpyHostToDevice, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GG_OK;
}

gg_status gg_prop_device_ptr(gg_prop *p, void **dptr) {
    if (!p || !dptr) return GG_ERR_ARG;
    *dptr = p->d;
    return GG_OK;
}

gg_status gg_prop_destroy(gg_prop *p) {
    if (!p) return GG_ERR_ARG;
    cudaStreamSynchronize(p->g->ctx->stream);
    cudaFree(p->d);
    delete p;
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Frontiers
// ---------------------------------------------------------------------------
gg_status gg_frontier_create(gg_graph *g, gg_frontier **out) {
    if (!g || !out) return GG_ERR_ARG;
    gg_frontier *f = new (std::nothrow) gg_frontier;
    if (!f) return GG_ERR_OOM;
    f->g = g;
    cudaError_t e = cudaSuccess;
    if (!g->pool_cnt.empty()) {
        f->d_cnt = g->pool_cnt.back();
        g->pool_cnt.pop_back();
    } else {
        e = cudaMalloc(&f->d_cnt, FC_WORDS * sizeof(uint64_t));
    }
    if (e != cudaSuccess) { delete f; return cuda_error(g->ctx, e, "gg_frontier_create"); }
    e = cudaMemsetAsync(f->d_cnt, 0, FC_WORDS * sizeof(uint64_t), g->ctx->stream);
    if (e != cudaSuccess) { cudaFree(f->d_cnt); delete f; return cuda_error(g->ctx, e, "memset"); }
    f->host_valid = true;
    *out = f;
    return GG_OK;
}

gg_status gg_frontier_destroy(gg_frontier *f) {
    if (!f) return GG_ERR_ARG;
    gg_graph *g = f->g;
    // buffers go back to the graph's pools (stream-ordered reuse)
    if (f->bins[0]) g->pool_bins.push_back(f->bins[0]);
    if (f->bitmap) g->pool_bitmaps.push_back(f->bitmap);
    if (f->d_cnt) g->pool_cnt.push_back(f->d_cnt);
    delete f;
    return GG_OK;
}

gg_status gg_frontier_clear(gg_frontier *f) {
    if (!f) return GG_ERR_ARG;
    GG_CHECK(frontier_reset_counts(f));
    f->all = false;
    f->has_list = true;  // an empty list
    f->has_bitmap = false;
    memset(f->h_cnt, 0, sizeof(f->h_cnt));
    f->host_valid = true;
    return GG_OK;
}

gg_status gg_frontier_set_single(gg_frontier *f, uint32_t v) {
    if (!f || v >= f->g->n) return GG_ERR_ARG;
    GG_CHECK(frontier_alloc_bins(f));
    gg_ctx *ctx = f->g->ctx;
    const Tuning &t = tuning();
    k_front_single<<<1, 1, 0, ctx->stream>>>(v, f->g->off, f->bins[0], f->bins[1], f->bins[2], f->d_cnt,
                                             t.bin_small_max, t.bin_medium_max);
    GG_LAUNCHED(ctx);
    f->all = false;
    f->has_list = true;
    f->has_bitmap = false;
    f->host_valid = false;
    return GG_OK;
}

gg_status gg_frontier_set_all(gg_frontier *f) {
    if (!f) return GG_ERR_ARG;
    gg_ctx *ctx = f->g->ctx;
    k_front_set_counts<<<1, 1, 0, ctx->stream>>>(f->d_cnt, f->g->n, f->g->m);
    GG_LAUNCHED(ctx);
    f->all = true;
    f->has_list = false;
    f->has_bitmap = false;
    memset(f->h_cnt, 0, sizeof(f->h_cnt));
    f->h_cnt[FC_NACTV] = f->g->n;
    f->h_cnt[FC_NACTE] = f->g->m;
    f->host_valid = true;
    return GG_OK;
}

gg_status gg_frontier_set_list(gg_frontier *f, const uint32_t *host_list, uint64_t k) {
    if (!f || (k && !host_list) || k > f->g->n) return GG_ERR_ARG;
    gg_graph *g = f->g;
    gg_ctx *ctx = g->ctx;
    for (uint64_t i = 0; i < k; ++i)
        if (host_list[i] >= g->n) return set_error(ctx, GG_ERR_ARG, "frontier vertex out of range");
    // through a bitmap: de-duplicates and bins in one pass
    GG_CHECK(frontier_alloc_bitmap(f));
    GG_CHECK(frontier_alloc_bins(f));
    size_t words = ((size_t)g->n + 31) / 32;
    std::vector<uint32_t> bm(words, 0);
    for (uint64_t i = 0; i < k; ++i) bm[host_list[i] >> 5] |= 1u << (host_list[i] & 31);
    GG_CUDA(ctx, cudaMemcpyAsync(f->bitmap, bm.data(), words * 4, cudaMemcpyHostToDevice, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    f->all = false;
    f->has_bitmap = true;
    f->has_list = false;
    GG_CHECK(frontier_ensure_list(f));
    return GG_OK;
}

gg_status gg_frontier_counts(gg_frontier *f, uint64_t *nactv, uint64_t *nacte) {
    if (!f) return GG_ERR_ARG;
    GG_CHECK(frontier_fetch_counts(f));
    if (nactv) *nactv = f->h_cnt[FC_NACTV];
    if (nacte) *nacte = f->h_cnt[FC_NACTE];
    return GG_OK;
}

gg_status gg_frontier_download(gg_frontier *f, uint32_t *host_list, uint64_t cap, uint64_t *k) {
    if (!f || !k) return GG_ERR_ARG;
    gg_graph *g = f->g;
    gg_ctx *ctx = g->ctx;
    GG_CHECK(frontier_fetch_counts(f));
    uint64_t nv = f->h_cnt[FC_NACTV];
    *k = nv;
    if (!host_list) return GG_OK;
    if (cap < nv) return set_error(ctx, GG_ERR_ARG, "gg_frontier_download: capacity too small");
    if (f->all) {
        for (uint32_t v = 0; v < g->n; ++v) host_list[v] = v;
        return GG_OK;
    }
    GG_CHECK(frontier_ensure_bitmap(f));
    size_t words = ((size_t)g->n + 31) / 32;
    std::vector<uint32_t> bm(words);
    GG_CUDA(ctx, cudaMemcpyAsync(bm.data(), f->bitmap, words * 4, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    uint64_t j = 0;
    for (size_t w = 0; w < words; ++w)
        for (uint32_t b = bm[w]; b; b &= b - 1)
            if (j < cap) host_list[j++] = (uint32_t)(w * 32 + __builtin_ctz(b));
    *k = j;
    return GG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Internal frontier helpers
// ---------------------------------------------------------------------------
namespace gg {

// Frontier buffers come from per-graph pools: analytics create and delete a
// frontier every iteration (Graptor's frontier::del pattern), and all use of
// a buffer is ordered on the context's stream, so a released buffer can be
// handed to the next frontier without a cudaMalloc / cudaFree pair.
gg_status frontier_alloc_bins(gg_frontier *f) {
    if (f->bins[0]) return GG_OK;
    gg_graph *g = f->g;
    const size_t cap = (size_t)g->n + 1;
    uint32_t *blk = nullptr;
    if (!g->pool_bins.empty()) {
        blk = g->pool_bins.back();
        g->pool_bins.pop_back();
    } else {
        GG_CUDA(g->ctx, cudaMalloc(&blk, NBINS * cap * 4));
    }
    for (int b = 0; b < NBINS; ++b) f->bins[b] = blk + b * cap;
    return GG_OK;
}

gg_status frontier_alloc_bitmap(gg_frontier *f) {
    if (f->bitmap) return GG_OK;
    gg_graph *g = f->g;
    if (!g->pool_bitmaps.empty()) {
        f->bitmap = g->pool_bitmaps.back();
        g->pool_bitmaps.pop_back();
        return GG_OK;
    }
    size_t words = ((size_t)g->n + 31) / 32 + 1;
    GG_CUDA(g->ctx, cudaMalloc(&f->bitmap, words * 4));
    return GG_OK;
}

gg_status frontier_reset_counts(gg_frontier *f) {
    GG_CUDA(f->g->ctx, cudaMemsetAsync(f->d_cnt, 0, FC_WORDS * sizeof(uint64_t), f->g->ctx->stream));
    f->host_valid = false;
    return GG_OK;
}

gg_status frontier_fetch_counts(gg_frontier *f) {
    if (f->host_valid) return GG_OK;
    gg_ctx *ctx = f->g->ctx;
    GG_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, f->d_cnt, FC_WORDS * 8, cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    memcpy(f->h_cnt, ctx->h_pinned, FC_WORDS * 8);
    f->host_valid = true;
    return GG_OK;
}

gg_status frontier_ensure_bitmap(gg_frontier *f) {
    if (f->has_bitmap || f->all) return GG_OK;
    gg_graph *g = f->g;
    gg_ctx *ctx = g->ctx;
    GG_CHECK(frontier_alloc_bitmap(f));
    size_t words = ((size_t)g->n + 31) / 32;
    GG_CUDA(ctx, cudaMemsetAsync(f->bitmap, 0, words * 4, ctx->stream));
    if (f->has_list) {
        uint64_t tot = f->host_valid ? f->h_cnt[FC_NACTV] : (uint64_t)g->n;
        if (tot) {
            k_list_to_bitmap<<<grid_for(ctx, tot), 256, 0, ctx->stream>>>(f->bins[0], f->bins[1], f->bins[2],
                                                                           f->d_cnt, f->bitmap);
            GG_LAUNCHED(ctx);
        }
    }
    f->has_bitmap = true;
    return GG_OK;
}

gg_status frontier_ensure_list(gg_frontier *f) {
    if (f->has_list) return GG_OK;
    gg_graph *g = f->g;
    gg_ctx *ctx = g->ctx;
    GG_CHECK(frontier_alloc_bins(f));
    GG_CHECK(frontier_reset_counts(f));
    const Tuning &t = tuning();
    uint32_t nwords = (g->n + 31) / 32;
    k_bitmap_to_list<<<grid_for(ctx, (uint64_t)nwords * 32), 256, 0, ctx->stream>>>(
        f->all ? nullptr : f->bitmap, g->n, g->off, f->bins[0], f->bins[1], f->bins[2],
        (unsigned long long *)f->d_cnt, t.bin_small_max, t.bin_medium_max);
    GG_LAUNCHED(ctx);
    f->has_list = true;
    if (f->all) {
        f->all = false;
        f->has_bitmap = false;
    }
    return GG_OK;
}

}  // namespace gg
