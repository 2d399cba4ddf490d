// gg_internal.cuh -- internal types and device helpers of libgg.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "gg.h"
#include "gg_tune.h"
#include "gg_select.h"

namespace gg {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
gg_status set_error(gg_ctx *ctx, gg_status s, const std::string &msg);
gg_status cuda_error(gg_ctx *ctx, cudaError_t e, const char *what);

#define GG_CUDA(ctx, expr)                                              \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::gg::cuda_error((ctx), _e, #expr); \
    } while (0)

#define GG_CHECK(expr)                          \
    do {                                        \
        gg_status _s = (expr);                  \
        if (_s != GG_OK) return _s;             \
    } while (0)

// After a launch: count it and surface launch-configuration errors.
#define GG_LAUNCHED(ctx)                                                   \
    do {                                                                   \
        (ctx)->launches++;                                                 \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) return ::gg::cuda_error((ctx), _e, "kernel launch"); \
    } while (0)

// Device error word bits (set by kernels with bounds checks / bounded waits).
enum : uint32_t {
    DEV_ERR_BOUNDS = 1u,
    DEV_ERR_TIMEOUT = 2u,
    DEV_ERR_OVERFLOW = 4u,
};

}  // namespace gg

// ---------------------------------------------------------------------------
// Handles
// ---------------------------------------------------------------------------
struct gg_ctx {
    int device = 0;
    int sm_count = 148;
    size_t l2_bytes = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    uint64_t launches = 0;
    uint32_t *d_err = nullptr;  // device error word
    uint64_t *h_pinned = nullptr;  // small pinned staging buffer (counts)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;    // whole-run timing
    cudaEvent_t evk0 = nullptr, evk1 = nullptr;  // traversal-kernel timing
    bool time_kernels = false;                   // record evk0/evk1 around the next traversal kernel
};

// Frontier counters live on the device in this layout.
enum {
    FC_NACTV = 0,   // active vertices
    FC_NACTE = 1,   // sum of out-degrees of active vertices
    FC_BIN0 = 2,    // list bin sizes (small / medium / large out-degree)
    FC_BIN1 = 3,
    FC_BIN2 = 4,
    FC_SCANNED = 5, // edges examined by the step that produced this frontier
    FC_WORDS = 8
};

enum { NBINS = 3 };

struct gg_graph;

// In-rows of the CSC longer than `T` edges ("heavy" rows: R-MAT hubs, all
// at low ids) are cut into chunks of `CH` edges so that no warp walks a hub
// row alone.  first[h]..first[h+1] are the chunks of heavy vertex v[h].
struct HeavyRows {
    uint32_t *v = nullptr;      // heavy vertices, ascending
    uint64_t *first = nullptr;  // [nheavy + 1] chunk prefix
    uint32_t *crow = nullptr;   // [nchunks] heavy index of each chunk
    // Per 32-vertex word work estimates (inclusive prefix over words) used to
    // give every warp a contiguous range of equal estimated work:
    //   light_prefix: PageRank light-row gather, light in-edges + 4 per vertex
    //   pull_prefix : dense pull, min(in-degree, 16) + 2 per vertex
    uint64_t *light_prefix = nullptr;
    uint64_t *pull_prefix = nullptr;
    uint32_t nheavy = 0;
    uint64_t nchunks = 0;
    uint32_t T = 0, CH = 0;
};

// Pull candidate lists of a driver run: destinations that still pass the
// dst filter (double-buffered, device counts).
struct CandLists {
    uint32_t *list[2] = {nullptr, nullptr};
    uint64_t *cnt = nullptr;  // [2] device counters
    int cur = 0;
    bool valid = false;       // list[cur] holds the candidates
    uint64_t host_n = 0;      // count of list[cur] if known on the host, else UINT64_MAX
};

struct gg_frontier {
    gg_graph *g = nullptr;
    bool all = false;         // every vertex active (frontier::all_true)
    bool has_list = false;    // bins valid
    bool has_bitmap = false;  // bitmap valid
    uint32_t *bins[NBINS] = {nullptr, nullptr, nullptr};  // each n entries
    uint32_t *bitmap = nullptr;                            // ceil(n/32) words
    uint64_t *d_cnt = nullptr;                             // FC_WORDS counters
    // host copy of counters (valid when host_valid)
    uint64_t h_cnt[FC_WORDS] = {0};
    bool host_valid = false;
};

struct gg_graph {
    gg_ctx *ctx = nullptr;
    uint32_t n = 0;
    uint64_t m = 0;
    int symmetric = 0;
    bool rows_sorted = false;    // every CSR row ascending (device-built graphs; checked on upload)
    uint64_t *off = nullptr;     // CSR offsets [n+1]
    uint32_t *adj = nullptr;     // CSR targets [m]
    uint64_t *in_off = nullptr;  // CSC (== off when symmetric)
    uint32_t *in_adj = nullptr;
    uint32_t maxdeg_v = 0, maxdeg = 0;
    // scratch owned by the graph (grown on demand)
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    gg_frontier *tmp_front[2] = {nullptr, nullptr};
    uint64_t *aux_cnt = nullptr;  // counters of steps that record no frontier
    HeavyRows heavy;              // chunked long rows of the CSC (pull / gather)
    // per vertex {first two in-neighbours (CSC row order; 0xFFFFFFFF past the
    // row's end), in-degree, third in-neighbour}: most dense-pull rows find
    // their parent there
    uint4 *first_in = nullptr;
    // per vertex {first in-neighbour, in-degree} (8 bytes; pull_first 4),
    // built on first use
    uint2 *first1 = nullptr;
    // gg_bfs_level_host_async: two level buffers used in turn, the stream
    // their host copies run on, and an event per buffer marking its copy done
    gg_prop *async_level[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_done[2] = {nullptr, nullptr};
    bool copy_pending[2] = {false, false};
    int async_next = 0;
    gg_prop *tmp_prop[4] = {nullptr, nullptr, nullptr, nullptr};  // cached run temporaries
    uint32_t *nonisolated = nullptr;    // vertices with in-edges, ascending
    uint64_t *nonisolated_n = nullptr;  // its length (device)
    // gg_kcore: the two alive lists (vertices not yet peeled; n entries
    // each) and their counters {count A, count B, smallest count left}
    uint32_t *kc_alive[2] = {nullptr, nullptr};
    unsigned long long *kc_cnt = nullptr;
    CandLists cand;               // pull candidate lists (driver runs)
    bool cand_active = false;     // a driver run uses them for its pull steps
    // released frontier buffers, reused in stream order
    std::vector<uint32_t *> pool_bins, pool_bitmaps;
    std::vector<uint64_t *> pool_cnt;
    void *pstate = nullptr;       // device state block of persistent traversals
    void *pstate2 = nullptr;      // a second one (the CC run of a BFS + CC batch)
    void *gbfs = nullptr;         // graph-driven BFS: instantiated CUDA graph + control block
    uint32_t *wq = nullptr;       // work queue of fused (asynchronous) pushes
    size_t wq_cap = 0;
    float gini = -1.0f;           // degree Gini coefficient (selector feature), <0: unknown
    // learned variant selector (GG_THRESH_LEARNED): the graph's own copy of
    // the attached selector's weights (float on the host, bfloat16 on the device)
    bool sel_on = false;
    float *sel_h = nullptr;
    void *sel_d = nullptr;
    int force_iter = -1, force_variant = -1;  // timing collection: one forced choice
    struct ForceRecord {          // what the last device-driven run saw at force_iter
        bool seen = false;
        double iter_ms = 0, rest_ms = 0;  // that iteration; from its start to the run's end
        double nactv = 0, nacte = 0, reached = 0;
    } force_rec;
};

struct gg_prop {
    gg_graph *g = nullptr;
    gg_dtype t = GG_I32;
    size_t esz = 4;
    void *d = nullptr;
    bool managed = false;  // gg_prop_create_managed
};

namespace gg {

size_t dtype_size(gg_dtype t);
gg_status graph_scratch(gg_graph *g, size_t bytes, void **p);
gg_status frontier_alloc_bins(gg_frontier *f);
gg_status frontier_alloc_bitmap(gg_frontier *f);
gg_status frontier_fetch_counts(gg_frontier *f);     // device -> host (syncs)
gg_status frontier_ensure_bitmap(gg_frontier *f);    // from list
gg_status frontier_ensure_list(gg_frontier *f);      // from bitmap / all
gg_status frontier_reset_counts(gg_frontier *f);     // async zero of d_cnt
uint32_t bin_of_degree(uint64_t deg);
gg_status build_heavy_rows(gg_graph *g);
// A BFS-levels run handed over to the device-driven traversal part way:
// iter0 iterations done, the frontier in the graph's scratch frontier `cur`
// (its bitmap always set, its binned list when has_list), the other scratch
// frontier empty, reached_v / reached_e the counts so far.
struct PersistResume {
    int iter0;
    int cur;
    int has_list;
    unsigned long long reached_v, reached_e;
};
gg_status persistent_traverse(gg_graph *g, const gg_emap_desc &d, int level_k, bool start_all, uint32_t root,
                              const gg_run_opts &opt, gg_run_stats *stats, int *iters_out,
                              int force_iter = -1, int force_variant = -1,
                              const uint32_t *d_roots = nullptr, uint32_t nroots = 0,
                              const PersistResume *resume = nullptr);
gg_status enqueue_bfs_start(gg_graph *g, gg_prop *level, gg_prop *prev, const uint32_t *d_roots, uint32_t k);
gg_status enqueue_cc_start(gg_graph *g, gg_prop *label, gg_prop *prev);
gg_status run_tmp_prop(gg_graph *g, int slot, gg_dtype t, gg_prop **out);
gg_status graph_adopt_device_csr(gg_ctx *ctx, uint32_t n, uint64_t m, uint64_t *off, uint32_t *adj, int symmetric,
                                 bool rows_sorted,
                                 gg_graph **out);
gg_status graph_gini(gg_graph *g, float *out);
// builds g->first1 (the 8-byte pull records) if it is not there yet
gg_status graph_ensure_first1(gg_graph *g);
void graph_bfs_free(gg_graph *g);
void selector_features(float *x, double nactv, double nacte, double unreached, int iter, double n, double m,
                       float gini);

// Degree-bin thresholds of the sparse push (tunable by the autotuner).
struct Tuning {
    uint32_t bin_small_max = 32;    // deg <= this: thread per vertex
    uint32_t bin_medium_max = 2048; // deg <= this: warp per vertex, else CTA
    int pull_k = 8;                 // per-lane edges before warp cooperation (pull)
    int pull_split = 1;             // graph-driven BFS pulls in two passes (first two in-edges, then the rest)
    int graph_flat = 1;             // graph-driven BFS: the loop body as one chain of kernels, no step conditionals
    int graph_pdl = 0;              // graph-driven BFS (flat): the chain's kernels joined by programmatic edges
    int graph_unroll = 2;           // graph-driven BFS (flat): copies of the chain per loop iteration (1-4)
    int push_k = 8;
    int block = 256;
    int blocks_per_sm = 8;
    uint32_t heavy_deg = 256;    // CSC rows longer than this are chunked
    uint32_t heavy_chunk = 1024; // edges per chunk
    uint32_t large_chunk = 512;  // push: edges per chunk of a large-bin row
    int pr_stream = 0;           // PageRank light rows: warp-streamed segmented gather
    // PageRank kernels' grid cap in CTAs per SM (measured at R-MAT 25: 16
    // against 8 cuts an FP32 iteration 6.63 -> 6.17 ms, BF16 4.07 -> 4.01)
    int pr_blocks_per_sm = 16;
    // analytics run as one device-driven cooperative launch: bit 0 BFS levels,
    // bit 1 BFS parents, bit 2 CC (the persistent grid reads values written
    // during the launch through L2, which costs the big dense phases more
    // than the per-iteration host round trips it saves on R-MAT BFS)
    int persistent = 4;
    // analytics run as one CUDA graph whose conditional nodes take each
    // iteration's push/pull decision on the device (host-driven kernels, no
    // per-iteration host round trip): bit 0 BFS levels
    int graph = 1;
    // graph-driven BFS levels: a run still going after this many iterations
    // (a high-diameter graph: many small frontiers, where the graph's
    // per-step node launches cost more than a grid barrier) continues in the
    // device-driven traversal; 0 = never
    int graph_handoff = 32;
    // CTAs of the device-driven launch that continues a handed-over run
    // (0 = all that fit; at most that many): its frontiers are small, and
    // fewer CTAs make each grid barrier cheaper
    int handoff_ctas = 148;
    // device-driven BFS levels: small frontiers (at most 8192 vertices and
    // 65536 edges) run in one thread-block cluster with the frontier in
    // shared memory
    int small_frontier = 1;
    // sparse push steps run fused (asynchronous multi-hop, as CCv with
    // api::fusion) in device-driven runs: bit 2 CC.  Off by default: on
    // B200 the shared work queue (three contended counters per vertex, and
    // vertices revisited as ever smaller labels arrive) lost to both the
    // level-synchronous steps and hooking on every graph measured.
    int fusion = 0;
    uint32_t fusion_queue = 0;  // queue entries (0: 2n + 65536)
    // device-driven CC of a symmetric graph: after the first step, CCv's
    // road-network test (fewer than n/10 zero labels) and, where it holds,
    // min-id hooking for the rest of the run (1); 2: where it fails, hooking
    // too, of the vertices label 0 has not reached (vertex 0's component is
    // done).  Measured on R-MAT 24: 1.04 ms with 2 against 0.69 ms with label
    // propagation after the first step, so 1 stays the default
    int cc_hook = 1;
    // dense pull: each row's first in-neighbours read from a per-vertex
    // record (coalesced with the row's offsets) before the row itself.
    // 1: the 16-byte record's first two, offsets loaded with the record;
    // 2: the same two, the record's degree standing in for the offsets, which
    // are loaded only for rows the two edges do not settle; 3: as 2 with the
    // record's three in-neighbours; 4: an 8-byte record {first in-neighbour,
    // degree}, offsets as in 2; 0: rows only.  3, the default, measured
    // fastest on R-MAT 24 BFS (dense pull 14 % under mode 1)
    int pull_first = 3;
    // graph-driven BFS pull: KiB of the frontier bitmap's first words (the
    // lowest vertex ids) copied into each CTA's shared memory by a bulk copy
    // (TMA) before the pull; probes of those ids read shared memory; 0: none
    int pull_stage = 0;
    // graph-driven BFS pull after a pull: its candidates are the previous
    // pull's unsettled rows, so their levels are known (unvisited) and not
    // loaded
    int pull_fresh = 1;
    // graph-driven BFS pull kernels compiled for this many resident CTAs per
    // SM (4 to 8: more CTAs, fewer registers per thread)
    int pull_ctas = 6;
    int push_ctas = 6;  // the same for the graph-driven BFS push kernel
    unsigned long long barrier_timeout_ns = 5000000000ull;  // grid-barrier wait limit
};
Tuning &tuning();

// Grid of `block`-thread CTAs for a grid-stride kernel: resident CTAs per SM
// (occupancy query, cached per kernel) x SM count, capped by the work.
int resident_ctas(const void *kernel, int block);
unsigned occ_grid(gg_ctx *ctx, const void *kernel, int block, uint64_t work_threads);

}  // namespace gg

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
namespace gg {
namespace dev {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Contiguous word range [lo, hi) of warp `wid` of `nw` warps such that every
// warp gets an equal share of the work estimate.  pre[w] is the inclusive
// prefix of the per-word costs (nwords entries); word w covers cost units
// [pre[w-1], pre[w]) and belongs to the warp whose share [t0, t1) holds its
// first unit.  Binary searches only, no atomics.
__device__ __forceinline__ uint32_t prefix_lower(const uint64_t *__restrict__ pre, uint32_t nwords,
                                                 uint64_t target) {
    uint32_t a = 0, b = nwords;  // smallest w with pre[w] >= target
    while (a < b) {
        const uint32_t mid = (a + b) >> 1;
        if (pre[mid] >= target) b = mid; else a = mid + 1;
    }
    return a;
}

__device__ __forceinline__ void balanced_range(const uint64_t *__restrict__ pre, uint32_t nwords,
                                               uint64_t wid, uint64_t nw, uint32_t &lo, uint32_t &hi) {
    if (nwords == 0) { lo = hi = 0; return; }
    const uint64_t total = pre[nwords - 1];
    const uint64_t t0 = (total * wid) / nw, t1 = (total * (wid + 1)) / nw;
    lo = t0 == 0 ? 0u : min(prefix_lower(pre, nwords, t0) + 1, nwords);
    hi = wid + 1 >= nw ? nwords : (t1 == 0 ? 0u : min(prefix_lower(pre, nwords, t1) + 1, nwords));
    if (hi < lo) hi = lo;
}

// bfloat16 encode: round to nearest, ties to even, on the bit pattern (add
// 0x7FFF plus the lowest kept bit, keep the top 16 bits; infinities stay
// infinite, NaN stays NaN).  The conversion intrinsic measured 12x slower in
// the PageRank update kernel on this GPU.
__device__ __forceinline__ uint16_t bf16_rne(float f) {
    const uint32_t u = __float_as_uint(f);
    if ((u & 0x7FFFFFFFu) > 0x7F800000u) return (uint16_t)((u >> 16) | 0x40u);  // NaN
    return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

__device__ __forceinline__ bool bit_test(const uint32_t *__restrict__ bm, uint32_t v) {
    return (__ldg(bm + (v >> 5)) >> (v & 31u)) & 1u;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Per-warp staging of list appends in shared memory: one global atomic per
// ~CAP appended items instead of one per 32.  push() and flush() must be
// called by all 32 lanes together.
template <int CAP>
struct WarpAppender {
    uint32_t *buf;                // this warp's CAP entries of shared memory
    uint32_t n = 0;               // staged count (same in every lane)
    uint32_t *dst;
    unsigned long long *dst_n;
    __device__ __forceinline__ void push(bool keep, uint32_t v) {
        const uint32_t lane = threadIdx.x & 31u;
        const unsigned mk = __ballot_sync(0xffffffffu, keep);
        if (keep) buf[n + __popc(mk & ((1u << lane) - 1u))] = v;
        n += __popc(mk);
        if (n > CAP - 32) flush();
    }
    __device__ __forceinline__ void flush() {
        __syncwarp();
        if (n) {
            const uint32_t lane = threadIdx.x & 31u;
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(dst_n, (unsigned long long)n);
            base = __shfl_sync(0xffffffffu, base, 0);
            for (uint32_t i = lane; i < n; i += 32) dst[base + i] = buf[i];
        }
        __syncwarp();
        n = 0;
    }
};

// Frontier bitmap -> degree-binned vertex lists, one warp per group of 32
// bitmap words.  Each lane loads one word (a coalesced 128-byte read), the
// warp then walks the non-zero words four at a time: the degree loads of the
// four words are issued before any append, so a warp keeps four offset
// reads in flight instead of one.  bm == nullptr stands for all vertices.
// nv / ne accumulate, per lane, the vertices and out-edges appended.  CG:
// the bitmap was written earlier in the same kernel (read through L2).
template <int CAP, bool CG = false>
__device__ __forceinline__ void bitmap_to_bins(const uint32_t *bm, uint32_t n, const uint64_t *off, uint32_t smax,
                                               uint32_t mmax, WarpAppender<CAP> &ap0, WarpAppender<CAP> &ap1,
                                               WarpAppender<CAP> &ap2, unsigned long long &nv,
                                               unsigned long long &ne) {
    const uint32_t nwords = (n + 31) / 32;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = (uint64_t)warp * 32; base < nwords; base += (uint64_t)nw * 32) {
        const uint64_t w = base + lane;
        const uint32_t mine = w < nwords ? (bm ? (CG ? __ldcg(bm + w) : bm[w]) : 0xFFFFFFFFu) : 0u;
        unsigned nz = __ballot_sync(0xffffffffu, mine != 0);
        while (nz) {  // warp-uniform
            uint32_t vv[4];
            uint64_t dd[4];
            bool aa[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int j = nz ? __ffs(nz) - 1 : -1;
                if (j >= 0) nz &= nz - 1;
                const uint32_t word = __shfl_sync(0xffffffffu, mine, j >= 0 ? j : 0);
                vv[k] = (uint32_t)((base + (uint32_t)max(j, 0)) * 32 + lane);
                aa[k] = j >= 0 && vv[k] < n && ((word >> lane) & 1u);
                dd[k] = aa[k] ? off[vv[k] + 1] - off[vv[k]] : 0;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t bin = dd[k] <= smax ? 0 : (dd[k] <= mmax ? 1 : 2);
                if (aa[k]) {
                    nv++;
                    ne += dd[k];
                }
                ap0.push(aa[k] && bin == 0, vv[k]);
                ap1.push(aa[k] && bin == 1, vv[k]);
                ap2.push(aa[k] && bin == 2, vv[k]);
            }
        }
    }
}

// Push over the small rows held by a warp, one row per lane (beg, deg and
// the offered value sv; deg = 0 for a lane without a row).  The 32 rows'
// edges are walked as one flattened list: lane l takes edges l, l+32, ...,
// U of them in flight, each mapped to its row by a binary search over the
// lanes' exclusive degree prefix.  Work is balanced whatever the degree mix
// (a lane-per-row walk waits for the warp's longest row, one dependent
// round trip per edge).  offer(d, sv) -> recorded; emit(rec, d) is called
// by all 32 lanes together.
template <int U, typename V, typename Offer, typename Emit>
__device__ __forceinline__ void warp_flat_rows(const uint32_t *adj, uint64_t beg, uint32_t deg, V sv,
                                               Offer &&offer, Emit &&emit) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - deg;
    for (uint32_t e0 = 0; e0 < total; e0 += 32u * U) {  // warp-uniform
        uint32_t d[U];
        V x[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t idx = e0 + (uint32_t)u * 32u + lane;
            uint32_t r = 0;  // the last lane whose prefix is <= idx
#pragma unroll
            for (uint32_t step = 16; step; step >>= 1) {
                const uint32_t pr = __shfl_sync(0xffffffffu, excl, r + step);
                if (pr <= idx) r += step;
            }
            const uint64_t b = __shfl_sync(0xffffffffu, beg, r);
            const uint32_t ex = __shfl_sync(0xffffffffu, excl, r);
            x[u] = __shfl_sync(0xffffffffu, sv, r);
            ok[u] = idx < total;
            d[u] = ok[u] ? __ldg(adj + b + (idx - ex)) : 0u;
        }
        bool rec[U];
#pragma unroll
        for (int u = 0; u < U; ++u) rec[u] = ok[u] && offer(d[u], x[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (e0 + (uint32_t)u * 32u >= total) break;  // warp-uniform
            emit(rec[u], d[u]);
        }
    }
}

// Block-wide sum of a per-thread value; result valid in thread 0.
template <typename T, int BLOCK>
__device__ __forceinline__ T block_sum(T x) {
    __shared__ T sh[BLOCK / 32];
    x = warp_sum(x);
    if (lane_id() == 0) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    T r = 0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < BLOCK / 32) ? sh[threadIdx.x] : T(0);
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

}  // namespace dev
}  // namespace gg
