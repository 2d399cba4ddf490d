// gg_persist.cu -- device-driven frontier traversal: one cooperative launch
// runs every iteration of a BFS-level, BFS-parent or CC analytic.
//
// The host-driven loop (gg_emap.cu) synchronises once per iteration to read
// the frontier counts that decide between sparse push and dense pull
// (include/graptor/api.h:2223-2288).  Here every CTA of a persistent grid
// reads those counts from device memory after a grid barrier and takes the
// same decision, so a whole traversal is one launch with no host round trip
// and no per-iteration launch latency.  Phases of an iteration:
//   [push F->O  or  pull F->O]  barrier  [copy prev / clear old F]  barrier
// A push writes O's degree-binned list and bitmap; a pull writes O's bitmap
// (the list is built by a conversion phase only when a push follows).
//
// Coherence: data written during the launch (values, frontiers, counters,
// candidate lists) are read with ld.global.cg (L2), never through the
// non-coherent L1; the read-only graph uses the read-only path.
//
// The grid barrier is the kernel's only wait.  It is bounded by a
// %globaltimer deadline (timeout_ns); a CTA that gives up sets
// DEV_ERR_TIMEOUT in the state block and every CTA returns at its next
// barrier check, so the host sees GG_ERR_TIMEOUT and the context stays
// usable.  Co-residency of all CTAs is guaranteed by the cooperative launch.
#include <algorithm>
#include <climits>
#include <cuda_bf16.h>

#include <cstring>
#include <type_traits>

#include "gg_internal.cuh"
#include "gg_batch.h"
#include "gg_mlp.cuh"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace gg {

constexpr unsigned FULLP = 0xffffffffu;
constexpr int kPB = 256;           // threads per CTA
constexpr uint32_t kLargeScan = 1024;  // large-bin rows chunked when at most this many
// BFS levels: a listed frontier of at most this many vertices and edges
// continues in the one-cluster kernel k_small_bfs
constexpr unsigned long long kSmallEnterV = 8192, kSmallEnterE = 65536;

struct PFront {
    uint32_t *bins[NBINS];
    uint32_t *bitmap;
    unsigned long long *cnt;  // FC_WORDS
};

struct PState {
    unsigned int bar_count;
    unsigned int bar_gen;
    unsigned int err;
    int iterations;
    int has_list[2];
    int all[2];
    unsigned long long cand_n[2];
    int cand_valid;
    int cand_cur;
    int variant[GG_MAX_ITERS];
    unsigned long long nactv[GG_MAX_ITERS];
    unsigned long long nacte[GG_MAX_ITERS];
    unsigned long long scanned[GG_MAX_ITERS];
    unsigned long long t_ns[GG_MAX_ITERS + 1];
    unsigned long long reached_v, reached_e;
    // timing collection: the forced iteration's input counts, its start and
    // end, and the end of the run (any iteration index)
    unsigned long long f_nactv, f_nacte, f_reached, f_t0, f_t1, t_end;
    int f_seen;
    unsigned long long zeros;  // CC: vertices labelled 0 after the first step
    // fused push work queue counters (reset between iterations), one
    // 128-byte line each so that claims, appends and completions do not
    // contend for one L2 line
    struct alignas(128) Line { unsigned long long v; };
    Line wq_head, wq_tail, wq_done;
    // small-frontier hand-over (BFS levels): the traversal left the frontier
    // at small_cur after small_iter iterations for k_small_bfs (exit_small),
    // which either finishes the run (small_done) or hands back the same way
    int exit_small, small_done, small_iter, small_cur;
    // learned policy: the next step's choice, taken by one warp of CTA 0
    // while the grid finishes the current step (slot = iteration & 1)
    int next_choice[2];
};

struct PArgs {
    const uint64_t *off, *in_off;
    const uint32_t *adj, *in_adj;
    uint32_t n;
    uint64_t m;
    PFront fr[2];
    uint32_t *cand[2];
    const uint32_t *nonisolated;
    const unsigned long long *nonisolated_n;
    void *a, *prev;
    int relax, record, filter, level_k, level_sync;
    int64_t fk;
    int threshold, threshold_k, variant;
    uint32_t smax, mmax, large_ch;
    int K;
    int max_iters;
    unsigned long long timeout_ns;
    PState *st;
    unsigned long long *merge;         // merge-path scratch: list length + CTA count
    const __nv_bfloat16 *sel_w;        // learned selector weights (bfloat16), or null
    float gini;
    int force_iter, force_variant;     // timing collection: one forced (iteration, variant)
    int fusion;                        // sparse pushes run fused (asynchronous) through wq
    int hook;                          // CC: road-network test after step 0, then hooking
    int rows_sorted;                   // CSR rows ascending: hooking stops a row at its first larger id
    uint32_t *wq;                      // fused push work queue, wq_cap entries, all kWqEmpty between phases
    unsigned long long wq_cap;
    int iter0;                         // iterations done before this launch (a resumed run)
    int cur0;                          // index in fr[] of the frontier it starts from
    int small_ok;                      // BFS levels: small frontiers go to k_small_bfs
    int small_from;                    // ... from this iteration on
};

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <typename T> __device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

// Bounded grid barrier (sense = generation counter).  Returns false when any
// CTA has flagged an error (timeout): the caller then returns.
__device__ __forceinline__ bool grid_barrier(PState *st, unsigned long long timeout_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        volatile unsigned int *genp = &st->bar_gen;
        const unsigned int gen = *genp;
        if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
            atomicExch(&st->bar_count, 0u);
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else {
            const unsigned long long t0 = globaltimer();
            while (*genp == gen) {
                if (globaltimer() - t0 > timeout_ns) {
                    atomicOr(&st->err, DEV_ERR_TIMEOUT);
                    break;
                }
                if (*(volatile unsigned int *)&st->err) break;
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile unsigned int *)&st->err == 0;
}

// ---- relax semantics (same table as the host-driven kernels) --------------
template <int R> struct POp {
    using V = typename std::conditional<R == GG_RELAX_MIN_PLUS1_I32, int32_t, uint32_t>::type;
    V *a, *prev;
    int filter;
    int64_t fk;
    int level_sync;
    __device__ __forceinline__ static V none() {
        if constexpr (R == GG_RELAX_MIN_PLUS1_I32) return INT_MAX;
        else return 0xFFFFFFFFu;
    }
    __device__ __forceinline__ V load(uint32_t v) const { return ldcg(a + v); }
    __device__ __forceinline__ bool dst_ok(V cur) const {
        switch (filter) {
        case GG_FILTER_GT_CONST: return (int64_t)cur > fk;
        case GG_FILTER_NE_ZERO: return cur != 0;
        case GG_FILTER_MSB_SET: return ((uint32_t)cur >> 31) != 0;
        default: return true;
        }
    }
    __device__ __forceinline__ V src_val(uint32_t s) const {
        if constexpr (R == GG_RELAX_MIN_PLUS1_I32) return level_sync ? (V)fk : ldcg(a + s) + 1;
        else if constexpr (R == GG_RELAX_MIN_U32) return ldcg(a + s);
        else return (V)s;
    }
    __device__ __forceinline__ bool better(V x, V best) const {
        if constexpr (R == GG_RELAX_SETIF_U32) return ((uint32_t)best >> 31) != 0;
        else return x < best;
    }
    __device__ __forceinline__ V warp_pick(bool ok, V x, unsigned okm) const {
        if constexpr (R == GG_RELAX_SETIF_U32) return __shfl_sync(FULLP, x, __ffs(okm) - 1);
        else return __reduce_min_sync(FULLP, ok ? x : none());
    }
    // push: true iff this thread records d (first change away from prev)
    __device__ __forceinline__ bool offer(uint32_t d, V sv, int record) const {
        V cur = ldcg(a + d);
        if (!dst_ok(cur)) return false;
        V old;
        if constexpr (R == GG_RELAX_SETIF_U32) {
            if (((uint32_t)cur >> 31) == 0) return false;
            old = atomicCAS(a + d, cur, sv);
            if (old != cur) return false;
        } else {
            if (!(sv < cur)) return false;
            old = atomicMin(a + d, sv);
            if (!(sv < old)) return false;
        }
        // level-synchronous: d passed the filter, so it was unvisited and its
        // prev equals the value this thread replaced (no prev load)
        if (R == GG_RELAX_MIN_PLUS1_I32 && level_sync) return true;
        return record == GG_RECORD_NE_PREV ? old == ldcg(prev + d) : true;
    }
};

__device__ __forceinline__ bool bit_cg(const uint32_t *bm, uint32_t v) {
    return (ldcg(bm + (v >> 5)) >> (v & 31u)) & 1u;
}

// warp-aggregated append into O's degree bins + bitmap bit + counts
__device__ __forceinline__ void p_emit(const PArgs &P, const PFront &O, bool rec, uint32_t d,
                                       unsigned long long &nv, unsigned long long &ne) {
    uint64_t deg = 0;
    if (rec) {
        deg = P.off[d + 1] - P.off[d];
        nv++;
        ne += deg;
        atomicOr(O.bitmap + (d >> 5), 1u << (d & 31));
    }
    const uint32_t bin = deg <= P.smax ? 0u : (deg <= P.mmax ? 1u : 2u);
    const unsigned am = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t b = 0; b < NBINS; ++b) {
        const unsigned mk = __ballot_sync(am, rec && bin == b);
        if (mk == 0) continue;
        const int leader = __ffs(mk) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(O.cnt + FC_BIN0 + b, (unsigned long long)__popc(mk));
        base = __shfl_sync(am, base, leader);
        if (rec && bin == b) O.bins[b][base + __popc(mk & ((1u << lane) - 1u))] = d;
    }
}

__device__ __forceinline__ void p_flush(const PFront &O, unsigned long long nv, unsigned long long ne,
                                        unsigned long long sc) {
    nv = dev::block_sum<unsigned long long, kPB>(nv);
    ne = dev::block_sum<unsigned long long, kPB>(ne);
    sc = dev::block_sum<unsigned long long, kPB>(sc);
    if (threadIdx.x == 0) {
        if (nv) atomicAdd(O.cnt + FC_NACTV, nv);
        if (ne) atomicAdd(O.cnt + FC_NACTE, ne);
        if (sc) atomicAdd(O.cnt + FC_SCANNED, sc);
    }
}

// Edges [beg, end) of one source pushed by W cooperating threads (a warp or
// the CTA; `t` = this thread's index among them), four edges per thread in
// flight so that the target loads and atomics of the four overlap.
template <int R, int W>
__device__ __forceinline__ void p_push_edges(const PArgs &P, const POp<R> &op, const PFront &O,
                                             typename POp<R>::V sv, uint64_t beg, uint64_t end, uint32_t t,
                                             unsigned long long &nv, unsigned long long &ne) {
    constexpr int U = 4;
    for (uint64_t base = beg; base < end; base += (uint64_t)W * U) {
        uint32_t d[U];
        bool rec[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t e = base + (uint64_t)u * W + t;
            d[u] = e < end ? __ldg(P.adj + e) : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t e = base + (uint64_t)u * W + t;
            rec[u] = e < end && op.offer(d[u], sv, P.record);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (base + (uint64_t)u * W >= end) break;  // uniform across the W threads
            p_emit(P, O, rec[u], d[u], nv, ne);
        }
    }
}

// ---- sparse push F -> O ------------------------------------------------------
// One shared buffer serves all phases (they never overlap in time).
constexpr int kSmemWords = 3 * (kPB / 32) * 256;  // 24 KiB

template <int R>
__device__ void phase_push(const PArgs &P, const POp<R> &op, const PFront &F, const PFront &O,
                           uint32_t *smem) {
    using V = typename POp<R>::V;
    unsigned long long *s_first = reinterpret_cast<unsigned long long *>(smem);  // kLargeScan + 1
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t c0 = (uint32_t)ldcg(F.cnt + FC_BIN0), c1 = (uint32_t)ldcg(F.cnt + FC_BIN1),
                   c2 = (uint32_t)ldcg(F.cnt + FC_BIN2);
    unsigned long long nv = 0, ne = 0, sc = 0;
    // large bin: rows cut into chunks (chunk table built per CTA in shared memory)
    if (c2 && c2 <= kLargeScan) {
        for (uint32_t i = threadIdx.x; i < c2; i += kPB) {
            const uint32_t v = ldcg(F.bins[2] + i);
            s_first[i + 1] = (P.off[v + 1] - P.off[v] + P.large_ch - 1) / P.large_ch;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_first[0] = 0;
            for (uint32_t i = 1; i <= c2; ++i) s_first[i] += s_first[i - 1];
        }
        __syncthreads();
        const unsigned long long nch = s_first[c2];
        for (unsigned long long c = blockIdx.x; c < nch; c += gridDim.x) {
            uint32_t lo = 0, hi = c2;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_first[mid] <= c) lo = mid; else hi = mid;
            }
            const uint32_t s = ldcg(F.bins[2] + lo);
            const V sv = op.src_val(s);
            const uint64_t beg = P.off[s] + (c - s_first[lo]) * P.large_ch;
            const uint64_t end = min(beg + P.large_ch, P.off[s + 1]);
            if (threadIdx.x == 0) sc += end - beg;
            p_push_edges<R, kPB>(P, op, O, sv, beg, end, threadIdx.x, nv, ne);
        }
    } else if (c2) {
        for (uint32_t i = blockIdx.x; i < c2; i += gridDim.x) {  // a CTA per row
            const uint32_t s = ldcg(F.bins[2] + i);
            const V sv = op.src_val(s);
            const uint64_t beg = P.off[s], end = P.off[s + 1];
            if (threadIdx.x == 0) sc += end - beg;
            p_push_edges<R, kPB>(P, op, O, sv, beg, end, threadIdx.x, nv, ne);
        }
    }
    // medium bin: a warp per row
    const uint64_t gw = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * kPB) >> 5;
    for (uint64_t i = gw; i < c1; i += nw) {
        const uint32_t s = ldcg(F.bins[1] + i);
        const V sv = op.src_val(s);
        const uint64_t beg = P.off[s], end = P.off[s + 1];
        if (lane == 0) sc += end - beg;
        p_push_edges<R, 32>(P, op, O, sv, beg, end, lane, nv, ne);
    }
    // small bin: a warp per 32 rows, their edges flattened
    for (uint64_t base = gw * 32; base < c0; base += nw * 32) {
        const uint64_t i = base + lane;
        const bool have = i < c0;
        uint32_t s = 0;
        uint64_t beg = 0, end = 0;
        V sv = POp<R>::none();
        if (have) {
            s = ldcg(F.bins[0] + i);
            beg = P.off[s];
            end = P.off[s + 1];
            sv = op.src_val(s);
        }
        const uint32_t deg = (uint32_t)(end - beg);
        sc += deg;
        dev::warp_flat_rows<4>(
            P.adj, beg, deg, sv, [&](uint32_t d, V x) { return op.offer(d, x, P.record); },
            [&](bool rec, uint32_t d) { p_emit(P, O, rec, d, nv, ne); });
    }
    p_flush(O, nv, ne, sc);
}

// ---- fused (asynchronous) sparse push ------------------------------------------
// CCv's sparse steps with api::fusion (bench/CCv.C:564-566, executed by
// dsl/emap/fusion.h:163-377): a destination whose label dropped is processed
// at once instead of waiting for the next iteration, so labels cross many hops
// in one step.  Here the pending vertices form one queue in device memory
// shared by all warps: a warp claims the next slot (wq_head), waits until the
// slot is written, processes that vertex's out-edges and appends every
// destination it lowered (wq_tail).  wq_done counts finished entries; the
// phase ends when wq_done == wq_tail (every appended entry finished, so none
// is being processed and no more can appear).  Entries that find the queue
// full are spilled into O (the next iteration's frontier) and counted done.
// Every wait is bounded: a warp gives up after timeout_ns without progress,
// sets DEV_ERR_TIMEOUT and the traversal returns.
constexpr uint32_t kWqEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long *p) {
    return *(const volatile unsigned long long *)p;
}

// spill d into O once (bitmap test-and-set), warp-aggregated list append
__device__ __forceinline__ void p_spill(const PArgs &P, const PFront &O, bool sp, uint32_t d, unsigned long long &nv,
                                        unsigned long long &ne) {
    bool rec = false;
    if (sp) {
        const uint32_t bit = 1u << (d & 31);
        rec = (atomicOr(O.bitmap + (d >> 5), bit) & bit) == 0;
    }
    uint64_t deg = 0;
    if (rec) {
        deg = P.off[d + 1] - P.off[d];
        nv++;
        ne += deg;
    }
    const uint32_t bin = deg <= P.smax ? 0u : (deg <= P.mmax ? 1u : 2u);
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t b = 0; b < NBINS; ++b) {
        const unsigned mk = __ballot_sync(FULLP, rec && bin == b);
        if (mk == 0) continue;
        const int leader = __ffs(mk) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(O.cnt + FC_BIN0 + b, (unsigned long long)__popc(mk));
        base = __shfl_sync(FULLP, base, leader);
        if (rec && bin == b) O.bins[b][base + __popc(mk & ((1u << lane) - 1u))] = d;
    }
}

// append the lanes' vertices (mask `want`) to the queue; overflow spills
__device__ __forceinline__ void wq_append(const PArgs &P, const PFront &O, bool want, uint32_t d,
                                          unsigned long long &nv, unsigned long long &ne) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned mk = __ballot_sync(FULLP, want);
    if (mk == 0) return;
    unsigned long long pos = 0;
    if (lane == 0) pos = atomicAdd(&P.st->wq_tail.v, (unsigned long long)__popc(mk));
    pos = __shfl_sync(FULLP, pos, 0);
    const unsigned long long slot = pos + __popc(mk & ((1u << lane) - 1u));
    const bool spill = want && slot >= P.wq_cap;
    if (want && !spill) *(volatile uint32_t *)(P.wq + slot) = d;
    p_spill(P, O, spill, d, nv, ne);
    const unsigned ns = __popc(__ballot_sync(FULLP, spill));
    if (ns && lane == 0) {
        __threadfence();
        atomicAdd(&P.st->wq_done.v, (unsigned long long)ns);
    }
}

// seed the queue with F's list (all warps), then a grid barrier follows
__device__ void phase_fused_seed(const PArgs &P, const PFront &F, const PFront &O) {
    const unsigned long long b0 = ldcg(F.cnt + FC_BIN0), b1 = ldcg(F.cnt + FC_BIN1), b2 = ldcg(F.cnt + FC_BIN2);
    const unsigned long long tot = b0 + b1 + b2;
    const uint64_t tid = (uint64_t)blockIdx.x * kPB + threadIdx.x, nth = (uint64_t)gridDim.x * kPB;
    unsigned long long nv = 0, ne = 0;
    for (uint64_t base = tid - (threadIdx.x & 31u); base < tot; base += nth) {
        const uint64_t i = base + (threadIdx.x & 31u);
        uint32_t v = 0;
        if (i < tot) v = i < b0 ? ldcg(F.bins[0] + i) : (i < b0 + b1 ? ldcg(F.bins[1] + i - b0) : ldcg(F.bins[2] + i - b0 - b1));
        wq_append(P, O, i < tot, v, nv, ne);
    }
    p_flush(O, nv, ne, 0);
}

template <int R>
__device__ void phase_fused_run(const PArgs &P, const POp<R> &op, const PFront &O) {
    using V = typename POp<R>::V;
    PState *st = P.st;
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long nv = 0, ne = 0, sc = 0;
    for (;;) {
        unsigned long long idx = 0;
        uint32_t v = 0;
        int state = 0;  // 1: got an entry, 2: finished, 3: error
        if (lane == 0) {
            idx = atomicAdd(&st->wq_head.v, 1ull);
            unsigned long long t0 = globaltimer(), seen = ~0ull;
            unsigned nap = 32, polls = 0;  // backoff: idle warps poll less often
            for (;;) {
                // poll the claimed slot itself (a different address per warp);
                // the shared counters only every 8th time
                if (idx < P.wq_cap) {
                    v = *(volatile uint32_t *)(P.wq + idx);
                    if (v != kWqEmpty) { state = 1; break; }
                }
                if ((++polls & 7u) == 0 || idx >= P.wq_cap) {
                    const unsigned long long dn = ld_volatile(&st->wq_done.v);
                    __threadfence();
                    if (dn == ld_volatile(&st->wq_tail.v)) { state = 2; break; }
                    if (dn != seen) {  // progress elsewhere: restart the clock
                        seen = dn;
                        t0 = globaltimer();
                    }
                }
                if (*(volatile unsigned int *)&st->err) { state = 3; break; }
                if (globaltimer() - t0 > P.timeout_ns) {
                    atomicOr(&st->err, DEV_ERR_TIMEOUT);
                    state = 3;
                    break;
                }
                __nanosleep(nap);
                if (nap < 1024) nap <<= 1;
            }
            if (state == 1) *(volatile uint32_t *)(P.wq + idx) = kWqEmpty;  // clean for the next phase
        }
        state = __shfl_sync(FULLP, state, 0);
        if (state != 1) break;
        v = __shfl_sync(FULLP, v, 0);
        V lv = 0;
        if (lane == 0) {
            lv = ldcg((const V *)P.a + v);
            if (P.record == GG_RECORD_NE_PREV) ((V *)P.prev)[v] = lv;  // prev == value once processed
        }
        lv = __shfl_sync(FULLP, lv, 0);
        const uint64_t beg = P.off[v], end = P.off[v + 1];
        if (lane == 0) sc += end - beg;
        for (uint64_t base = beg; base < end; base += 32) {
            const uint64_t e = base + lane;
            bool want = false;
            uint32_t d = 0;
            if (e < end) {
                d = __ldg(P.adj + e);
                const V cur = ldcg((const V *)P.a + d);
                if (op.dst_ok(cur) && lv < cur) want = lv < atomicMin((V *)P.a + d, lv);
            }
            if (__any_sync(FULLP, want)) {
                __threadfence();  // the lowered values before the queue entries
                wq_append(P, O, want, d, nv, ne);
            }
        }
        if (lane == 0) {
            __threadfence();  // appended entries before this one counts as done
            atomicAdd(&st->wq_done.v, 1ull);
        }
    }
    p_flush(O, nv, ne, sc);
}

// ---- CC by min-id hooking -------------------------------------------------------
// label[] is a forest: every label is the id of a vertex of the same
// component and never above the vertex's own id, so following labels ends at
// a vertex labelled with itself (a root).  Hooking an edge's two roots, the
// larger under the smaller (compare-and-swap on the larger root), and
// repeating until they agree merges the trees; the root of a component is
// then its minimum id, the CCv label.  Finds halve paths with plain stores
// (a label only ever moves to an ancestor, so racing stores stay valid).
__device__ __forceinline__ uint32_t uf_find(uint32_t *lab, uint32_t x) {
    for (int guard = 0; guard < (1 << 26); ++guard) {  // a chain of n links at most
        const uint32_t p = ldcg(lab + x);
        if (p == x) return x;
        const uint32_t gp = ldcg(lab + p);
        if (gp != p) lab[x] = gp;
        x = gp;
    }
    return x;
}

__device__ __forceinline__ void uf_hook(uint32_t *lab, uint32_t u, uint32_t v) {
    uint32_t ru = uf_find(lab, u), rv = uf_find(lab, v);
    for (int guard = 0; ru != rv && guard < (1 << 26); ++guard) {
        const uint32_t lo = ru < rv ? ru : rv, hi = ru ^ rv ^ lo;
        const uint32_t old = atomicCAS(lab + hi, hi, lo);
        if (old == hi) break;
        ru = uf_find(lab, old);
        rv = uf_find(lab, lo);
    }
}

__device__ void phase_hook(const PArgs &P) {
    uint32_t *lab = (uint32_t *)P.a;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t gw = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * kPB) >> 5;
    // a warp per 32 vertices; each vertex's edges to smaller ids (each
    // undirected edge once): rows of up to 32 edges by their lane, longer
    // rows by the whole warp in turn
    for (uint64_t w = gw; w * 32 < P.n; w += nw) {
        const uint32_t u = (uint32_t)(w * 32 + lane);
        uint64_t beg = 0, end = 0;
        if (u < P.n) {
            beg = P.off[u];
            end = P.off[u + 1];
        }
        const bool longrow = end - beg > 32;
        if (!longrow)
            for (uint64_t e = beg; e < end; ++e) {
                const uint32_t v = __ldg(P.adj + e);
                if (v >= u) {
                    if (P.rows_sorted) break;  // the rest of the row is larger
                    continue;
                }
                uf_hook(lab, u, v);
            }
        unsigned pend = __ballot_sync(FULLP, longrow);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint32_t uj = __shfl_sync(FULLP, u, j);
            const uint64_t bj = __shfl_sync(FULLP, beg, j), ej = __shfl_sync(FULLP, end, j);
            for (uint64_t e = bj + lane; e < ej; e += 32) {
                const uint32_t v = __ldg(P.adj + e);
                if (v < uj) uf_hook(lab, uj, v);
            }
        }
    }
}

// After CCv's first step on a graph that fails the road-network test, vertex
// 0's label 0 has reached most of its component.  A vertex whose root is 0
// is in vertex 0's component, whose CCv label is 0, so its row is skipped;
// every other vertex hooks all its edges (both directions: an edge to a
// skipped vertex is taken from this side).  A warp per 32 vertices, rows of
// up to 32 edges by their lane, longer ones by the whole warp in turn.
__device__ void phase_hook_rest(const PArgs &P) {
    uint32_t *lab = (uint32_t *)P.a;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t gw = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * kPB) >> 5;
    for (uint64_t w = gw; w * 32 < P.n; w += nw) {
        const uint32_t u = (uint32_t)(w * 32 + lane);
        uint64_t beg = 0, end = 0;
        if (u < P.n && uf_find(lab, u) != 0) {
            beg = P.off[u];
            end = P.off[u + 1];
        }
        const bool longrow = end - beg > 32;
        if (!longrow)
            for (uint64_t e = beg; e < end; ++e) uf_hook(lab, u, __ldg(P.adj + e));
        unsigned pend = __ballot_sync(FULLP, longrow);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint32_t uj = __shfl_sync(FULLP, u, j);
            const uint64_t bj = __shfl_sync(FULLP, beg, j), ej = __shfl_sync(FULLP, end, j);
            for (uint64_t e = bj + lane; e < ej; e += 32) uf_hook(lab, uj, __ldg(P.adj + e));
        }
    }
}

// The root of x without path halving: in the final pass every vertex's
// entry is written once, by its own thread, with its root; a halving store
// from another thread's walk could land after it and leave a non-root there.
__device__ __forceinline__ uint32_t uf_root(const uint32_t *lab, uint32_t x) {
    for (int guard = 0; guard < (1 << 26); ++guard) {  // a chain of n links at most
        const uint32_t p = ldcg(lab + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

__device__ void phase_hook_finish(const PArgs &P) {
    uint32_t *lab = (uint32_t *)P.a;
    const uint64_t tid = (uint64_t)blockIdx.x * kPB + threadIdx.x, nth = (uint64_t)gridDim.x * kPB;
    for (uint64_t v = tid; v < P.n; v += nth) {
        const uint32_t r = uf_root(lab, (uint32_t)v);
        lab[v] = r;
        if (P.prev) ((uint32_t *)P.prev)[v] = r;
    }
}

// ---- dense pull F -> O over a candidate list -------------------------------
template <int R, bool SRCF>
__device__ void phase_pull(const PArgs &P, const POp<R> &op, const PFront &F, const PFront &O,
                           const uint32_t *cand, unsigned long long ncand, uint32_t *cand_out,
                           unsigned long long *cand_out_n, uint32_t *smem) {
    using V = typename POp<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    dev::WarpAppender<256> keepers{smem + (threadIdx.x >> 5) * 256, 0, cand_out, cand_out_n};
    unsigned long long nv = 0, ne = 0, sc = 0;
    const uint64_t nw = ((uint64_t)gridDim.x * kPB) >> 5;
    for (uint64_t w = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5; (w << 5) < ncand; w += nw) {
        const uint64_t item = (w << 5) + lane;
        const bool valid = item < ncand;
        const uint32_t d = valid ? ldcg(cand + item) : 0u;
        V best = POp<R>::none();
        uint64_t e = 0, end = 0;
        if (valid) {
            best = op.load(d);
            e = P.in_off[d];
            end = P.in_off[d + 1];
        }
        bool act = valid && op.dst_ok(best);
        bool changed = false;
        const uint64_t beg = e;
        const uint64_t lim = min(end, e + (uint64_t)P.K);
        while (act && e < lim) {
            const int cnt = (int)min((uint64_t)4, lim - e);
            uint32_t sv[4];
            bool inF[4];
            V xv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) sv[j] = j < cnt ? __ldg(P.in_adj + e + j) : 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                inF[j] = j < cnt && (!SRCF || bit_cg(F.bitmap, sv[j]));
                xv[j] = j < cnt ? op.src_val(sv[j]) : POp<R>::none();
            }
            int used = cnt;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j < cnt && act && inF[j] && op.better(xv[j], best)) {
                    best = xv[j];
                    changed = true;
                    if (!op.dst_ok(best)) {
                        act = false;
                        used = j + 1;
                    }
                }
            }
            e += used;
        }
        sc += e - beg;
        unsigned pend = __ballot_sync(FULLP, act && e < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULLP, e, j);
            const uint64_t endj = __shfl_sync(FULLP, end, j);
            V bj = __shfl_sync(FULLP, best, j);
            bool chj = false, actj = true;
            for (uint64_t base = ej; base < endj; base += 32) {
                const uint64_t idx = base + lane;
                bool ok = false;
                V x = POp<R>::none();
                if (idx < endj) {
                    const uint32_t s = __ldg(P.in_adj + idx);
                    if (!SRCF || bit_cg(F.bitmap, s)) {
                        x = op.src_val(s);
                        ok = op.better(x, bj);
                    }
                }
                if (lane == 0) sc += min((uint64_t)32, endj - base);
                const unsigned okm = __ballot_sync(FULLP, ok);
                if (okm) {
                    bj = op.warp_pick(ok, x, okm);
                    chj = true;
                    if (!op.dst_ok(bj)) {
                        actj = false;
                        break;
                    }
                }
            }
            if ((int)lane == j) {
                best = bj;
                changed = changed || chj;
                act = actj;
            }
        }
        bool rec = false;
        if (changed) {
            op.a[d] = best;
            if (P.record == GG_RECORD_NE_PREV) {
                // level-synchronous: d was unvisited, so its prev equals the
                // value replaced; prev is neither read nor written
                if (R == GG_RELAX_MIN_PLUS1_I32 && op.level_sync) {
                    rec = true;
                } else if (best != ldcg(op.prev + d)) {
                    op.prev[d] = best;
                    rec = true;
                }
            } else if (P.record == GG_RECORD_REDUCTION) {
                rec = true;
            }
        }
        // O bitmap: one atomicOr per distinct word of the warp
        unsigned todo = __ballot_sync(FULLP, rec);
        while (todo) {
            const int leader = __ffs(todo) - 1;
            const uint32_t w0 = __shfl_sync(FULLP, d >> 5, leader);
            const bool mine = rec && (d >> 5) == w0;
            const unsigned bits = __reduce_or_sync(FULLP, mine ? (1u << (d & 31)) : 0u);
            if ((int)lane == leader) atomicOr(O.bitmap + w0, bits);
            todo &= ~__ballot_sync(FULLP, mine);
        }
        if (rec) {
            nv++;
            // out-degree: for a symmetric graph the CSC is the CSR, and d's
            // row bounds are already in registers
            ne += P.off == P.in_off ? end - beg : P.off[d + 1] - P.off[d];
        }
        keepers.push(valid && act && end > beg, d);
    }
    keepers.flush();
    p_flush(O, nv, ne, sc);
}

// F's bitmap -> F's binned list (only before a push that follows a pull)
__device__ void phase_bitmap_to_list(const PArgs &P, const PFront &F, uint32_t *smem) {
    const uint32_t wib = threadIdx.x >> 5;
    constexpr int per = (kPB / 32) * 256;
    dev::WarpAppender<256> ap0{smem + 0 * per + wib * 256, 0, F.bins[0], F.cnt + FC_BIN0};
    dev::WarpAppender<256> ap1{smem + 1 * per + wib * 256, 0, F.bins[1], F.cnt + FC_BIN1};
    dev::WarpAppender<256> ap2{smem + 2 * per + wib * 256, 0, F.bins[2], F.cnt + FC_BIN2};
    unsigned long long nv = 0, ne = 0;  // the counts are known already
    dev::bitmap_to_bins<256, true>(F.bitmap, P.n, P.off, P.smax, P.mmax, ap0, ap1, ap2, nv, ne);
    ap0.flush();
    ap1.flush();
    ap2.flush();
}

// ---- dense push from F's bitmap ----------------------------------------------
template <int R>
__device__ void phase_push_dense(const PArgs &P, const POp<R> &op, const PFront &F, const PFront &O, bool all) {
    using V = typename POp<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwords = (P.n + 31) / 32;
    const uint64_t nw = ((uint64_t)gridDim.x * kPB) >> 5;
    unsigned long long nv = 0, ne = 0, sc = 0;
    for (uint64_t w = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5; w < nwords; w += nw) {
        const uint32_t word = all ? 0xFFFFFFFFu : ldcg(F.bitmap + w);
        if (word == 0) continue;  // warp-uniform
        const uint32_t s = (uint32_t)w * 32 + lane;
        const bool act = s < P.n && ((word >> lane) & 1u);
        uint64_t beg = 0, end = 0;
        V sv = POp<R>::none();
        if (act) {
            beg = P.off[s];
            end = P.off[s + 1];
            sv = op.src_val(s);
        }
        const uint32_t k1 = (uint32_t)min(end - beg, (uint64_t)P.K);
        const uint32_t maxk = __reduce_max_sync(FULLP, k1);
        for (uint32_t k = 0; k < maxk; ++k) {
            bool rec = false;
            uint32_t d = 0;
            if (k < k1) {
                d = __ldg(P.adj + beg + k);
                rec = op.offer(d, sv, P.record);
            }
            p_emit(P, O, rec, d, nv, ne);
        }
        sc += k1;
        unsigned pend = __ballot_sync(FULLP, act && beg + k1 < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULLP, beg + k1, j), endj = __shfl_sync(FULLP, end, j);
            const V svj = __shfl_sync(FULLP, sv, j);
            if (lane == 0) sc += endj - ej;
            for (uint64_t base = ej; base < endj; base += 32) {
                const uint64_t e = base + lane;
                bool rec = false;
                uint32_t d = 0;
                if (e < endj) {
                    d = __ldg(P.adj + e);
                    rec = op.offer(d, svj, P.record);
                }
                p_emit(P, O, rec, d, nv, ne);
            }
        }
    }
    p_flush(O, nv, ne, sc);
}

// ---- edge-balanced ("merge path") push ---------------------------------------
// Rows of F's list are cut into chunks of kMergeCh edges; a device-wide scan
// of the chunk counts (M1 per-CTA slice sums, M2 slice prefixes) lets every
// warp take equal chunk ranges in M3 and find each chunk's row by binary
// search.  Uses the scratch array P.merge (list length + CTA count entries).
constexpr uint32_t kMergeCh = 64;

__device__ __forceinline__ uint32_t list_at(const PFront &F, uint64_t i, uint64_t c0, uint64_t c1) {
    return i < c0 ? ldcg(F.bins[0] + i) : (i < c0 + c1 ? ldcg(F.bins[1] + i - c0) : ldcg(F.bins[2] + i - c0 - c1));
}

__device__ void phase_merge_count(const PArgs &P, const PFront &F) {
    const uint64_t c0 = ldcg(F.cnt + FC_BIN0), c1 = ldcg(F.cnt + FC_BIN1), c2 = ldcg(F.cnt + FC_BIN2);
    const uint64_t L = c0 + c1 + c2, G = gridDim.x;
    const uint64_t lo = L * blockIdx.x / G, hi = L * (blockIdx.x + 1) / G;
    unsigned long long sum = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kPB) {
        const uint32_t v = list_at(F, i, c0, c1);
        const unsigned long long ch = (P.off[v + 1] - P.off[v] + kMergeCh - 1) / kMergeCh;
        P.merge[i] = ch;
        sum += ch;
    }
    sum = dev::block_sum<unsigned long long, kPB>(sum);
    if (threadIdx.x == 0) P.merge[L + blockIdx.x] = sum;
}

// Block-wide exclusive scan of one value per thread (kPB threads).
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long x, unsigned long long *total) {
    __shared__ unsigned long long s_w[kPB / 32];
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    unsigned long long inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(FULLP, inc, o);
        if (lane >= (uint32_t)o) inc += t;
    }
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    unsigned long long wbase = 0, tot = 0;
    for (int w = 0; w < kPB / 32; ++w) {
        if (w < (int)wid) wbase += s_w[w];
        tot += s_w[w];
    }
    __syncthreads();
    *total = tot;
    return wbase + inc - x;
}

__device__ void phase_merge_scan(const PArgs &P, const PFront &F) {
    const uint64_t c0 = ldcg(F.cnt + FC_BIN0), c1 = ldcg(F.cnt + FC_BIN1), c2 = ldcg(F.cnt + FC_BIN2);
    const uint64_t L = c0 + c1 + c2, G = gridDim.x;
    const uint64_t lo = L * blockIdx.x / G, hi = L * (blockIdx.x + 1) / G;
    // offset of this CTA's slice: sum of the earlier CTAs' slice sums
    unsigned long long o = 0;
    for (uint64_t b = threadIdx.x; b < blockIdx.x; b += kPB) o += ldcg(P.merge + L + b);
    o = dev::block_sum<unsigned long long, kPB>(o);
    __shared__ unsigned long long s_run;
    if (threadIdx.x == 0) s_run = o;
    __syncthreads();
    // exclusive prefix of the slice, kPB entries at a time, in place
    for (uint64_t base = lo; base < hi; base += kPB) {
        const uint64_t i = base + threadIdx.x;
        const unsigned long long c = i < hi ? ldcg(P.merge + i) : 0ull;
        unsigned long long tot;
        const unsigned long long ex = block_exclusive_scan(c, &tot);
        const unsigned long long run = s_run;
        if (i < hi) P.merge[i] = run + ex;
        __syncthreads();
        if (threadIdx.x == 0) s_run = run + tot;
        __syncthreads();
    }
}

template <int R>
__device__ void phase_merge_push(const PArgs &P, const POp<R> &op, const PFront &F, const PFront &O) {
    using V = typename POp<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t c0 = ldcg(F.cnt + FC_BIN0), c1 = ldcg(F.cnt + FC_BIN1), c2 = ldcg(F.cnt + FC_BIN2);
    const uint64_t L = c0 + c1 + c2, G = gridDim.x;
    __shared__ unsigned long long s_total;
    unsigned long long part = 0;
    for (uint64_t b = threadIdx.x; b < G; b += kPB) part += ldcg(P.merge + L + b);
    part = dev::block_sum<unsigned long long, kPB>(part);
    if (threadIdx.x == 0) s_total = part;
    __syncthreads();
    const unsigned long long total = s_total;
    unsigned long long nv = 0, ne = 0, sc = 0;
    const uint64_t nw = ((uint64_t)G * kPB) >> 5;
    for (uint64_t c = ((uint64_t)blockIdx.x * kPB + threadIdx.x) >> 5; c < total; c += nw) {
        uint64_t a = 0, b = L;  // last row i with prefix[i] <= c
        while (b - a > 1) {
            const uint64_t mid = (a + b) >> 1;
            if (ldcg(P.merge + mid) <= c) a = mid; else b = mid;
        }
        const uint32_t s = list_at(F, a, c0, c1);
        const V sv = op.src_val(s);
        const uint64_t beg = P.off[s] + (c - ldcg(P.merge + a)) * kMergeCh;
        const uint64_t end = min(beg + kMergeCh, P.off[s + 1]);
        if (lane == 0) sc += end - beg;
        for (uint64_t base = beg; base < end; base += 32) {
            const uint64_t e = base + lane;
            bool rec = false;
            uint32_t d = 0;
            if (e < end) {
                d = __ldg(P.adj + e);
                rec = op.offer(d, sv, P.record);
            }
            p_emit(P, O, rec, d, nv, ne);
        }
    }
    p_flush(O, nv, ne, sc);
}

// Threshold / fixed / learned choice; identical in every CTA (same inputs,
// same arithmetic).  Returns a gg_variant.
// Last network evaluation of this CTA: consecutive iterations of a
// high-diameter traversal have nearly the same features, and the choice is
// reused while every feature stays within kSelReuse of the evaluated ones
// (every CTA sees the same sequence, so all CTAs still agree).
struct SelCache {
    unsigned long long nactv, nacte, unreached;
    int iter;
    int choice;
    int valid;
};

// within a factor 1 + 1/16 (log2 change below 0.09: under 1/256 of a
// log-scaled feature)
__device__ __forceinline__ bool sel_close(unsigned long long a, unsigned long long b) {
    const unsigned long long d = a > b ? a - b : b - a, mx = a > b ? a : b;
    return d * 16 <= mx;
}

// The learned choice for a step with these frontier counts, unreached count
// and iteration (one warp: every lane returns it; lane 0 updates the cache).
__device__ int learned_choice(const PArgs &P, const __nv_bfloat16 *selw, unsigned long long nactv,
                              unsigned long long nacte, unsigned long long unr, int it, SelCache *cache) {
    const double n = P.n, m = (double)P.m, fv = (double)nactv, fe = (double)nacte;
    const int tv = (nactv + nacte) <= P.m / 20 ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
    // CC: a frontier far from the threshold's boundary (more than 8x on
    // either side) keeps the threshold's choice without an evaluation -- a CC
    // step's records differ by a few per cent between variants there, less
    // than an evaluation in the step's critical path costs
    if (P.relax == GG_RELAX_MIN_U32 && ((nactv + nacte) * 8 < P.m / 20 || (nactv + nacte) > (P.m / 20) * 8)) {
        if ((threadIdx.x & 31) == 0) {
            cache->nactv = nactv;
            cache->nacte = nacte;
            cache->unreached = unr;
            cache->iter = it;
            cache->choice = tv;
            cache->valid = 1;
        }
        return tv;
    }
    float x[GG_SEL_FEATURES];
    x[0] = (float)(log2(1.0 + fv) / 32);
    x[1] = (float)(log2(1.0 + fe) / 40);
    x[2] = (float)(log2(1.0 + (double)unr) / 32);
    x[3] = (float)(log2(1.0 + it) / 8);
    x[4] = (float)(log2(1.0 + (n > 0 ? m / n : 0)) / 8);
    x[5] = P.gini;
    x[6] = (float)(n > 0 ? fv / n : 0);
    x[7] = (float)(m > 0 ? fe / m : 0);
    x[8] = (float)fmin(4.0, m > 0 ? (fv + fe) / m : 0.0);
    x[9] = (float)(log2(n > 1 ? n : 1.0) / 32);
    float o[GG_SEL_VARIANTS], z1, a1, z2, a2;
    mlp::warp_forward(selw, x, o, z1, a1, z2, a2);
    int best = 0;
    for (int v = 1; v < GG_SEL_VARIANTS; ++v)
        if (o[v] < o[best]) best = v;
    // the threshold's choice stands unless the network predicts a clear gain over it
    const float margin = P.relax == GG_RELAX_MIN_U32 ? mlp::kSelMarginCC : mlp::kSelMargin;
    if (!(o[best] < o[tv] - margin)) best = tv;
    if ((threadIdx.x & 31) == 0) {
        cache->nactv = nactv;
        cache->nacte = nacte;
        cache->unreached = unr;
        cache->iter = it;
        cache->choice = best;
        cache->valid = 1;
    }
    return best;
}

__device__ int choose_variant(const PArgs &P, int iter, unsigned long long nactv, unsigned long long nacte,
                              bool f_all, const PState *st, int *s_choice, SelCache *cache,
                              const __nv_bfloat16 *selw) {
    if (f_all) return GG_VAR_PULL_DENSE;
    if (iter == P.force_iter) return P.force_variant;
    if (P.variant >= 0) return P.variant;
    switch (P.threshold) {
    case GG_THRESH_ALWAYS_SPARSE: return GG_VAR_PUSH_SPARSE;
    case GG_THRESH_ALWAYS_DENSE: return GG_VAR_PULL_DENSE;
    case GG_THRESH_FRAC:
        return (float)(nactv + nacte) <= (float)P.m / (float)(100.0 / (float)P.threshold_k) ? GG_VAR_PUSH_SPARSE
                                                                                            : GG_VAR_PULL_DENSE;
    case GG_THRESH_LEARNED:
        if (P.sel_w) {
            // reuse the last evaluation while the inputs stay close (every
            // thread tests the shared cache: no barrier on the common path;
            // the frontier counts and the iteration decide a reuse, the
            // unreached count, one more L2 load, only feeds an evaluation)
            const int it = min(iter, 255);
            if (cache->valid && sel_close(nactv, cache->nactv) && sel_close(nacte, cache->nacte) &&
                it - cache->iter < 8)
                return cache->choice;
            // warp 0 evaluates the network, the CTA reads its choice
            if (threadIdx.x < 32) {
                const unsigned long long reached = ldcg(&st->reached_v);
                const unsigned long long unr = reached < P.n ? P.n - reached : 0ull;
                learned_choice(P, selw, nactv, nacte, unr, it, cache);
            }
            __syncthreads();
            return cache->choice;
        }
        // no network attached: the default threshold
    default:
        return (nactv + nacte) <= P.m / 20 ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
    }
}

template <int R>
__global__ void __launch_bounds__(kPB) k_traverse(PArgs P) {
    __shared__ __align__(16) uint32_t smem[kSmemWords];
    __shared__ int s_choice;
    __shared__ SelCache s_sel;
    // the selector's weights in shared memory: an evaluation then waits on
    // no global load (3 KiB, copied once per launch)
    __shared__ __nv_bfloat16 s_selw[GG_SEL_NPARAMS];
    if (threadIdx.x == 0) s_sel.valid = 0;
    if (P.sel_w && P.threshold == GG_THRESH_LEARNED)
        for (int i = threadIdx.x; i < GG_SEL_NPARAMS; i += kPB) s_selw[i] = P.sel_w[i];
    __syncthreads();
    static_assert(kSmemWords * 4 >= (kLargeScan + 1) * 8, "chunk table fits the shared buffer");
    PState *st = P.st;
    POp<R> op;
    op.a = (typename POp<R>::V *)P.a;
    op.prev = (typename POp<R>::V *)P.prev;
    op.filter = P.filter;
    op.fk = P.fk;
    op.level_sync = P.level_sync;
    const uint64_t tid = (uint64_t)blockIdx.x * kPB + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * kPB;
    int cur = P.cur0;
    int iter = P.iter0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned long long t0 = globaltimer();
        if (iter <= GG_MAX_ITERS) st->t_ns[iter] = t0;
        if (P.force_iter == iter) st->f_t0 = t0;
    }
    for (; iter < P.max_iters; ++iter) {
        const PFront F = P.fr[cur], O = P.fr[cur ^ 1];
        const unsigned long long nactv = ldcg(F.cnt + FC_NACTV), nacte = ldcg(F.cnt + FC_NACTE);
        const int f_all = ldcg(&st->all[cur]);
        if (nactv == 0 && !f_all) break;
        if (P.level_k) op.fk = iter + 1;
        // learned policy: the choice was taken during the previous step's
        // post-processing, except for a launch's first step
        const bool pre = P.sel_w && P.threshold == GG_THRESH_LEARNED && P.variant < 0 && iter > P.iter0 &&
                         !f_all && iter != P.force_iter;
        const int var = pre ? ldcg(&st->next_choice[iter & 1])
                            : choose_variant(P, iter, nactv, nacte, f_all != 0, st, &s_choice, &s_sel, s_selw);
        // (the reached count this step starts from, for the next choice)
        const unsigned long long reached_top =
            (blockIdx.x == 0 && (threadIdx.x >> 5) == 1 && P.sel_w) ? ldcg(&st->reached_v) : 0ull;
        // a small listed frontier to push: the run continues in one CTA
        // cluster (k_small_bfs); every CTA reads the same counts, so all
        // leave together
        if (P.small_ok && var == GG_VAR_PUSH_SPARSE && iter >= P.small_from && !f_all && nactv <= kSmallEnterV &&
            nacte <= kSmallEnterE && ldcg(&st->has_list[cur])) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->exit_small = 1;
                st->small_iter = iter;
                st->small_cur = cur;
                st->iterations = iter;
            }
            return;
        }
        const bool pushes = var != GG_VAR_PULL_DENSE;
        if (blockIdx.x == 0 && threadIdx.x == 0 && iter == P.force_iter) {
            st->f_nactv = nactv;
            st->f_nacte = nacte;
            st->f_reached = ldcg(&st->reached_v);
            st->f_seen = 1;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0 && iter < GG_MAX_ITERS) {
            st->variant[iter] = var;
            st->nactv[iter] = nactv;
            st->nacte[iter] = nacte;
        }
        if (var == GG_VAR_PUSH_SPARSE || var == GG_VAR_PUSH_MERGE) {
            if (!ldcg(&st->has_list[cur])) {
                __syncthreads();
                phase_bitmap_to_list(P, F, smem);
                if (!grid_barrier(st, P.timeout_ns)) return;
            }
            __syncthreads();
            if (var == GG_VAR_PUSH_SPARSE && P.fusion) {
                phase_fused_seed(P, F, O);
                if (!grid_barrier(st, P.timeout_ns)) return;
                phase_fused_run<R>(P, op, O);
            } else if (var == GG_VAR_PUSH_SPARSE) {
                phase_push<R>(P, op, F, O, smem);
            } else {
                phase_merge_count(P, F);
                if (!grid_barrier(st, P.timeout_ns)) return;
                phase_merge_scan(P, F);
                if (!grid_barrier(st, P.timeout_ns)) return;
                phase_merge_push<R>(P, op, F, O);
            }
        } else if (var == GG_VAR_PUSH_DENSE) {
            __syncthreads();
            phase_push_dense<R>(P, op, F, O, f_all != 0);
        } else {
            const int cc = ldcg(&st->cand_cur);
            const bool cv = ldcg(&st->cand_valid) != 0;
            const uint32_t *cin = cv ? P.cand[cc] : P.nonisolated;
            const unsigned long long nin = cv ? ldcg(&st->cand_n[cc]) : ldcg(P.nonisolated_n);
            __syncthreads();
            if (f_all)
                phase_pull<R, false>(P, op, F, O, cin, nin, P.cand[cc ^ 1], &st->cand_n[cc ^ 1], smem);
            else
                phase_pull<R, true>(P, op, F, O, cin, nin, P.cand[cc ^ 1], &st->cand_n[cc ^ 1], smem);
        }
        if (!grid_barrier(st, P.timeout_ns)) return;
        // post: maintain copies for a push, recycle the old frontier as next output
        if (pushes && P.record == GG_RECORD_NE_PREV && !(P.relax == GG_RELAX_MIN_PLUS1_I32 && P.level_sync)) {
            const unsigned long long b0 = ldcg(O.cnt + FC_BIN0), b1 = ldcg(O.cnt + FC_BIN1),
                                     b2 = ldcg(O.cnt + FC_BIN2);
            for (uint64_t i = tid; i < b0 + b1 + b2; i += nthreads) {
                const uint32_t v = i < b0 ? ldcg(O.bins[0] + i)
                                          : (i < b0 + b1 ? ldcg(O.bins[1] + i - b0) : ldcg(O.bins[2] + i - b0 - b1));
                if (P.relax == GG_RELAX_MIN_PLUS1_I32) ((int32_t *)P.prev)[v] = ldcg((int32_t *)P.a + v);
                else ((uint32_t *)P.prev)[v] = ldcg((uint32_t *)P.a + v);
            }
        }
        const uint32_t nwords = (P.n + 31) / 32;
        for (uint64_t w = tid; w < nwords; w += nthreads) F.bitmap[w] = 0u;
        if (P.sel_w && P.threshold == GG_THRESH_LEARNED && P.variant < 0 && blockIdx.x == 0 &&
            (threadIdx.x >> 5) == 1) {
            // the next step's choice from the output frontier's final counts
            const unsigned long long nv = ldcg(O.cnt + FC_NACTV), ne = ldcg(O.cnt + FC_NACTE);
            const unsigned long long reached = reached_top + nactv;
            const unsigned long long unr = reached < P.n ? P.n - reached : 0ull;
            const int it = min(iter + 1, 255);
            int c;
            if (s_sel.valid && sel_close(nv, s_sel.nactv) && sel_close(ne, s_sel.nacte) && it - s_sel.iter < 8)
                c = s_sel.choice;
            else
                c = learned_choice(P, s_selw, nv, ne, unr, it, &s_sel);
            if ((threadIdx.x & 31) == 0) st->next_choice[(iter + 1) & 1] = c;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            // decision inputs change only here, between the two barriers, so
            // every CTA's next choice reads the same values
            st->reached_v += nactv;
            st->reached_e += nacte;
            st->wq_head.v = 0;
            st->wq_tail.v = 0;
            st->wq_done.v = 0;
            for (int i = 0; i < FC_WORDS; ++i) F.cnt[i] = 0;
            st->has_list[cur ^ 1] = pushes ? 1 : 0;
            st->all[cur] = 0;
            st->all[cur ^ 1] = 0;
            if (!pushes) {
                st->cand_valid = 1;
                st->cand_n[ldcg(&st->cand_cur)] = 0;
                st->cand_cur ^= 1;
            }
            if (iter < GG_MAX_ITERS) {
                st->scanned[iter] = ldcg(O.cnt + FC_SCANNED);
                st->t_ns[iter + 1] = globaltimer();
            }
            if (iter == P.force_iter || iter + 1 == P.force_iter) {
                const unsigned long long now = globaltimer();
                if (iter == P.force_iter) st->f_t1 = now; else st->f_t0 = now;
            }
        }
        if (!grid_barrier(st, P.timeout_ns)) return;
        cur ^= 1;
        if (P.hook && iter == 0) {
            // CCv's road-network test (PUSH_ZERO): few zero labels after the
            // first step.  Then the rest of the run is min-id hooking.
            unsigned long long z = 0;
            for (uint64_t v = tid; v < P.n; v += nthreads) z += ldcg((const uint32_t *)P.a + v) == 0;
            z = dev::block_sum<unsigned long long, kPB>(z);
            if (threadIdx.x == 0 && z) atomicAdd(&st->zeros, z);
            if (!grid_barrier(st, P.timeout_ns)) return;
            // (the count includes vertex 0 and its neighbours, CCv's initial_zeros)
            const bool road = ldcg(&st->zeros) * 10 < (unsigned long long)P.n;
            if (road || P.hook == 2) {
                if (road) phase_hook(P);
                else phase_hook_rest(P);
                if (!grid_barrier(st, P.timeout_ns)) return;
                phase_hook_finish(P);
                if (blockIdx.x == 0 && threadIdx.x == 0) {
                    ++iter;
                    if (iter < GG_MAX_ITERS) {
                        st->variant[iter] = GG_VAR_HOOK;
                        st->nactv[iter] = P.n;
                        st->nacte[iter] = P.m;
                        st->scanned[iter] = P.m;
                        st->t_ns[iter + 1] = globaltimer();
                    }
                    st->iterations = iter + 1;
                    st->t_end = globaltimer();
                }
                return;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->iterations = iter;
        st->t_end = globaltimer();
    }
}

__global__ void k_traverse_init(PFront F, uint32_t root, const uint64_t *off, uint32_t smax, uint32_t mmax,
                                int single) {
    if (single) {
        const uint64_t deg = off[root + 1] - off[root];
        const int b = deg <= smax ? 0 : (deg <= mmax ? 1 : 2);
        F.bins[b][0] = root;
        F.cnt[FC_BIN0 + b] = 1;
        F.cnt[FC_NACTV] = 1;
        F.cnt[FC_NACTE] = deg;
        F.bitmap[root >> 5] |= 1u << (root & 31);
    }
}

// Initial frontier from a list of distinct roots (multi-root traversals).
__global__ void k_traverse_init_list(PFront F, const uint32_t *roots, uint32_t k, const uint64_t *off, uint32_t smax,
                                     uint32_t mmax) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint32_t r = roots[i];
        const uint64_t deg = off[r + 1] - off[r];
        const int b = deg <= smax ? 0 : (deg <= mmax ? 1 : 2);
        const unsigned long long slot = atomicAdd(&F.cnt[FC_BIN0 + b], 1ull);
        F.bins[b][slot] = r;
        atomicAdd(&F.cnt[FC_NACTV], 1ull);
        atomicAdd(&F.cnt[FC_NACTE], (unsigned long long)deg);
        atomicOr(&F.bitmap[r >> 5], 1u << (r & 31));
    }
}

// ---- small frontiers: one thread-block cluster, the frontier in shared memory --
// A BFS-levels run whose frontier is small (a high-diameter graph: thousands
// of levels of a few thousand vertices) pays, per level of the cooperative
// kernel, two grid barriers and a dozen dependent global round trips.  Here
// one cluster of kSmallCtas CTAs (1024 threads each, on kSmallCtas SMs) runs
// those levels with the cluster barrier: each CTA keeps the frontier
// vertices it discovered (vertex, first edge, degree) in its own shared
// memory and expands them in the next level, each warp walking its 32 rows'
// edges as one flattened list; the level's totals are read from the other
// CTAs' shared memory (distributed shared memory) after the barrier, so
// every CTA takes the same decisions.  A level costs the adjacency load, the
// level test and atomicMin, and the new vertex's offsets.  The run leaves
// the cluster when the frontier outgrows a CTA's queue, kSmallExitE edges or
// the threshold's push choice (it is then written back as the binned list +
// bitmap the cooperative kernel expects) or when it empties.
constexpr int kSB = 1024;
constexpr int kSmallCtas = 8;
constexpr uint32_t kSmallCap = 4096;  // queue entries per CTA
constexpr unsigned long long kSmallExitE = 262144;
constexpr size_t kSmallSmem = (size_t)2 * kSmallCap * (8 + 4 + 4);

struct SmallArgs {
    const uint64_t *off;
    const uint32_t *adj;
    int32_t *level;
    PFront fr[2];
    PState *st;
    int max_iters;
    uint32_t smax, mmax;
    uint64_t m;
    int threshold, threshold_k;
};

// The threshold's push/pull choice (choose_variant's formulas; the learned
// policy falls back to the default threshold here: it only ever overrides
// it with a predicted gain, and a frontier this small is pushed).
__device__ __forceinline__ bool small_pushes(const SmallArgs &S, unsigned long long v, unsigned long long e) {
    switch (S.threshold) {
    case GG_THRESH_ALWAYS_SPARSE: return true;
    case GG_THRESH_ALWAYS_DENSE: return false;
    case GG_THRESH_FRAC: return (float)(v + e) <= (float)S.m / (float)(100.0 / (float)S.threshold_k);
    default: return (v + e) <= S.m / 20;
    }
}

// Global frontier O: append v (out-degree dg) to its degree bin and bitmap.
__device__ __forceinline__ void small_to_global(const SmallArgs &S, const PFront &O, uint32_t v, uint32_t dg) {
    const uint32_t bin = dg <= S.smax ? 0u : (dg <= S.mmax ? 1u : 2u);
    const unsigned long long pos = atomicAdd(O.cnt + FC_BIN0 + bin, 1ull);
    O.bins[bin][pos] = v;
    atomicOr(O.bitmap + (v >> 5), 1u << (v & 31));
}

// Appends the warp's recorded vertices to this CTA's queue (count *qn,
// out-degree sum *qe); entries beyond kSmallCap go to the global frontier O.
__device__ __forceinline__ void small_append(const SmallArgs &S, const PFront &O, bool rec, uint32_t d,
                                             uint64_t b, uint32_t dg, uint32_t *qv, uint64_t *qb, uint32_t *qd,
                                             unsigned *qn, unsigned long long *qe, int *over) {
    if (!rec) dg = 0;
    const unsigned mk = __ballot_sync(0xffffffffu, rec);
    if (mk == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(mk) - 1;
    const unsigned long long esum = dev::warp_sum((unsigned long long)dg);
    unsigned base = 0;
    if ((int)lane == leader) {
        base = atomicAdd(qn, (unsigned)__popc(mk));
        atomicAdd(qe, esum);
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!rec) return;
    const unsigned slot = base + __popc(mk & ((1u << lane) - 1u));
    if (slot < kSmallCap) {
        qv[slot] = d;
        qb[slot] = b;
        qd[slot] = dg;
    } else {
        small_to_global(S, O, d, dg);
        *over = 1;
    }
}

__global__ void __cluster_dims__(kSmallCtas, 1, 1) __launch_bounds__(kSB, 1) k_small_bfs(SmallArgs S) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    // queue k (0 / 1): first edges, vertices, degrees
    auto qb = [&](int k) { return (uint64_t *)small_smem + (size_t)k * kSmallCap; };
    auto qv = [&](int k) { return (uint32_t *)(small_smem + 16 * (size_t)kSmallCap) + (size_t)k * kSmallCap; };
    auto qd = [&](int k) { return (uint32_t *)(small_smem + 24 * (size_t)kSmallCap) + (size_t)k * kSmallCap; };
    __shared__ unsigned s_n[2];
    __shared__ unsigned long long s_e[2];
    __shared__ int s_over[2];
    __shared__ unsigned s_bin[NBINS], s_pos[NBINS];
    __shared__ unsigned long long s_base[NBINS];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    PState *st = S.st;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    auto fr = [&](int k) { return k ? S.fr[1] : S.fr[0]; };  // no dynamic index into the parameters
    int cur = st->small_cur;
    int iter = st->small_iter;
    if (tid == 0) {
        s_n[0] = s_n[1] = 0;
        s_e[0] = s_e[1] = 0;
        s_over[0] = s_over[1] = 0;
    }
    __syncthreads();
    // the frontier left by the cooperative kernel, dealt round-robin to the
    // CTAs; its bitmap words and counters are cleared (it becomes an output)
    {
        const PFront F = fr(cur);
        const unsigned long long c0 = F.cnt[FC_BIN0], c1 = F.cnt[FC_BIN1], c2 = F.cnt[FC_BIN2];
        const unsigned total = (unsigned)(c0 + c1 + c2);  // <= kSmallEnterV <= kSmallCtas * kSmallCap
        for (unsigned i = rank + kSmallCtas * tid; i < total; i += kSmallCtas * kSB) {
            const uint32_t v = i < c0 ? F.bins[0][i] : (i < c0 + c1 ? F.bins[1][i - c0] : F.bins[2][i - c0 - c1]);
            const uint64_t b = S.off[v];
            const uint32_t dg = (uint32_t)(S.off[v + 1] - b);
            const unsigned slot = atomicAdd(&s_n[0], 1u);
            atomicAdd(&s_e[0], (unsigned long long)dg);
            qv(0)[slot] = v;
            qb(0)[slot] = b;
            qd(0)[slot] = dg;
            F.bitmap[v >> 5] = 0u;  // every set bit of this bitmap is a frontier vertex
        }
        cl.sync();
        if (rank == 0 && tid < FC_WORDS) F.cnt[tid] = 0;
    }
    int q = 0;
    bool first = true;
    while (true) {
        // this level's totals over the cluster (every CTA reads the same)
        // lane r < kSmallCtas of every warp reads CTA r's counts; shuffles
        // give each lane the totals and its exclusive prefix
        unsigned nr = 0;
        unsigned long long er = 0;
        int ovr = 0;
        if (lane < kSmallCtas) {
            nr = *cl.map_shared_rank(&s_n[q], lane);
            er = *cl.map_shared_rank(&s_e[q], lane);
            ovr = *cl.map_shared_rank(&s_over[q], lane);
        }
        const unsigned long long tot_n = dev::warp_sum((unsigned long long)nr);
        const unsigned long long tot_e = dev::warp_sum(er);
        const int over = __any_sync(0xffffffffu, ovr != 0);
        unsigned incl = min(nr, kSmallCap);  // prefix of the CTAs' queue lengths
#pragma unroll
        for (int o = 1; o < kSmallCtas; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += t;
        }
        const unsigned n_all = __shfl_sync(0xffffffffu, incl, kSmallCtas - 1);
        const unsigned excl = incl - min(nr, kSmallCap);  // lane r: first row of CTA r
        if (tot_n == 0 || iter >= S.max_iters) {
            if (rank == 0 && tid == 0) {
                st->iterations = iter;
                st->small_done = 1;
                st->exit_small = 0;
                st->t_end = globaltimer();
            }
            cl.sync();  // no CTA leaves while another may still read its counts
            return;
        }
        if (!first && (over || tot_e > kSmallExitE || !small_pushes(S, tot_n, tot_e))) {  // uniform
            // back to the cooperative kernel: every CTA's queue (entries past
            // its cap are there already) becomes fr[cur]'s list and bitmap
            const PFront Fo = fr(cur);
            const unsigned inq = min(s_n[q], kSmallCap);
            if (tid < NBINS) s_bin[tid] = s_pos[tid] = 0;
            __syncthreads();
            for (unsigned i = tid; i < inq; i += kSB) {
                const uint32_t dg = qd(q)[i];
                atomicAdd(&s_bin[dg <= S.smax ? 0 : (dg <= S.mmax ? 1 : 2)], 1u);
            }
            __syncthreads();
            if (tid < NBINS) s_base[tid] = atomicAdd(Fo.cnt + FC_BIN0 + tid, (unsigned long long)s_bin[tid]);
            __syncthreads();
            for (unsigned i = tid; i < inq; i += kSB) {
                const uint32_t v = qv(q)[i], dg = qd(q)[i];
                const uint32_t bin = dg <= S.smax ? 0 : (dg <= S.mmax ? 1 : 2);
                Fo.bins[bin][s_base[bin] + atomicAdd(&s_pos[bin], 1u)] = v;
                atomicOr(Fo.bitmap + (v >> 5), 1u << (v & 31));
            }
            if (rank == 0 && tid == 0) {
                Fo.cnt[FC_NACTV] = tot_n;
                Fo.cnt[FC_NACTE] = tot_e;
                st->has_list[cur] = 1;
                st->has_list[cur ^ 1] = 0;
                st->all[0] = st->all[1] = 0;
                st->cand_valid = 0;
                st->small_iter = iter;
                st->small_cur = cur;
                st->small_done = 0;
                st->exit_small = 0;
                st->iterations = iter;
            }
            cl.sync();
            return;
        }
        first = false;
        const PFront O = fr(cur ^ 1);
        if (rank == 0 && tid == 0) {
            if (iter < GG_MAX_ITERS) {
                st->variant[iter] = GG_VAR_PUSH_SPARSE;
                st->nactv[iter] = tot_n;
                st->nacte[iter] = tot_e;
                st->scanned[iter] = tot_e;
            }
            st->reached_v += tot_n;
            st->reached_e += tot_e;
        }
        // the other queue's counters: read by the other CTAs last level,
        // before the barrier that ended it
        if (tid == 0) {
            s_n[q ^ 1] = 0;
            s_e[q ^ 1] = 0;
            s_over[q ^ 1] = 0;
        }
        __syncthreads();
        const int32_t fk = iter + 1;
        // the level's rows are the concatenation of all CTAs' queues, dealt
        // to the cluster's warps in groups of 32 (a CTA's discoveries stay
        // in its queue, so without this one CTA would expand a frontier that
        // grew from one root); other CTAs' entries are read through
        // distributed shared memory
        // (group g of 32 rows goes to CTA g mod kSmallCtas: a level of a few
        // thousand rows then spreads over every SM's load/store units)
        for (unsigned base = (wid * kSmallCtas + rank) * 32; base < n_all; base += kSmallCtas * kSB) {
            const unsigned i = base + lane;
            const bool have = i < n_all;
            unsigned r = 0;  // the CTA holding row i: last r whose first row <= i
#pragma unroll
            for (unsigned k = 1; k < kSmallCtas; ++k) r += __shfl_sync(0xffffffffu, excl, k) <= i;
            const unsigned first_r = __shfl_sync(0xffffffffu, excl, r);
            uint64_t b = 0;
            uint32_t dg = 0;
            if (have) {
                const unsigned li = i - first_r;
                b = cl.map_shared_rank(qb(q), r)[li];
                dg = cl.map_shared_rank(qd(q), r)[li];
            }
            // the 32 rows' edges as one list, 4 per lane in flight; a target's
            // offsets are loaded beside its atomicMin (needed only if it is
            // new, but then without another round trip)
            uint32_t incl_e = dg;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl_e, o);
                if (lane >= (uint32_t)o) incl_e += t;
            }
            const uint32_t tot = __shfl_sync(0xffffffffu, incl_e, 31), ex = incl_e - dg;
            for (uint32_t e0 = 0; e0 < tot; e0 += 128) {  // warp-uniform
                uint32_t dd[4];
                bool ok[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t idx = e0 + (uint32_t)u * 32u + lane;
                    uint32_t rr = 0;
#pragma unroll
                    for (uint32_t step = 16; step; step >>= 1)
                        if (__shfl_sync(0xffffffffu, ex, rr + step) <= idx) rr += step;
                    const uint64_t rb = __shfl_sync(0xffffffffu, b, rr);
                    const uint32_t rx = __shfl_sync(0xffffffffu, ex, rr);
                    ok[u] = idx < tot;
                    dd[u] = ok[u] ? __ldg(S.adj + rb + (idx - rx)) : 0u;
                }
                int32_t old[4];
                uint64_t ob[4], oe[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    old[u] = ok[u] ? atomicMin(S.level + dd[u], fk) : fk;
                    ob[u] = ok[u] ? __ldg(S.off + dd[u]) : 0;
                    oe[u] = ok[u] ? __ldg(S.off + dd[u] + 1) : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (e0 + (uint32_t)u * 32u >= tot) break;  // warp-uniform
                    small_append(S, O, old[u] > fk, dd[u], ob[u], (uint32_t)(oe[u] - ob[u]), qv(q ^ 1), qb(q ^ 1),
                                 qd(q ^ 1), &s_n[q ^ 1], &s_e[q ^ 1], &s_over[q ^ 1]);
                }
            }
        }
        cl.sync();  // the level's appends and counts are complete in every CTA
        ++iter;
        cur ^= 1;
        q ^= 1;
        if (rank == 0 && tid == 0 && iter <= GG_MAX_ITERS) st->t_ns[iter] = globaltimer();
    }
}

// Host side -----------------------------------------------------------------
template <int R>
static const void *traverse_kernel() { return (const void *)k_traverse<R>; }

const void *selector_weights(gg_graph *g);

// The run's state starts from a device-side write (no host memory is read
// when the stream runs, so the enqueue below can be captured in a graph).
__global__ void k_state_init(PState *st, PFront f0, int all, int has_list, unsigned long long n,
                             unsigned long long m) {
    if (all) {
        st->all[0] = 1;
        f0.cnt[FC_NACTV] = n;
        f0.cnt[FC_NACTE] = m;
    }
    if (has_list) st->has_list[0] = 1;
}

// Enqueues a device-driven run on the context's stream: buffers, the initial
// frontier and state, and the cooperative launch; nothing waits on the host.
// With a resumed run the state is copied from host values (not capture-safe).
gg_status persistent_enqueue(gg_graph *g, const gg_emap_desc &d, int level_k, bool start_all, uint32_t root,
                             const gg_run_opts &opt, int force_iter, int force_variant, const uint32_t *d_roots,
                             uint32_t nroots, const PersistResume *resume, void *state, PArgs &P,
                             const void **kfn_out, unsigned *grid_out, void *merge_scratch = nullptr) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    const Tuning &t = tuning();
    // buffers: the graph's two scratch frontiers, candidate lists, state block
    for (auto &f : g->tmp_front)
        if (!f) GG_CHECK(gg_frontier_create(g, &f));
    for (auto *f : g->tmp_front) {
        GG_CHECK(frontier_alloc_bins(f));
        GG_CHECK(frontier_alloc_bitmap(f));
    }
    CandLists &c = g->cand;
    if (!c.list[0]) {
        for (auto &l : c.list) GG_CUDA(ctx, cudaMalloc(&l, ((size_t)g->n + 1) * 4));
        GG_CUDA(ctx, cudaMalloc(&c.cnt, 2 * sizeof(uint64_t)));
    }
    PState *st = (PState *)state;
    const size_t words = ((size_t)g->n + 31) / 32 + 1;
    std::memset(&P, 0, sizeof(P));
    P.off = g->off;
    P.adj = g->adj;
    P.in_off = g->in_off;
    P.in_adj = g->in_adj;
    P.n = g->n;
    P.m = g->m;
    for (int i = 0; i < 2; ++i) {
        // a resumed run starts from the scratch frontier it was left in
        gg_frontier *f = g->tmp_front[resume ? (i ^ resume->cur) : i];
        for (int b = 0; b < NBINS; ++b) P.fr[i].bins[b] = f->bins[b];
        P.fr[i].bitmap = f->bitmap;
        P.fr[i].cnt = (unsigned long long *)f->d_cnt;
        if (!resume) {
            GG_CUDA(ctx, cudaMemsetAsync(f->bitmap, 0, words * 4, s));
            GG_CUDA(ctx, cudaMemsetAsync(f->d_cnt, 0, FC_WORDS * 8, s));
        }
        f->host_valid = false;
        f->has_list = f->has_bitmap = f->all = false;
    }
    P.iter0 = resume ? resume->iter0 : 0;
    P.cur0 = 0;
    // small frontiers after the iterations that mark a high-diameter run
    // (a low-diameter one alternates between small and large frontiers,
    // and each switch costs a host round trip)
    P.small_from = std::max(P.iter0, t.graph_handoff > 0 ? t.graph_handoff : 32);
    P.cand[0] = c.list[0];
    P.cand[1] = c.list[1];
    P.nonisolated = g->nonisolated;
    P.nonisolated_n = (const unsigned long long *)g->nonisolated_n;
    P.a = d.a->d;
    P.prev = d.prev ? d.prev->d : nullptr;
    P.relax = d.relax;
    P.record = d.record;
    P.filter = d.dst_filter;
    P.level_k = level_k;
    P.level_sync = (d.src_level_sync && d.dst_filter == GG_FILTER_GT_CONST) ? 1 : 0;
    P.fk = d.dst_filter_k;
    P.threshold = opt.threshold;
    P.threshold_k = opt.threshold_k;
    P.variant = opt.variant;
    P.smax = t.bin_small_max;
    P.mmax = t.bin_medium_max;
    P.large_ch = t.large_chunk;
    P.K = t.pull_k;
    P.max_iters = (int)std::min<uint64_t>((uint64_t)g->n + 2, (uint64_t)INT_MAX / 2);
    P.timeout_ns = t.barrier_timeout_ns;
    P.st = st;
    P.force_iter = force_iter >= 0 ? force_iter : g->force_iter;
    P.force_variant = force_iter >= 0 ? force_variant : g->force_variant;
    P.sel_w = (const __nv_bfloat16 *)selector_weights(g);
    // CC of a symmetric graph: road-network test after step 0, then hooking
    P.hook = (t.cc_hook && d.relax == GG_RELAX_MIN_U32 && d.dst_filter == GG_FILTER_NE_ZERO && g->symmetric &&
              start_all && force_iter < 0 && g->force_iter < 0 && g->n > 0) ? t.cc_hook : 0;
    P.rows_sorted = g->rows_sorted ? 1 : 0;
    // fused sparse pushes (CC): the queue holds up to 2n + 64Ki entries, more spill
    P.fusion = (t.fusion & 4) && d.relax == GG_RELAX_MIN_U32 && d.dst_filter == GG_FILTER_NE_ZERO;
    if (P.fusion) {
        const size_t cap = t.fusion_queue ? (size_t)t.fusion_queue : 2 * (size_t)g->n + 65536;
        if (g->wq_cap != cap) {
            cudaFree(g->wq);
            g->wq = nullptr;
            g->wq_cap = 0;
            GG_CUDA(ctx, cudaMalloc(&g->wq, cap * 4));
            g->wq_cap = cap;
        }
        GG_CUDA(ctx, cudaMemsetAsync(g->wq, 0xFF, g->wq_cap * 4, s));
        P.wq = g->wq;
        P.wq_cap = g->wq_cap;
    }
    // (not for multi-root runs: a batch of graphs stays one launch)
    P.small_ok = t.small_frontier && d.relax == GG_RELAX_MIN_PLUS1_I32 && P.level_sync && level_k &&
                 d.record == GG_RECORD_NE_PREV && P.force_iter < 0 && !start_all && !d_roots &&
                 (opt.variant == GG_VAR_AUTO || opt.variant == GG_VAR_PUSH_SPARSE);
    P.gini = g->gini < 0 ? 0.0f : g->gini;
    if (opt.threshold == GG_THRESH_LEARNED && P.sel_w && g->gini < 0) {
        float gi;
        GG_CHECK(graph_gini(g, &gi));
        P.gini = gi;
    }
    GG_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(PState), s));
    if (resume) {
        const int hl = resume->has_list ? 1 : 0;
        const unsigned long long rc[2] = {resume->reached_v, resume->reached_e};
        GG_CUDA(ctx, cudaMemcpyAsync(&st->has_list[0], &hl, sizeof(int), cudaMemcpyHostToDevice, s));
        GG_CUDA(ctx, cudaMemcpyAsync(&st->reached_v, rc, sizeof(rc), cudaMemcpyHostToDevice, s));
    } else if (start_all) {
        // the all-true frontier: n vertices, m edges
        k_state_init<<<1, 1, 0, s>>>(st, P.fr[0], 1, 0, g->n, g->m);
        GG_LAUNCHED(ctx);
    } else {
        if (d_roots) {
            if (nroots)
                k_traverse_init_list<<<(nroots + 255) / 256, 256, 0, s>>>(P.fr[0], d_roots, nroots, g->off, P.smax,
                                                                          P.mmax);
        } else {
            k_traverse_init<<<1, 1, 0, s>>>(P.fr[0], root, g->off, P.smax, P.mmax, 1);
        }
        GG_LAUNCHED(ctx);
        k_state_init<<<1, 1, 0, s>>>(st, P.fr[0], 0, 1, 0, 0);
        GG_LAUNCHED(ctx);
    }
    const void *kfn = d.relax == GG_RELAX_MIN_PLUS1_I32 ? traverse_kernel<GG_RELAX_MIN_PLUS1_I32>()
                    : d.relax == GG_RELAX_MIN_U32      ? traverse_kernel<GG_RELAX_MIN_U32>()
                                                        : traverse_kernel<GG_RELAX_SETIF_U32>();
    const int per_sm = resident_ctas(kfn, kPB);
    unsigned grid = (unsigned)(ctx->sm_count * per_sm);
    if (resume && t.handoff_ctas > 0) grid = std::min(grid, (unsigned)t.handoff_ctas);
    // merge-path scratch: one count per list entry (<= n) + one per CTA
    void *mp = merge_scratch;
    if (!mp) GG_CHECK(graph_scratch(g, ((size_t)g->n + grid + 1) * 8, &mp));
    P.merge = (unsigned long long *)mp;
    void *args[] = {&P};
    GG_CUDA(ctx, cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kPB), args, 0, s));
    ctx->launches++;
    if (kfn_out) *kfn_out = kfn;
    if (grid_out) *grid_out = grid;
    return GG_OK;
}

// The records of a finished run from its state block (read to the host).
static void persistent_collect(gg_graph *g, const PArgs &P, const PState &hs, gg_run_stats *stats, int *iters_out) {
    *iters_out = hs.iterations;
    g->force_rec.seen = P.force_iter >= 0 && P.force_iter < INT_MAX && hs.f_seen && hs.f_t1 >= hs.f_t0;
    if (g->force_rec.seen) {
        g->force_rec.iter_ms = (double)(hs.f_t1 - hs.f_t0) * 1e-6;
        g->force_rec.rest_ms = (double)(hs.t_end - hs.f_t0) * 1e-6;
        g->force_rec.nactv = (double)hs.f_nactv;
        g->force_rec.nacte = (double)hs.f_nacte;
        g->force_rec.reached = (double)hs.f_reached;
    }
    if (stats) {
        stats->vertices_reached = hs.reached_v;
        stats->edges_reached = hs.reached_e;
        const int k = std::min(hs.iterations, GG_MAX_ITERS);
        for (int i = 0; i < k; ++i) {
            stats->variant[i] = hs.variant[i];
            stats->nactv[i] = hs.nactv[i];
            stats->nacte[i] = hs.nacte[i];
            stats->scanned[i] = hs.scanned[i];
            stats->iter_ms[i] = (double)(hs.t_ns[i + 1] - hs.t_ns[i]) * 1e-6;
            stats->kernel_ms[i] = stats->iter_ms[i];
            stats->scanned_edges += hs.scanned[i];
        }
    }
}

gg_status persistent_state_read(gg_graph *g, void *state, const PArgs &P, gg_run_stats *stats, int *iters_out) {
    gg_ctx *ctx = g->ctx;
    PState hs;
    GG_CUDA(ctx, cudaMemcpyAsync(&hs, state, sizeof(PState), cudaMemcpyDeviceToHost, ctx->stream));
    GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs.err & DEV_ERR_TIMEOUT) return set_error(ctx, GG_ERR_TIMEOUT, "traversal grid barrier timed out");
    if (hs.err) return set_error(ctx, GG_ERR_STATE, "traversal device error");
    persistent_collect(g, P, hs, stats, iters_out);
    return GG_OK;
}

gg_status persistent_traverse(gg_graph *g, const gg_emap_desc &d, int level_k, bool start_all, uint32_t root,
                              const gg_run_opts &opt, gg_run_stats *stats, int *iters_out, int force_iter,
                              int force_variant, const uint32_t *d_roots, uint32_t nroots,
                              const PersistResume *resume) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    if (!g->pstate) GG_CUDA(ctx, cudaMalloc(&g->pstate, sizeof(PState)));
    PState *st = (PState *)g->pstate;
    PArgs P;
    const void *kfn = nullptr;
    unsigned grid = 0;
    GG_CHECK(persistent_enqueue(g, d, level_k, start_all, root, opt, force_iter, force_variant, d_roots, nroots,
                                resume, st, P, &kfn, &grid));
    void *args[] = {&P};
    PState hs;
    GG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(PState), cudaMemcpyDeviceToHost, s));
    GG_CUDA(ctx, cudaStreamSynchronize(s));
    if (hs.err & DEV_ERR_TIMEOUT) return set_error(ctx, GG_ERR_TIMEOUT, "traversal grid barrier timed out");
    if (hs.err) return set_error(ctx, GG_ERR_STATE, "traversal device error");
    // small frontiers: the cluster kernel, then back to the cooperative one
    // whenever the frontier outgrows it (records accumulate in the state block)
    while (P.small_ok && hs.exit_small) {
        // shared memory above 48 KiB is opt-in (set on the current device)
        GG_CUDA(ctx, cudaFuncSetAttribute(k_small_bfs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem));
        SmallArgs S;
        S.off = g->off;
        S.adj = g->adj;
        S.level = (int32_t *)P.a;
        S.fr[0] = P.fr[0];
        S.fr[1] = P.fr[1];
        S.st = st;
        S.max_iters = P.max_iters;
        S.smax = P.smax;
        S.mmax = P.mmax;
        S.m = P.m;
        S.threshold = P.threshold;
        S.threshold_k = P.threshold_k;
        k_small_bfs<<<kSmallCtas, kSB, kSmallSmem, s>>>(S);
        GG_LAUNCHED(ctx);
        GG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(PState), cudaMemcpyDeviceToHost, s));
        GG_CUDA(ctx, cudaStreamSynchronize(s));
        if (hs.small_done) break;
        P.iter0 = hs.small_iter;
        P.cur0 = hs.small_cur;
        P.small_from = P.iter0 + 1;  // at least one cooperative step before the next hand-over
        GG_CUDA(ctx, cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kPB), args, 0, s));
        ctx->launches++;
        GG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(PState), cudaMemcpyDeviceToHost, s));
        GG_CUDA(ctx, cudaStreamSynchronize(s));
        if (hs.err & DEV_ERR_TIMEOUT) return set_error(ctx, GG_ERR_TIMEOUT, "traversal grid barrier timed out");
        if (hs.err) return set_error(ctx, GG_ERR_STATE, "traversal device error");
    }
    persistent_collect(g, P, hs, stats, iters_out);
    // the final frontier is empty; no host state to keep
    return GG_OK;
}

// Device time between construction and stop_record() (CUDA events on the
// context's stream, recorded outside any capture).
struct RunTimerP {
    gg_ctx *ctx;
    explicit RunTimerP(gg_ctx *c) : ctx(c) { cudaEventRecord(ctx->ev0, ctx->stream); }
    void stop_record() { cudaEventRecord(ctx->ev1, ctx->stream); }
    double elapsed() {
        cudaEventSynchronize(ctx->ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        return ms;
    }
};

// BFS levels from many roots and CC labels of one graph (the disjoint union
// of many small graphs: every part's BFS from its first vertex and its
// components), submitted as ONE CUDA graph launch: the BFS start, the
// multi-root device-driven BFS, the CC start (PRESET_ZERO) and the
// device-driven CC, captured on the context's stream.  The graph is captured
// per call (every buffer it names is fixed for the call) and released after
// it; the host waits once.  A capture the runtime refuses leaves the same
// launches on the stream, one after the other.
gg_status batch_bfs_cc(gg_graph *g, const uint32_t *roots, uint32_t k, gg_prop *level, gg_prop *label,
                       gg_run_stats *bfs_st, gg_run_stats *cc_st, int *graph_launches, uint64_t *kernel_nodes) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t s = ctx->stream;
    std::vector<uint32_t> r(roots, roots + k);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    if (!r.empty() && r.back() >= g->n) return set_error(ctx, GG_ERR_ARG, "gg_batch_bfs_cc: root out of range");
    if (!level) GG_CHECK(run_tmp_prop(g, 0, GG_I32, &level));
    if (!label) GG_CHECK(run_tmp_prop(g, 2, GG_U32, &label));
    gg_prop *prev1, *prev2;
    GG_CHECK(run_tmp_prop(g, 1, GG_I32, &prev1));
    GG_CHECK(run_tmp_prop(g, 3, GG_U32, &prev2));
    // every buffer the captured launches name exists before the capture
    for (auto &f : g->tmp_front)
        if (!f) GG_CHECK(gg_frontier_create(g, &f));
    for (auto *f : g->tmp_front) {
        GG_CHECK(frontier_alloc_bins(f));
        GG_CHECK(frontier_alloc_bitmap(f));
    }
    CandLists &c = g->cand;
    if (!c.list[0]) {
        for (auto &l : c.list) GG_CUDA(ctx, cudaMalloc(&l, ((size_t)g->n + 1) * 4));
        GG_CUDA(ctx, cudaMalloc(&c.cnt, 2 * sizeof(uint64_t)));
    }
    if (!g->pstate) GG_CUDA(ctx, cudaMalloc(&g->pstate, sizeof(PState)));
    if (!g->pstate2) GG_CUDA(ctx, cudaMalloc(&g->pstate2, sizeof(PState)));
    void *merge;
    GG_CHECK(graph_scratch(g, ((size_t)g->n + (size_t)ctx->sm_count * 32 + 1) * 8, &merge));
    uint32_t *d_roots = nullptr;
    GG_CUDA(ctx, cudaMalloc(&d_roots, (r.size() + 1) * 4));
    if (!r.empty()) GG_CUDA(ctx, cudaMemcpyAsync(d_roots, r.data(), r.size() * 4, cudaMemcpyHostToDevice, s));
    GG_CUDA(ctx, cudaStreamSynchronize(s));
    gg_run_opts opt_b, opt_c;
    std::memset(&opt_b, 0, sizeof(opt_b));
    opt_b.threshold = GG_THRESH_DEFAULT;
    opt_b.variant = GG_VAR_AUTO;
    opt_c = opt_b;
    opt_c.threshold = GG_THRESH_FRAC;  // CCv.C:309 emap_step(F, 5)
    opt_c.threshold_k = 5;
    gg_emap_desc db, dc;
    std::memset(&db, 0, sizeof(db));
    db.relax = GG_RELAX_MIN_PLUS1_I32;
    db.a = level;
    db.dst_filter = GG_FILTER_GT_CONST;
    db.src_level_sync = 1;
    db.record = GG_RECORD_NE_PREV;
    db.prev = prev1;
    db.threshold = opt_b.threshold;
    db.variant = GG_VAR_AUTO;
    std::memset(&dc, 0, sizeof(dc));
    dc.relax = GG_RELAX_MIN_U32;
    dc.a = label;
    dc.dst_filter = GG_FILTER_NE_ZERO;
    dc.record = GG_RECORD_NE_PREV;
    dc.prev = prev2;
    dc.threshold = opt_c.threshold;
    dc.threshold_k = opt_c.threshold_k;
    dc.variant = GG_VAR_AUTO;
    PArgs P1, P2;
    auto enqueue_all = [&]() -> gg_status {
        GG_CHECK(enqueue_bfs_start(g, level, prev1, d_roots, (uint32_t)r.size()));
        GG_CHECK(persistent_enqueue(g, db, 1, false, 0, opt_b, -1, -1, d_roots, (uint32_t)r.size(), nullptr,
                                    g->pstate, P1, nullptr, nullptr, merge));
        GG_CHECK(enqueue_cc_start(g, label, prev2));
        GG_CHECK(persistent_enqueue(g, dc, 0, true, 0, opt_c, -1, -1, nullptr, 0, nullptr, g->pstate2, P2, nullptr,
                                    nullptr, merge));
        return GG_OK;
    };
    RunTimerP tm(ctx);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const uint64_t l0 = ctx->launches;
    gg_status st = GG_OK;
    bool captured = false;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        st = enqueue_all();
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st == GG_OK && e == cudaSuccess && graph &&
            cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess && cudaGraphLaunch(exec, s) == cudaSuccess)
            captured = true;
        cudaGetLastError();  // a refused capture leaves no sticky error
    }
    if (kernel_nodes) *kernel_nodes = ctx->launches - l0;
    if (!captured) {
        // the same launches, one after the other
        ctx->launches = l0;
        st = enqueue_all();
    } else {
        ctx->launches = l0 + 1;
    }
    if (graph_launches) *graph_launches = captured ? 1 : 0;
    tm.stop_record();
    int it1 = 0, it2 = 0;
    if (st == GG_OK) st = persistent_state_read(g, g->pstate, P1, bfs_st, &it1);
    if (st == GG_OK) st = persistent_state_read(g, g->pstate2, P2, cc_st, &it2);
    const double ms = tm.elapsed();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_roots);
    GG_CHECK(st);
    if (bfs_st) {
        bfs_st->iterations = it1;
        bfs_st->total_ms = ms;
        bfs_st->kernels = captured ? 1 : ctx->launches - l0;
    }
    if (cc_st) {
        cc_st->iterations = it2;
        cc_st->total_ms = ms;
        cc_st->kernels = 0;
    }
    return GG_OK;
}

}  // namespace gg

extern "C" gg_status gg_batch_bfs_cc(gg_graph *g, const uint32_t *roots, uint32_t k, gg_prop *level,
                                     gg_prop *label, int32_t *host_level, uint32_t *host_label,
                                     gg_run_stats *bfs_stats, gg_run_stats *cc_stats, int *graph_launches,
                                     uint64_t *kernel_launches) {
    using namespace gg;
    if (!g || (k && !roots)) return GG_ERR_ARG;
    if (level && (level->g != g || level->t != GG_I32)) return set_error(g->ctx, GG_ERR_ARG, "level must be an I32 property of g");
    if (label && (label->g != g || label->t != GG_U32)) return set_error(g->ctx, GG_ERR_ARG, "label must be a U32 property of g");
    if (bfs_stats) std::memset(bfs_stats, 0, sizeof(*bfs_stats));
    if (cc_stats) std::memset(cc_stats, 0, sizeof(*cc_stats));
    if (g->n == 0) return GG_OK;
    GG_CHECK(batch_bfs_cc(g, roots, k, level, label, bfs_stats, cc_stats, graph_launches, kernel_launches));
    if (host_level) {
        gg_prop *lv = level;
        if (!lv) GG_CHECK(run_tmp_prop(g, 0, GG_I32, &lv));
        GG_CHECK(gg_prop_download(lv, host_level));
    }
    if (host_label) {
        gg_prop *lb = label;
        if (!lb) GG_CHECK(run_tmp_prop(g, 2, GG_U32, &lb));
        GG_CHECK(gg_prop_download(lb, host_label));
    }
    return GG_OK;
}
