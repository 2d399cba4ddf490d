// gg_emap.cu -- edgemap traversal kernels, the variant dispatcher, and the
// BFS-level / BFS-parent / connected-components drivers.
//
// Reference behaviour (include/graptor/api.h:2143-2415): one edgemap call
// evaluates relax(s,d) over the edges leaving the active (src-filtered)
// vertices into dst-filtered vertices and records the output frontier; the
// traversal is chosen per call by the sparse/dense threshold
// (api.h:130-222): sparse => CSR push (dsl/edgemap.h:1397-1740 with
// edge-balanced chunks, dsl/emap/edgechunk.h:315-620), dense => CSC pull with
// per-vertex early exit (dsl/emap/GraptorCSCDataParCached.h:60-302, 348-496).
//
// B200 design
//   * push_sparse : the frontier list is kept in three degree bins (produced
//     directly by the kernel that made the frontier); one launch processes
//     large-degree sources with a CTA each, medium ones with a warp each and
//     small ones with a thread each (warp-uniform loops).
//   * push_merge  : edge-balanced push: degree prefix sum over the frontier,
//     each CTA takes an equal slice of edges and finds its sources by binary
//     search (merge-path partitioning).
//   * pull_dense  : one warp owns 32 consecutive destinations (one frontier
//     bitmap word); each lane first scans up to K in-edges of its own vertex,
//     then the warp cooperatively scans the remaining long rows 32 edges at a
//     time (coalesced), exiting as soon as the dst filter turns false.  The
//     output bitmap word is written with a single store, counts reduced per
//     CTA, and the output list is appended warp-aggregated.
//   * push_dense  : push from a frontier bitmap with the same two-phase warp
//     scheme, for large frontiers whose operator does not early-exit.
// Records: NE_PREV (a[d] != prev[d], then prev[d] = a[d]) is detected without
// a dedup pass: in push the thread whose atomic moved a[d] away from prev[d]
// records d; in pull the owner of d does.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <climits>
#include <cstring>
#include <type_traits>

#include "gg_batch.h"
#include "gg_internal.cuh"
#include "gg_mlp.cuh"

namespace gg {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t kLargeLocal = 1024;  // push: large bins up to this size chunked in shared memory
constexpr int kAppCap = 128;            // push: staged list appends per warp and bin

struct EmapArgs {
    const uint64_t *off;      // CSR (push, out-degree)
    const uint32_t *adj;
    const uint64_t *in_off;   // CSC (pull)
    const uint32_t *in_adj;
    uint32_t n;
    int record;
    // input frontier
    const uint32_t *in_bits;  // bitmap or nullptr (all vertices)
    const uint32_t *in_b0, *in_b1, *in_b2;
    uint32_t c0, c1, c2;
    // output frontier
    uint32_t *out_bits;       // pull: every word written; push: test-and-set dedup (pre-cleared)
    uint32_t *out_b0, *out_b1, *out_b2;
    unsigned long long *out_cnt;
    uint32_t smax, mmax;
    int K;
    const uint64_t *large_first;  // [c2 + 1] chunk prefix of the large bin (push)
    uint32_t large_ch;            // edges per large-bin chunk
    int merge_med;                // push: medium bin chunked with the large one (small frontiers)
    int large_as_med;             // push: large bin walked a warp per row with the medium one
    // pull candidate lists (drivers only): the destinations that can still
    // pass the (monotone) dst filter.  cand == nullptr: scan all vertices.
    const uint32_t *cand;
    const unsigned long long *cand_n;   // device count of cand
    uint32_t *cand_out;                 // vertices still passing after this step
    unsigned long long *cand_out_n;
    const uint64_t *word_prefix;        // full-scan pull: per-word cost prefix
    const uint4 *first_in;              // pull: {first two in-neighbours, in-degree, third} per vertex, or null
    const uint2 *first1;                // pull: {first in-neighbour, in-degree} per vertex, or null
    int rec_n;                          // pull: in-neighbours taken from the record (1 to 3)
    int lazy_off;                       // pull: offsets only for rows the record's edges do not settle
    int fresh;                          // pull: every candidate is unvisited (level not loaded)
    // split pull, first pass: candidates still open after their first two
    // in-edges are appended here for the second pass (graph-driven BFS)
    uint32_t *rest_out;
    unsigned long long *rest_out_n;
    // bitwise-or pulls: rows with more in-edges than this are left to the
    // heavy-row chunk kernels (0: none)
    uint32_t heavy_T;
};

template <int R>
struct Op {
    using V = typename std::conditional<R == GG_RELAX_MIN_PLUS1_I32, int32_t, uint32_t>::type;
    V *a;
    V *prev;
    const V *b;      // OR_U32: the source property (a[d] |= b[s])
    int filter;
    int64_t fk;
    int level_sync;  // MIN_PLUS1: active sources hold fk-1, offer fk without a load

    __device__ __forceinline__ V load(uint32_t v) const { return a[v]; }
    __device__ __forceinline__ static V none() {
        if constexpr (R == GG_RELAX_MIN_PLUS1_I32) return INT_MAX;
        else return 0xFFFFFFFFu;
    }
    __device__ __forceinline__ bool dst_ok(V cur) const {
        switch (filter) {
        case GG_FILTER_GT_CONST: return (int64_t)cur > fk;
        case GG_FILTER_NE_ZERO: return cur != 0;
        case GG_FILTER_MSB_SET: return ((uint32_t)cur >> 31) != 0;
        case GG_FILTER_NE_CONST: return (uint32_t)cur != (uint32_t)fk;
        default: return true;
        }
    }
    // value offered along an edge s->d
    __device__ __forceinline__ V src_val(uint32_t s) const {
        if constexpr (R == GG_RELAX_MIN_PLUS1_I32) return level_sync ? (V)fk : a[s] + 1;
        else if constexpr (R == GG_RELAX_MIN_U32) return a[s];
        else if constexpr (R == GG_RELAX_OR_U32) return b[s];
        else if constexpr (R == GG_RELAX_COUNT_DOWN_U32) return 1u;  // every active source takes one
        else return (V)s;
    }
    __device__ __forceinline__ bool better(V x, V best) const {
        if constexpr (R == GG_RELAX_SETIF_U32) return ((uint32_t)best >> 31) != 0;
        else if constexpr (R == GG_RELAX_OR_U32) return (best | x) != best;
        else if constexpr (R == GG_RELAX_COUNT_DOWN_U32) return (int64_t)best > fk;
        else return x < best;
    }
    // the value after a better offer x
    __device__ __forceinline__ V combine(V best, V x) const {
        if constexpr (R == GG_RELAX_OR_U32) return best | x;
        else if constexpr (R == GG_RELAX_COUNT_DOWN_U32) return best - 1u;
        else return x;
    }
    // the row's value after the lanes with ok set (mask okm) offered theirs
    __device__ __forceinline__ V warp_merge(V best, bool ok, V x, unsigned okm) const {
        if constexpr (R == GG_RELAX_SETIF_U32) {
            return __shfl_sync(FULL, x, __ffs(okm) - 1);
        } else if constexpr (R == GG_RELAX_OR_U32) {
            return best | __reduce_or_sync(FULL, ok ? x : 0u);
        } else if constexpr (R == GG_RELAX_COUNT_DOWN_U32) {
            // one off per active source, not below the floor
            const int64_t v = (int64_t)best - (int64_t)__popc(okm);
            return v > fk ? (V)v : (V)fk;
        } else {
            V mine = ok ? x : none();
            return __reduce_min_sync(FULL, mine);
        }
    }
    // push: offer sv to d; true iff this thread records d
    __device__ __forceinline__ bool offer(uint32_t d, V sv, int record, uint32_t *dedup) const {
        V cur = a[d];
        if (!dst_ok(cur)) return false;
        V old;
        if constexpr (R == GG_RELAX_SETIF_U32) {
            if (((uint32_t)cur >> 31) == 0) return false;
            old = atomicCAS(a + d, cur, sv);
            if (old != cur) return false;
        } else if constexpr (R == GG_RELAX_OR_U32) {
            if ((cur | sv) == cur) return false;
            old = atomicOr(a + d, sv);
            if ((old | sv) == old) return false;
        } else if constexpr (R == GG_RELAX_COUNT_DOWN_U32) {
            // count_down_value(k): the filter saw a[d] > k; a take that finds
            // the count at the floor already (others took it meanwhile) is
            // given back, so the count never stays below k, and exactly one
            // take sees k + 1: the one that brings d to the floor.  Many
            // concurrent takes can carry the count below zero for a moment:
            // counts are below 2^31, so a count read as negative is below
            // the floor too.
            old = atomicSub(a + d, 1u);
            if ((int32_t)old < 0 || (int64_t)old <= fk) {
                atomicAdd(a + d, 1u);
                return false;
            }
            if (record == GG_RECORD_AT_FLOOR) return (int64_t)old == fk + 1;
        } else {
            if (!(sv < cur)) return false;
            old = atomicMin(a + d, sv);
            if (!(sv < old)) return false;
        }
        // level-synchronous: d passed the filter, so it was unvisited and its
        // prev equals the value this thread replaced (no prev load)
        if (record == GG_RECORD_NE_PREV) return (R == GG_RELAX_MIN_PLUS1_I32 && level_sync) || old == prev[d];
        if (record == GG_RECORD_REDUCTION) {
            uint32_t bit = 1u << (d & 31);
            return (atomicOr(dedup + (d >> 5), bit) & bit) == 0;
        }
        return false;
    }
};

__device__ __forceinline__ void emit_out(const EmapArgs &A, bool rec, uint32_t d,
                                         unsigned long long &nv, unsigned long long &ne) {
    uint64_t deg = 0;
    if (rec) {
        deg = A.off[d + 1] - A.off[d];
        nv++;
        ne += deg;
    }
    uint32_t bin = deg <= A.smax ? 0u : (deg <= A.mmax ? 1u : 2u);
    // warp-aggregated append (see gg_core.cu emit_binned)
    const unsigned am = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t b = 0; b < NBINS; ++b) {
        unsigned mk = __ballot_sync(am, rec && bin == b);
        if (mk == 0) continue;
        int leader = __ffs(mk) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(A.out_cnt + FC_BIN0 + b, (unsigned long long)__popc(mk));
        base = __shfl_sync(am, base, leader);
        if (rec && bin == b) {
            uint32_t *dst = b == 0 ? A.out_b0 : (b == 1 ? A.out_b1 : A.out_b2);
            dst[base + __popc(mk & ((1u << lane) - 1u))] = d;
        }
    }
}

template <int BLOCK>
__device__ __forceinline__ void flush_counts(const EmapArgs &A, unsigned long long nv,
                                             unsigned long long ne, unsigned long long sc) {
    nv = dev::block_sum<unsigned long long, BLOCK>(nv);
    ne = dev::block_sum<unsigned long long, BLOCK>(ne);
    sc = dev::block_sum<unsigned long long, BLOCK>(sc);
    if (threadIdx.x == 0) {
        if (nv) atomicAdd(A.out_cnt + FC_NACTV, nv);
        if (ne) atomicAdd(A.out_cnt + FC_NACTE, ne);
        if (sc) atomicAdd(A.out_cnt + FC_SCANNED, sc);
    }
}

// ---------------------------------------------------------------------------
// Dense pull over the CSC
// ---------------------------------------------------------------------------
// One lane owns one destination d.  Full-scan mode walks 32-vertex words
// (one output bitmap word per warp, plain store); candidate mode walks a
// list of destinations (output bitmap pre-cleared, bits set with atomicOr).
// Loads are issued ahead of use: d's value and both offsets together, then
// up to 4 neighbour ids, then their frontier bits and source values.
//
// Split pull (level-synchronous BFS, candidate lists, first_in records):
// PASS 1 settles what each candidate's first two in-edges settle and appends
// the candidates with more edges still to look at to rest_out; PASS 2 walks
// that list from each row's third edge.  A warp of PASS 1 then waits for no
// lane's long row, and a warp of PASS 2 has every lane on an open row.
// frontier bit of source s: from the CTA's shared-memory copy of the
// bitmap's first words when s falls there (STAGE), else through L1/L2
template <bool STAGE>
__device__ __forceinline__ bool probe_bit(const uint32_t *__restrict__ gbits, const uint32_t *sbits, uint32_t sn,
                                          uint32_t s) {
    if constexpr (STAGE) {
        if (s < sn) return (sbits[s >> 5] >> (s & 31u)) & 1u;
    }
    return dev::bit_test(gbits, s);
}

// Shared-memory staging of the pull's list appends: 256 entries per warp for
// the candidate list and, in a split pull's first pass, for the rest list.
// Kernels that run several pull passes declare one and hand it to each.
template <int BLOCK, bool REST>
struct PullSmem {
    uint32_t cand[BLOCK / 32][256];
    uint32_t rest[REST ? BLOCK / 32 : 1][256];
};

template <int R, bool SRCF, bool CAND, int BLOCK, int PASS = 0, bool STAGE = false, bool REST>
__device__ __forceinline__ void pull_body(const EmapArgs &A, const Op<R> &op, PullSmem<BLOCK, REST> &sm,
                                          const uint32_t *sbits = nullptr, uint32_t sn = 0) {
    static_assert(PASS != 1 || REST, "a split pull's first pass stages its rest list");
    static_assert(PASS == 0 || (CAND && R == GG_RELAX_MIN_PLUS1_I32), "split pull: BFS levels, candidate lists");
    using V = typename Op<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nitems = CAND ? *A.cand_n : (uint64_t)A.n;
    const uint64_t nw = (gridDim.x * BLOCK) >> 5;
    const uint64_t gw = (blockIdx.x * BLOCK + threadIdx.x) >> 5;
    // candidate lists: grid-stride over list words; full scan: a contiguous
    // range of vertex words of equal estimated work per warp
    uint32_t wlo = 0, whi = 0;
    if (!CAND) dev::balanced_range(A.word_prefix, (A.n + 31u) >> 5, gw, nw, wlo, whi);
    const uint64_t wstep = CAND ? nw : 1;
    unsigned long long nv = 0, ne = 0, sc = 0;
    dev::WarpAppender<256> keepers{sm.cand[threadIdx.x >> 5], 0, A.cand_out, A.cand_out_n};
    dev::WarpAppender<256> rest{sm.rest[REST ? threadIdx.x >> 5 : 0], 0, A.rest_out, A.rest_out_n};
    for (uint64_t w = CAND ? gw : wlo; CAND ? ((w << 5) < nitems) : (w < whi); w += wstep) {
        const uint64_t item = (w << 5) + lane;
        const bool valid = item < nitems;
        const uint32_t d = CAND ? (valid ? A.cand[item] : 0u) : (uint32_t)item;
        V best = Op<R>::none();
        uint64_t e = 0, end = 0;
        uint4 f2 = make_uint4(0u, 0u, 0u, 0u);
        const bool has_rec = PASS != 2 && (A.first_in || A.first1);
        const bool lazy = has_rec && A.lazy_off;
        if (valid) {
            best = (CAND && A.fresh) ? Op<R>::none() : op.load(d);
            if (has_rec) {
                if (A.first1) {
                    const uint2 r1 = A.first1[d];
                    f2 = make_uint4(r1.x, 0xFFFFFFFFu, r1.y, 0xFFFFFFFFu);
                } else {
                    f2 = A.first_in[d];
                }
            }
            if (!lazy) {
                e = A.in_off[d];
                end = A.in_off[d + 1];
            } else {
                end = f2.z;  // row bounds relative to its start until the offsets are needed
            }
        }
        bool act = valid && op.dst_ok(best);
        if constexpr (R == GG_RELAX_OR_U32) {
            // a bitwise-or row has no early exit: long rows go to k_or_heavy_chunks
            if (A.heavy_T && act && (lazy ? (uint64_t)f2.z : end - e) > A.heavy_T) act = false;
        }
        bool changed = false;
        uint64_t beg = e;
        // the first pass took the record's edges (as many as K allowed)
        const uint64_t skip = PASS == 2 ? (uint64_t)min(A.rec_n, A.K) : 0u;
        e += skip;
        uint64_t lim = min(end, e + (uint64_t)A.K);
        if (has_rec && act && e < lim) {
            // the row's first in-neighbours, loaded beside its offsets: the
            // same edges in the same order as the loop below takes them
            const int cnt = (int)min((uint64_t)A.rec_n, lim - e);
            const uint32_t sv[3] = {f2.x, f2.y, f2.w};
            int used = cnt;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                if (j < cnt && act && (!SRCF || probe_bit<STAGE>(A.in_bits, sbits, sn, sv[j]))) {
                    const V x = op.src_val(sv[j]);
                    if (op.better(x, best)) {
                        best = op.combine(best, x);
                        changed = true;
                        if (!op.dst_ok(best)) {
                            act = false;
                            used = j + 1;
                        }
                    }
                }
            }
            e += used;
        }
        // first pass: rows still open after two edges go to the second
        bool deferred = false;
        if (PASS == 1) {
            deferred = act && e < end;
            rest.push(deferred, d);
            if (deferred) act = false;
        }
        if (lazy && valid) {
            // the row's offsets, for rows still open after their first two edges
            if (act && e < end) {
                const uint64_t b0 = A.in_off[d];
                e += b0;
                end += b0;
                beg = b0;
                lim = min(end, b0 + (uint64_t)A.K);
            }
        }
        while (act && e < lim) {
            const int cnt = (int)min((uint64_t)4, lim - e);
            uint32_t sv[4];
            bool inF[4];
            V xv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) sv[j] = j < cnt ? __ldg(A.in_adj + e + j) : 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                inF[j] = j < cnt && (!SRCF || probe_bit<STAGE>(A.in_bits, sbits, sn, sv[j]));
                xv[j] = j < cnt ? op.src_val(sv[j]) : Op<R>::none();
            }
            int used = cnt;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j < cnt && act && inF[j] && op.better(xv[j], best)) {
                    best = op.combine(best, xv[j]);
                    changed = true;
                    if (!op.dst_ok(best)) {
                        act = false;
                        used = j + 1;
                    }
                }
            }
            e += used;
        }
        sc += e - beg - skip;
        unsigned pend = __ballot_sync(FULL, act && e < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULL, e, j);
            const uint64_t endj = __shfl_sync(FULL, end, j);
            V bj = __shfl_sync(FULL, best, j);
            bool chj = false, actj = true;
            for (uint64_t base = ej; base < endj; base += 32) {
                const uint64_t idx = base + lane;
                bool ok = false;
                V x = Op<R>::none();
                if (idx < endj) {
                    const uint32_t s = __ldg(A.in_adj + idx);
                    if (!SRCF || probe_bit<STAGE>(A.in_bits, sbits, sn, s)) {
                        x = op.src_val(s);
                        ok = op.better(x, bj);
                    }
                }
                if (lane == 0) sc += min((uint64_t)32, endj - base);
                const unsigned okm = __ballot_sync(FULL, ok);
                if (okm) {
                    bj = op.warp_merge(bj, ok, x, okm);
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
            if (A.record == GG_RECORD_NE_PREV) {
                // level-synchronous: d was unvisited, so its prev equals the
                // value replaced; prev is neither read nor written
                if (R == GG_RELAX_MIN_PLUS1_I32 && op.level_sync) {
                    rec = true;
                } else if constexpr (R == GG_RELAX_OR_U32) {
                    // prev may be the relax's source: the copy runs after the step
                    rec = best != op.prev[d];
                } else if (best != op.prev[d]) {
                    op.prev[d] = best;
                    rec = true;
                }
            } else if (A.record == GG_RECORD_REDUCTION) {
                rec = true;
            } else if (A.record == GG_RECORD_AT_FLOOR) {
                rec = (int64_t)best == op.fk;  // COUNT_DOWN: counted down to the floor now
            }
        }
        if (A.out_bits) {
            if (CAND) {
                // lanes holding vertices of the same bitmap word combine
                // their bits; one atomicOr per word and warp
                const uint32_t wd = d >> 5;
                unsigned todo = __ballot_sync(FULL, rec);
                while (todo) {  // one round per distinct word (list is mostly ascending)
                    const int leader = __ffs(todo) - 1;
                    const uint32_t w0 = __shfl_sync(FULL, wd, leader);
                    const bool mine = rec && wd == w0;
                    const unsigned bits = __reduce_or_sync(FULL, mine ? (1u << (d & 31)) : 0u);
                    if ((int)lane == leader) atomicOr(A.out_bits + w0, bits);
                    todo &= ~__ballot_sync(FULL, mine);
                }
            } else {
                const unsigned bits = __ballot_sync(FULL, rec);
                if (lane == 0) A.out_bits[w] = bits;
            }
        }
        if (rec) {
            // the output list is built from the bitmap only if a push needs it
            nv++;
            // out-degree: for a symmetric graph the CSC is the CSR, and d's
            // row bounds are already in registers
            ne += A.off == A.in_off ? end - beg : A.off[d + 1] - A.off[d];
        }
        // still a candidate: passes the filter and has in-edges
        if (A.cand_out) keepers.push(valid && act && end > beg, d);
    }
    if (A.cand_out) keepers.flush();
    if (PASS == 1) rest.flush();
    if (A.out_cnt) flush_counts<BLOCK>(A, nv, ne, sc);
}

template <int R, bool SRCF, bool CAND, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 6) k_pull(EmapArgs A, Op<R> op) {
    __shared__ PullSmem<BLOCK, false> sm;
    pull_body<R, SRCF, CAND, BLOCK>(A, op, sm);
}

// Bitwise-or pulls over the long rows (FMv's all-source steps): a warp per
// chunk of a heavy row (the CSC's heavy-row chunk table) ORs its sources'
// bits, four edges per lane in flight, and merges them into the row's value
// with one atomicOr; then a thread per heavy row records it (NE_PREV: its
// value differs from prev) into the output frontier.
template <bool SRCF>
__global__ void __launch_bounds__(256) k_or_heavy_chunks(EmapArgs A, Op<GG_RELAX_OR_U32> op, HeavyRows H) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < H.nchunks; c += nw) {
        const uint32_t lo = H.crow[c];
        const uint32_t d = H.v[lo];
        const uint32_t cur = *(volatile const uint32_t *)(op.a + d);
        if (!op.dst_ok(cur)) continue;  // the same row for the whole warp
        const uint64_t rb = A.in_off[d], re = A.in_off[d + 1];
        const uint64_t e0 = rb + (c - H.first[lo]) * H.CH;
        const uint64_t e1 = min(e0 + H.CH, re);
        uint32_t acc = 0;
        for (uint64_t base = e0; base < e1; base += 128) {
            uint32_t sv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint64_t e = base + j * 32 + lane;
                sv[j] = e < e1 ? __ldg(A.in_adj + e) : 0xFFFFFFFFu;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (sv[j] != 0xFFFFFFFFu && (!SRCF || dev::bit_test(A.in_bits, sv[j]))) acc |= op.b[sv[j]];
        }
        acc = __reduce_or_sync(FULL, acc);
        if (lane == 0 && (cur | acc) != cur) atomicOr(op.a + d, acc);
    }
}

__global__ void __launch_bounds__(256) k_or_heavy_finalize(EmapArgs A, Op<GG_RELAX_OR_U32> op, HeavyRows H) {
    unsigned long long nv = 0, ne = 0;
    const uint32_t nth = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < H.nheavy; i0 += nth) {
        const uint32_t i = i0 + threadIdx.x;
        bool rec = false;
        uint32_t d = 0;
        if (i < H.nheavy) {
            d = H.v[i];
            rec = A.record == GG_RECORD_NE_PREV && op.a[d] != op.prev[d];
        }
        if (rec && A.out_bits) atomicOr(A.out_bits + (d >> 5), 1u << (d & 31));
        if (A.out_b0) emit_out(A, rec, d, nv, ne);
    }
    if (A.out_cnt) flush_counts<256>(A, nv, ne, 0);
}

// ---------------------------------------------------------------------------
// Degree-binned sparse push
// ---------------------------------------------------------------------------
// Edges [beg, end) of one source pushed by W cooperating threads (a warp,
// W = 32, or a CTA, W = BLOCK; `t` = this thread's index among them), four
// edges per thread in flight: the loads of the four targets' values and the
// four atomics overlap instead of forming four dependent round trips.
// Output list appends of one warp staged in shared memory per degree bin:
// one global atomic per ~CAP records instead of one per warp round (the bin
// counters are the hottest addresses of a push that activates many vertices).
template <int CAP>
struct BinAppender {
    dev::WarpAppender<CAP> ap[NBINS];
    unsigned long long nv = 0, ne = 0;
    __device__ __forceinline__ void init(const EmapArgs &A, uint32_t *warp_buf) {
        uint32_t *dst[NBINS] = {A.out_b0, A.out_b1, A.out_b2};
#pragma unroll
        for (int b = 0; b < NBINS; ++b) ap[b] = {warp_buf + b * CAP, 0u, dst[b], A.out_cnt + FC_BIN0 + b};
    }
    // all 32 lanes together
    __device__ __forceinline__ void emit(const EmapArgs &A, bool rec, uint32_t d) {
        uint64_t deg = 0;
        if (rec) {
            deg = A.off[d + 1] - A.off[d];
            nv++;
            ne += deg;
        }
        const uint32_t bin = deg <= A.smax ? 0u : (deg <= A.mmax ? 1u : 2u);
#pragma unroll
        for (int b = 0; b < NBINS; ++b) ap[b].push(rec && bin == (uint32_t)b, d);
    }
    __device__ __forceinline__ void flush() {
#pragma unroll
        for (int b = 0; b < NBINS; ++b) ap[b].flush();
    }
};

template <int R, int W, typename Emit>
__device__ __forceinline__ void push_edges(const EmapArgs &A, const Op<R> &op, typename Op<R>::V sv, uint64_t beg,
                                           uint64_t end, uint32_t t, Emit &&emit) {
    constexpr int U = 4;
    for (uint64_t base = beg; base < end; base += (uint64_t)W * U) {
        uint32_t d[U];
        bool rec[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t e = base + (uint64_t)u * W + t;
            d[u] = e < end ? __ldg(A.adj + e) : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t e = base + (uint64_t)u * W + t;
            rec[u] = e < end && op.offer(d[u], sv, A.record, A.out_bits);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (base + (uint64_t)u * W >= end) break;  // uniform across the W threads
            emit(rec[u], d[u]);
        }
    }
}

template <int R, int BLOCK>
__device__ __forceinline__ void push_binned_body(const EmapArgs &A, const Op<R> &op, uint32_t nb_large,
                                                 uint32_t nb_med) {
    using V = typename Op<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long sc = 0;
    __shared__ uint64_t s_first[kLargeLocal + 1];
    __shared__ uint32_t s_app[BLOCK / 32][NBINS * kAppCap];
    BinAppender<kAppCap> app;
    app.init(A, s_app[threadIdx.x >> 5]);
    auto emit = [&](bool rec, uint32_t d) { app.emit(A, rec, d); };
    if (blockIdx.x < nb_large) {
        // large bin: rows cut into chunks of large_ch edges, a CTA per chunk,
        // so one hub row is spread over many SMs.  The chunk prefix is built
        // by each CTA in shared memory when the bin is small (no extra
        // launches), else read from large_first (built on the device before).
        // With merge_med the medium bin joins it (rows c2.. of the table):
        // a frontier of a few vertices then still spreads over many CTAs.
        const uint32_t cm = A.c2 + (A.merge_med ? A.c1 : 0u);
        auto row = [&](uint32_t i) { return i < A.c2 ? A.in_b2[i] : A.in_b1[i - A.c2]; };
        const uint64_t *first = A.large_first;
        if (!first) {
            for (uint32_t i = threadIdx.x; i < cm; i += BLOCK) {
                const uint32_t v = row(i);
                s_first[i + 1] = (A.off[v + 1] - A.off[v] + A.large_ch - 1) / A.large_ch;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_first[0] = 0;
                for (uint32_t i = 1; i <= cm; ++i) s_first[i] += s_first[i - 1];
            }
            __syncthreads();
            first = s_first;
        }
        const uint64_t nch = first[cm];
        for (uint64_t c = blockIdx.x; c < nch; c += nb_large) {
            uint32_t lo = 0, hi = cm;  // last h with first[h] <= c
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (first[mid] <= c) lo = mid; else hi = mid;
            }
            const uint32_t s = row(lo);
            const V sv = op.src_val(s);
            const uint64_t rb = A.off[s], re = A.off[s + 1];
            const uint64_t beg = rb + (c - first[lo]) * A.large_ch;
            const uint64_t end = min(beg + A.large_ch, re);
            if (threadIdx.x == 0) sc += end - beg;
            push_edges<R, BLOCK>(A, op, sv, beg, end, threadIdx.x, emit);
        }
    } else if (blockIdx.x < nb_large + nb_med) {
        // medium bin: a warp per source vertex
        const uint32_t wpb = BLOCK / 32;
        const uint32_t nwm = nb_med * wpb;
        const uint32_t wid = (blockIdx.x - nb_large) * wpb + (threadIdx.x >> 5);
        const uint32_t cmed = A.c1 + (A.large_as_med ? A.c2 : 0u);
        for (uint32_t i = wid; i < cmed; i += nwm) {
            const uint32_t s = i < A.c1 ? A.in_b1[i] : A.in_b2[i - A.c1];
            const V sv = op.src_val(s);
            const uint64_t beg = A.off[s], end = A.off[s + 1];
            if (lane == 0) sc += end - beg;
            push_edges<R, 32>(A, op, sv, beg, end, lane, emit);
        }
    } else {
        // small bin: a warp per 32 source vertices, their edges flattened
        const uint32_t wpb = BLOCK / 32;
        const uint32_t nws = (gridDim.x - nb_large - nb_med) * wpb;
        const uint32_t wid = (blockIdx.x - nb_large - nb_med) * wpb + (threadIdx.x >> 5);
        for (uint64_t base = (uint64_t)wid * 32; base < A.c0; base += (uint64_t)nws * 32) {
            const uint64_t i = base + lane;
            const bool have = i < A.c0;
            uint32_t s = 0;
            uint64_t beg = 0, end = 0;
            V sv = Op<R>::none();
            if (have) {
                s = A.in_b0[i];
                beg = A.off[s];
                end = A.off[s + 1];
                sv = op.src_val(s);
            }
            const uint32_t deg = (uint32_t)(end - beg);
            sc += deg;
            dev::warp_flat_rows<4>(
                A.adj, beg, deg, sv, [&](uint32_t d, V x) { return op.offer(d, x, A.record, A.out_bits); }, emit);
        }
    }
    app.flush();
    flush_counts<BLOCK>(A, app.nv, app.ne, sc);
}

template <int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_binned(EmapArgs A, Op<R> op, uint32_t nb_large, uint32_t nb_med) {
    push_binned_body<R, BLOCK>(A, op, nb_large, nb_med);
}

// chunks of each large-bin vertex's row (first[c2] = 0 before the scan)
__global__ void k_large_chunks(const uint32_t *b2, uint32_t c2, const uint64_t *off, uint32_t ch,
                               uint64_t *first) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c2) {
        const uint32_t v = b2[i];
        first[i] = (off[v + 1] - off[v] + ch - 1) / ch;
    } else if (i == c2) {
        first[i] = 0;
    }
}

// ---------------------------------------------------------------------------
// Edge-balanced (merge-path) push over a contiguous frontier list
// ---------------------------------------------------------------------------
// Gather the three bins into one list with out-degrees.
__global__ void k_concat_bins(const uint32_t *b0, const uint32_t *b1, const uint32_t *b2,
                              const uint64_t *cnt, const uint64_t *off, uint32_t *list,
                              uint64_t *deg) {
    const uint64_t c0 = cnt[FC_BIN0], c1 = cnt[FC_BIN1], c2 = cnt[FC_BIN2];
    const uint64_t tot = c0 + c1 + c2;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < tot; i += stride) {
        uint32_t v = i < c0 ? b0[i] : (i < c0 + c1 ? b1[i - c0] : b2[i - c0 - c1]);
        list[i] = v;
        deg[i] = off[v + 1] - off[v];
    }
}

// pre: exclusive prefix of degrees (k+1 entries, pre[k] = total edges).
template <int R, int BLOCK, int TILE>
__global__ void __launch_bounds__(BLOCK) k_push_merge(EmapArgs A, Op<R> op, const uint32_t *list,
                                                      const uint64_t *pre, uint64_t k) {
    using V = typename Op<R>::V;
    __shared__ uint64_t s_lo;
    unsigned long long nv = 0, ne = 0, sc = 0;
    const uint64_t total = pre[k];
    const uint64_t ntiles = (total + TILE - 1) / TILE;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint64_t t0 = t * TILE;
        if (threadIdx.x == 0) {
            // last source i with pre[i] <= t0
            uint64_t lo = 0, hi = k;
            while (hi - lo > 1) {
                uint64_t mid = (lo + hi) / 2;
                if (pre[mid] <= t0) lo = mid; else hi = mid;
            }
            s_lo = lo;
        }
        __syncthreads();
        const uint64_t lo = s_lo;
        __syncthreads();
        for (uint64_t e0 = t0; e0 < min(t0 + TILE, total); e0 += BLOCK) {
            const uint64_t e = e0 + threadIdx.x;
            bool rec = false;
            uint32_t d = 0;
            if (e < total && e < t0 + TILE) {
                // source index: last i >= lo with pre[i] <= e (search a short range)
                uint64_t a = lo, b = k;
                uint64_t step = 1;
                while (a + step < b && pre[a + step] <= e) { a += step; step <<= 1; }
                b = min(b, a + step);
                while (b - a > 1) {
                    uint64_t mid = (a + b) / 2;
                    if (pre[mid] <= e) a = mid; else b = mid;
                }
                const uint32_t s = list[a];
                const uint64_t pos = A.off[s] + (e - pre[a]);
                d = __ldg(A.adj + pos);
                rec = op.offer(d, op.src_val(s), A.record, A.out_bits);
                sc++;
            }
            emit_out(A, rec, d, nv, ne);
        }
    }
    flush_counts<BLOCK>(A, nv, ne, sc);
}

// ---------------------------------------------------------------------------
// Dense push from a frontier bitmap
// ---------------------------------------------------------------------------
template <int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_push_dense(EmapArgs A, Op<R> op) {
    using V = typename Op<R>::V;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwords = (A.n + 31u) >> 5;
    const uint32_t nw = (gridDim.x * BLOCK) >> 5;
    unsigned long long nv = 0, ne = 0, sc = 0;
    for (uint32_t w = (blockIdx.x * BLOCK + threadIdx.x) >> 5; w < nwords; w += nw) {
        const uint32_t s = (w << 5) + lane;
        const uint32_t word = A.in_bits ? A.in_bits[w] : FULL;
        const bool act = s < A.n && ((word >> lane) & 1u);
        uint64_t beg = 0, end = 0;
        V sv = Op<R>::none();
        if (act) {
            beg = A.off[s];
            end = A.off[s + 1];
            sv = op.src_val(s);
        }
        // phase 1: up to K edges per lane
        const uint32_t k1 = (uint32_t)min(end - beg, (uint64_t)A.K);
        const uint32_t maxk = __reduce_max_sync(FULL, k1);
        for (uint32_t k = 0; k < maxk; ++k) {
            bool rec = false;
            uint32_t d = 0;
            if (k < k1) {
                d = __ldg(A.adj + beg + k);
                rec = op.offer(d, sv, A.record, A.out_bits);
            }
            emit_out(A, rec, d, nv, ne);
        }
        sc += k1;
        // phase 2: warp-cooperative over long rows
        unsigned pend = __ballot_sync(FULL, act && beg + k1 < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint64_t ej = __shfl_sync(FULL, beg + k1, j);
            const uint64_t endj = __shfl_sync(FULL, end, j);
            const V svj = __shfl_sync(FULL, sv, j);
            if (lane == 0) sc += endj - ej;
            for (uint64_t base = ej; base < endj; base += 32) {
                const uint64_t e = base + lane;
                bool rec = false;
                uint32_t d = 0;
                if (e < endj) {
                    d = __ldg(A.adj + e);
                    rec = op.offer(d, svj, A.record, A.out_bits);
                }
                emit_out(A, rec, d, nv, ne);
            }
        }
    }
    flush_counts<BLOCK>(A, nv, ne, sc);
}

// prev[v] = a[v] over the output list (maintain_copies, vertexmap.h:2515-2535)
template <typename V>
__global__ void k_copy_prev(const uint32_t *b0, const uint32_t *b1, const uint32_t *b2,
                            const uint64_t *cnt, const V *a, V *prev) {
    const uint64_t c0 = cnt[FC_BIN0], c1 = cnt[FC_BIN1], c2 = cnt[FC_BIN2];
    const uint64_t tot = c0 + c1 + c2;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < tot; i += stride) {
        uint32_t v = i < c0 ? b0[i] : (i < c0 + c1 ? b1[i - c0] : b2[i - c0 - c1]);
        prev[v] = a[v];
    }
}

__global__ void k_scatter_zero_i32(int32_t *a, int32_t *b, const uint32_t *idx, uint32_t k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) {
        a[idx[i]] = 0;
        b[idx[i]] = 0;
    }
}

__global__ void k_iota_u32(uint32_t *a, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t stride = gridDim.x * blockDim.x;
    for (; i < n; i += stride) a[i] = i;
}

// neighbours of vertex z get label 0 in both copies (CCv PRESET_ZERO,
// bench/CCv.C:262-291, applied to vertex 0 whose component minimum is 0)
__global__ void k_preset_zero(const uint64_t *off, const uint32_t *adj, uint32_t z, uint32_t *lab,
                              uint32_t *prev) {
    for (uint64_t e = off[z] + blockIdx.x * blockDim.x + threadIdx.x; e < off[z + 1];
         e += (uint64_t)gridDim.x * blockDim.x) {
        lab[adj[e]] = 0;
        prev[adj[e]] = 0;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
constexpr int kBlock = 256;

static unsigned persistent_grid(gg_ctx *ctx, uint64_t warps_needed) {
    uint64_t blocks = (warps_needed + (kBlock / 32) - 1) / (kBlock / 32);
    uint64_t cap = (uint64_t)ctx->sm_count * tuning().blocks_per_sm;
    if (blocks > cap) blocks = cap;
    return (unsigned)std::max<uint64_t>(blocks, 1);
}

static bool threshold_sparse(int kind, int k, uint64_t nactv, uint64_t nacte, uint64_t m) {
    switch (kind) {
    case GG_THRESH_ALWAYS_SPARSE: return true;
    case GG_THRESH_ALWAYS_DENSE: return false;
    case GG_THRESH_FRAC:
        // api.h:137-140: float(nactv+nacte) <= float(m) / (100.0/(float)k)
        return (float)(nactv + nacte) <= (float)m / (float)(100.0 / (float)k);
    default:
        return (nactv + nacte) <= (m / 20);  // api.h:154-156
    }
}

int learned_select(gg_graph *g, uint64_t nactv, uint64_t nacte, int iter, bool can_early_exit);

// the dense pull's per-vertex records as knob pull_first selects them
static gg_status pull_records(gg_graph *g, const Tuning &t, const uint4 **fi, const uint2 **f1, int *rec_n,
                              int *lazy) {
    *fi = nullptr;
    *f1 = nullptr;
    *rec_n = 0;
    *lazy = 0;
    switch (t.pull_first) {
    case 1: *fi = g->first_in; *rec_n = 2; break;
    case 2: *fi = g->first_in; *rec_n = 2; *lazy = 1; break;
    case 3: *fi = g->first_in; *rec_n = 3; *lazy = 1; break;
    case 4:
        GG_CHECK(graph_ensure_first1(g));
        *f1 = g->first1;
        *rec_n = 1;
        *lazy = 1;
        break;
    default: break;
    }
    return GG_OK;
}

template <int R>
static gg_status launch_variant(gg_graph *g, const gg_emap_desc *d, gg_frontier *in,
                                gg_frontier *out, int variant) {
    gg_ctx *ctx = g->ctx;
    cudaStream_t st = ctx->stream;
    const Tuning &t = tuning();
    Op<R> op;
    op.a = (typename Op<R>::V *)d->a->d;
    op.prev = d->prev ? (typename Op<R>::V *)d->prev->d : nullptr;
    op.b = (R == GG_RELAX_OR_U32 && d->src) ? (const typename Op<R>::V *)d->src->d : nullptr;
    op.filter = d->dst_filter;
    op.fk = d->dst_filter_k;
    op.level_sync = (d->src_level_sync && d->dst_filter == GG_FILTER_GT_CONST) ? 1 : 0;

    EmapArgs A;
    memset(&A, 0, sizeof(A));
    A.off = g->off;
    A.adj = g->adj;
    A.in_off = g->in_off;
    A.in_adj = g->in_adj;
    A.n = g->n;
    A.record = d->record;
    A.smax = t.bin_small_max;
    A.mmax = t.bin_medium_max;
    A.K = variant == GG_VAR_PULL_DENSE ? t.pull_k : t.push_k;
    A.word_prefix = g->heavy.pull_prefix;
    GG_CHECK(pull_records(g, t, &A.first_in, &A.first1, &A.rec_n, &A.lazy_off));
    const bool have_out = out != nullptr && d->record != GG_RECORD_NONE;
    if (have_out) {
        GG_CHECK(frontier_alloc_bins(out));
        GG_CHECK(frontier_reset_counts(out));
        A.out_b0 = out->bins[0];
        A.out_b1 = out->bins[1];
        A.out_b2 = out->bins[2];
        A.out_cnt = (unsigned long long *)out->d_cnt;
    }
    const size_t words = ((size_t)g->n + 31) / 32;
    bool out_bitmap_valid = false;
    if (variant == GG_VAR_PULL_DENSE) {
        if (have_out) {
            GG_CHECK(frontier_alloc_bitmap(out));
            A.out_bits = out->bitmap;
            out_bitmap_valid = true;
        }
    } else if (have_out && d->record == GG_RECORD_REDUCTION) {
        GG_CHECK(frontier_alloc_bitmap(out));
        GG_CUDA(ctx, cudaMemsetAsync(out->bitmap, 0, words * 4, st));
        A.out_bits = out->bitmap;
        out_bitmap_valid = true;
    }
    if (!have_out && d->record != GG_RECORD_NONE) return set_error(ctx, GG_ERR_ARG, "record without output frontier");
    if (!have_out) {
        // counts still wanted for the scanned-edge statistic
        if (!g->aux_cnt) GG_CUDA(ctx, cudaMalloc(&g->aux_cnt, FC_WORDS * 8));
        GG_CUDA(ctx, cudaMemsetAsync(g->aux_cnt, 0, FC_WORDS * 8, st));
        A.out_cnt = (unsigned long long *)g->aux_cnt;
    }

    const bool all_in = in == nullptr || in->all;
    // kernel timing brackets only the traversal kernel (not conversions)
    auto tstart = [&]() { if (ctx->time_kernels) cudaEventRecord(ctx->evk0, st); };
    switch (variant) {
    case GG_VAR_PULL_DENSE: {
        if (!all_in) {
            GG_CHECK(frontier_ensure_bitmap(in));
            A.in_bits = in->bitmap;
        }
        CandLists *cl = g->cand_active ? &g->cand : nullptr;
        if (cl) {
            A.cand_out = cl->list[cl->cur ^ 1];
            A.cand_out_n = (unsigned long long *)(cl->cnt + (cl->cur ^ 1));
            GG_CUDA(ctx, cudaMemsetAsync(A.cand_out_n, 0, 8, st));
            if (cl->valid) {
                A.cand = cl->list[cl->cur];
                A.cand_n = (const unsigned long long *)(cl->cnt + cl->cur);
            } else if (g->nonisolated) {
                // first pull of a run: every vertex with in-edges
                A.cand = g->nonisolated;
                A.cand_n = (const unsigned long long *)g->nonisolated_n;
            }
            if (A.cand && A.out_bits) GG_CUDA(ctx, cudaMemsetAsync(A.out_bits, 0, words * 4, st));
        }
        if constexpr (R == GG_RELAX_OR_U32) {
            if (g->heavy.nchunks && (d->record == GG_RECORD_NE_PREV || d->record == GG_RECORD_NONE))
                A.heavy_T = g->heavy.T;
        }
        const uint64_t items = (A.cand && cl->host_n != UINT64_MAX) ? cl->host_n : (uint64_t)g->n;
        const void *kp = A.cand ? (all_in ? (const void *)k_pull<R, false, true, kBlock>
                                          : (const void *)k_pull<R, true, true, kBlock>)
                                : (all_in ? (const void *)k_pull<R, false, false, kBlock>
                                          : (const void *)k_pull<R, true, false, kBlock>);
        const unsigned grid = occ_grid(ctx, kp, kBlock, items);
        tstart();
        if (A.cand) {
            if (all_in) k_pull<R, false, true, kBlock><<<grid, kBlock, 0, st>>>(A, op);
            else k_pull<R, true, true, kBlock><<<grid, kBlock, 0, st>>>(A, op);
        } else {
            if (all_in) k_pull<R, false, false, kBlock><<<grid, kBlock, 0, st>>>(A, op);
            else k_pull<R, true, false, kBlock><<<grid, kBlock, 0, st>>>(A, op);
        }
        GG_LAUNCHED(ctx);
        if constexpr (R == GG_RELAX_OR_U32) {
            if (A.heavy_T) {
                const HeavyRows &H = g->heavy;
                const unsigned cap = (unsigned)(ctx->sm_count * 8);
                const unsigned cb = (unsigned)std::min<uint64_t>((H.nchunks * 32 + 255) / 256, cap);
                if (all_in) k_or_heavy_chunks<false><<<cb, 256, 0, st>>>(A, op, H);
                else k_or_heavy_chunks<true><<<cb, 256, 0, st>>>(A, op, H);
                GG_LAUNCHED(ctx);
                const unsigned fb = (unsigned)std::min<uint64_t>((H.nheavy + 255) / 256, cap);
                k_or_heavy_finalize<<<fb ? fb : 1, 256, 0, st>>>(A, op, H);
                GG_LAUNCHED(ctx);
            }
        }
        if (cl) {
            cl->cur ^= 1;
            cl->valid = true;
            cl->host_n = UINT64_MAX;  // known on the device only
        }
        break;
    }
    case GG_VAR_PUSH_DENSE: {
        if (!all_in) {
            GG_CHECK(frontier_ensure_bitmap(in));
            A.in_bits = in->bitmap;
        }
        unsigned grid = persistent_grid(ctx, words);
        tstart();
        k_push_dense<R, kBlock><<<grid, kBlock, 0, st>>>(A, op);
        GG_LAUNCHED(ctx);
        break;
    }
    case GG_VAR_PUSH_SPARSE: {
        if (all_in) {
            if (!in) return set_error(ctx, GG_ERR_ARG, "sparse push needs a frontier");
        }
        GG_CHECK(frontier_ensure_list(in));
        GG_CHECK(frontier_fetch_counts(in));
        A.in_b0 = in->bins[0];
        A.in_b1 = in->bins[1];
        A.in_b2 = in->bins[2];
        A.c0 = (uint32_t)in->h_cnt[FC_BIN0];
        A.c1 = (uint32_t)in->h_cnt[FC_BIN1];
        A.c2 = (uint32_t)in->h_cnt[FC_BIN2];
        const uint32_t cap = ctx->sm_count * t.blocks_per_sm;
        uint32_t nb_large = 0;
        A.large_ch = t.large_chunk;
        A.large_first = nullptr;  // small large bin: chunk table built inside the kernel
        // a few medium rows: chunk them like large rows, one CTA per chunk,
        // instead of one warp walking each row alone
        A.merge_med = A.c1 && A.c1 + A.c2 <= kLargeLocal && A.c1 < ctx->sm_count;
        if (A.c2 > kLargeLocal) {
            // chunk table of the large bin: counts, then an exclusive scan
            size_t cub_bytes = 0;
            GG_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (uint64_t *)nullptr,
                                                       (uint64_t *)nullptr, (int64_t)A.c2 + 1, st));
            const size_t fb = (((size_t)A.c2 + 1) * 8 + 255) / 256 * 256;
            void *p;
            GG_CHECK(graph_scratch(g, fb + cub_bytes, &p));
            uint64_t *first = (uint64_t *)p;
            k_large_chunks<<<(A.c2 + 256) / 256, 256, 0, st>>>(A.in_b2, A.c2, g->off, A.large_ch, first);
            GG_LAUNCHED(ctx);
            GG_CUDA(ctx, cub::DeviceScan::ExclusiveSum((char *)p + fb, cub_bytes, first, first,
                                                       (int64_t)A.c2 + 1, st));
            ctx->launches++;
            A.large_first = first;
        }
        if (A.c2 || A.merge_med) {
            // upper bound on the chunk count from the host-known edge total
            const uint64_t est = in->h_cnt[FC_NACTE] / A.large_ch + A.c2 + (A.merge_med ? A.c1 : 0);
            nb_large = (uint32_t)std::min<uint64_t>(est, cap);
        }
        uint32_t nb_med = A.merge_med ? 0 : std::min<uint32_t>((A.c1 + kBlock / 32 - 1) / (kBlock / 32), cap);
        uint32_t nb_small = std::min<uint32_t>((A.c0 + kBlock - 1) / kBlock, cap);
        uint32_t grid = nb_large + nb_med + nb_small;
        tstart();
        if (grid == 0) break;
        k_push_binned<R, kBlock><<<grid, kBlock, 0, st>>>(A, op, nb_large, nb_med);
        GG_LAUNCHED(ctx);
        break;
    }
    case GG_VAR_PUSH_MERGE: {
        if (!in) return set_error(ctx, GG_ERR_ARG, "merge push needs a frontier");
        GG_CHECK(frontier_ensure_list(in));
        GG_CHECK(frontier_fetch_counts(in));
        uint64_t k = in->h_cnt[FC_BIN0] + in->h_cnt[FC_BIN1] + in->h_cnt[FC_BIN2];
        if (k == 0) break;
        // scratch: list[k] u32, deg[k+1] u64, pre[k+1] u64, cub temp
        size_t cub_bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (uint64_t *)nullptr, (uint64_t *)nullptr, (int64_t)(k + 1), st);
        size_t lb = ((k * 4 + 255) / 256) * 256, db = (((k + 1) * 8 + 255) / 256) * 256;
        void *p;
        GG_CHECK(graph_scratch(g, lb + 2 * db + cub_bytes, &p));
        uint32_t *list = (uint32_t *)p;
        uint64_t *deg = (uint64_t *)((char *)p + lb);
        uint64_t *pre = (uint64_t *)((char *)p + lb + db);
        void *cub_tmp = (char *)p + lb + 2 * db;
        GG_CUDA(ctx, cudaMemsetAsync(deg + k, 0, 8, st));
        tstart();
        k_concat_bins<<<persistent_grid(ctx, (k + 31) / 32), kBlock, 0, st>>>(
            in->bins[0], in->bins[1], in->bins[2], in->d_cnt, g->off, list, deg);
        GG_LAUNCHED(ctx);
        GG_CUDA(ctx, cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, deg, pre, (int64_t)(k + 1), st));
        ctx->launches++;
        constexpr int TILE = 4096;
        uint64_t edges = in->h_cnt[FC_NACTE];
        unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((edges + TILE - 1) / TILE,
                                                                            (uint64_t)ctx->sm_count * t.blocks_per_sm));
        k_push_merge<R, kBlock, TILE><<<grid, kBlock, 0, st>>>(A, op, list, pre, k);
        GG_LAUNCHED(ctx);
        break;
    }
    default:
        return set_error(ctx, GG_ERR_ARG, "unknown variant");
    }
    if (ctx->time_kernels) cudaEventRecord(ctx->evk1, st);
    if (have_out) {
        const bool list_written = variant != GG_VAR_PULL_DENSE;
        // level-synchronous BFS: a push's unique first writer records d and no
        // later step compares prev of a visited vertex, so no copy is needed
        const bool sync_levels = d->src_level_sync && d->relax == GG_RELAX_MIN_PLUS1_I32;
        // (an OR pull leaves the copy to here: its prev may be its source)
        if (d->record == GG_RECORD_NE_PREV && (variant != GG_VAR_PULL_DENSE || R == GG_RELAX_OR_U32) &&
            !sync_levels) {
            if (!d->prev) return set_error(ctx, GG_ERR_ARG, "NE_PREV record needs prev");
            k_copy_prev<<<persistent_grid(ctx, words), kBlock, 0, st>>>(
                out->bins[0], out->bins[1], out->bins[2], out->d_cnt, op.a, op.prev);
            GG_LAUNCHED(ctx);
        }
        out->all = false;
        out->has_list = list_written;
        out->has_bitmap = out_bitmap_valid;
        out->host_valid = false;
    }
    return GG_OK;
}

gg_status pr_edgemap_gather(gg_graph *g, const gg_emap_desc *d, gg_frontier *in);

// The analytics' validation edgemaps: relax(s, d) returns a condition and
// the record is a reduction, so d is recorded when an active in-neighbour
// satisfies it; nothing is written.  CCv.C:612-617: a[d] != a[s] (labels);
// BFSLVLv.C:288-305: a[s] > a[d] + 1 || a[s] < a[d] - 1 (symmetric graph)
// or a[s] < a[d] - 1 (directed) on the levels.
template <int K>
__device__ __forceinline__ bool check_hit(uint32_t as, uint32_t ad) {
    if constexpr (K == GG_RELAX_NE_CHECK) return as != ad;
    else if constexpr (K == GG_RELAX_GAP_CHECK)
        return (int64_t)(int32_t)as > (int64_t)(int32_t)ad + 1 || (int64_t)(int32_t)as < (int64_t)(int32_t)ad - 1;
    else return (int64_t)(int32_t)as < (int64_t)(int32_t)ad - 1;
}

// A warp per 32-vertex word walks the word's in-rows one after the other,
// the lanes striding each row.
template <int K>
__global__ void __launch_bounds__(kBlock) k_check(EmapArgs A, const uint32_t *__restrict__ a,
                                                  const uint32_t *__restrict__ src_bits) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwords = (A.n + 31u) >> 5;
    const uint32_t nw = (gridDim.x * kBlock) >> 5;
    unsigned long long nv = 0, ne = 0;
    for (uint32_t w = (blockIdx.x * kBlock + threadIdx.x) >> 5; w < nwords; w += nw) {
        bool rec = false;
        for (uint32_t j = 0; j < 32; ++j) {
            const uint32_t d = (w << 5) + j;
            if (d >= A.n) break;
            const uint32_t ad = a[d];
            const uint64_t beg = A.in_off[d], end = A.in_off[d + 1];
            bool found = false;
            for (uint64_t base = beg; base < end && !found; base += 32) {
                bool hit = false;
                if (base + lane < end) {
                    const uint32_t s = A.in_adj[base + lane];
                    hit = (!src_bits || dev::bit_test(src_bits, s)) && check_hit<K>(a[s], ad);
                }
                found = __any_sync(FULL, hit);
            }
            if (lane == j) rec = found;
        }
        const uint32_t d = (w << 5) + lane;
        rec = rec && d < A.n;
        const unsigned bits = __ballot_sync(FULL, rec);
        if (lane == 0) A.out_bits[w] = bits;
        emit_out(A, rec, d, nv, ne);
    }
    flush_counts<kBlock>(A, nv, ne, 0);
}

static gg_status check_relax(gg_graph *g, const gg_emap_desc *d, gg_frontier *in, gg_frontier *out) {
    gg_ctx *ctx = g->ctx;
    if (d->a->t != (d->relax == GG_RELAX_NE_CHECK ? GG_U32 : GG_I32))
        return set_error(ctx, GG_ERR_ARG, "check relax: NE on a uint32 property, GAP / AHEAD on an int32 one");
    if (d->dst_filter != GG_FILTER_NONE) return set_error(ctx, GG_ERR_UNSUPPORTED, "check relaxes take no dst filter");
    if (!out) return GG_OK;  // nothing is written, so nothing to do without a record
    EmapArgs A;
    memset(&A, 0, sizeof(A));
    A.off = g->off;
    A.in_off = g->in_off;
    A.in_adj = g->in_adj;
    A.n = g->n;
    const Tuning &t = tuning();
    A.smax = t.bin_small_max;
    A.mmax = t.bin_medium_max;
    const uint32_t *src_bits = nullptr;
    if (in && !in->all) {
        GG_CHECK(frontier_ensure_bitmap(in));
        src_bits = in->bitmap;
    }
    GG_CHECK(frontier_alloc_bins(out));
    GG_CHECK(frontier_alloc_bitmap(out));
    GG_CHECK(frontier_reset_counts(out));
    A.out_bits = out->bitmap;
    A.out_b0 = out->bins[0];
    A.out_b1 = out->bins[1];
    A.out_b2 = out->bins[2];
    A.out_cnt = (unsigned long long *)out->d_cnt;
    const uint64_t words = ((uint64_t)g->n + 31) / 32;
    const unsigned grid = persistent_grid(ctx, words);
    const uint32_t *av = (const uint32_t *)d->a->d;
    if (d->relax == GG_RELAX_NE_CHECK) k_check<GG_RELAX_NE_CHECK><<<grid, kBlock, 0, ctx->stream>>>(A, av, src_bits);
    else if (d->relax == GG_RELAX_GAP_CHECK) k_check<GG_RELAX_GAP_CHECK><<<grid, kBlock, 0, ctx->stream>>>(A, av, src_bits);
    else k_check<GG_RELAX_AHEAD_CHECK><<<grid, kBlock, 0, ctx->stream>>>(A, av, src_bits);
    GG_LAUNCHED(ctx);
    out->all = false;
    out->has_list = true;
    out->has_bitmap = true;
    out->host_valid = false;
    return GG_OK;
}

// Maximal independent set step (MISv.C:235-255 with the dfsaop_MIS
// relation of dsl/ast/dfsaop.h:49-230).  Over its in-edges (s, d), s != d:
// d becomes out (2) when some s is in (3); else a conditionally-in (1) d
// becomes undecided (0) when some s < d is undecided or conditionally in.
// The relation is order-independent per d; states of sources that change
// during the step are read as the reference's parallel step reads them,
// before or after the change (either way the rounds converge to the same
// set: the greedy one in vertex-id order); the loads bypass L1 (ld.global.cg)
// so that they see other SMs' changes as soon as L2 does.  A lane per destination of a
// 32-vertex word walks its first 32 in-edges, four loads in flight, and stops
// at an in source; the rest of longer rows is walked by the whole warp, one
// row after the other.  Recorded (EQ_ZERO): the destinations left undecided.
__global__ void __launch_bounds__(kBlock) k_mis(EmapArgs A, uint8_t *__restrict__ st,
                                                const uint32_t *__restrict__ dst_bits) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwords = (A.n + 31u) >> 5;
    const uint32_t nw = (gridDim.x * kBlock) >> 5;
    unsigned long long nv = 0, ne = 0, sc = 0;
    for (uint32_t w = (blockIdx.x * kBlock + threadIdx.x) >> 5; w < nwords; w += nw) {
        const uint32_t d = (w << 5) + lane;
        const bool act = d < A.n && (!dst_bits || ((dst_bits[w] >> lane) & 1u));
        uint8_t old = 0;
        uint64_t e = 0, end = 0;
        if (act) {
            old = st[d];
            e = A.in_off[d];
            end = A.in_off[d + 1];
        }
        // rows longer than the heavy-row threshold: k_mis_heavy_chunks / _finalize
        const bool heavy = act && A.heavy_T && end - e > A.heavy_T;
        if (heavy) end = e;
        const uint64_t beg = e;
        bool in = false, low = false;
        const uint64_t lim = min(end, e + 32);
        while (e < lim && !in) {
            uint32_t sv[4];
            const int cnt = (int)min((uint64_t)4, lim - e);
#pragma unroll
            for (int j = 0; j < 4; ++j) sv[j] = j < cnt ? __ldg(A.in_adj + e + j) : d;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (sv[j] == d) continue;  // self loop or unused slot
                const uint8_t u = __ldcg(st + sv[j]);
                in |= u == 3;
                low |= sv[j] < d && u < 2;
            }
            e += cnt;
        }
        unsigned pend = __ballot_sync(FULL, act && !in && e < end);
        while (pend) {
            const int j = __ffs(pend) - 1;
            pend &= pend - 1;
            const uint32_t dj = (w << 5) + j;
            const uint64_t ej = __shfl_sync(FULL, e, j), endj = __shfl_sync(FULL, end, j);
            bool inj = false, lowj = false;
            for (uint64_t base = ej; base < endj && !inj; base += 32) {
                bool hi = false, lo = false;
                if (base + lane < endj) {
                    const uint32_t s = __ldg(A.in_adj + base + lane);
                    if (s != dj) {
                        const uint8_t u = __ldcg(st + s);
                        hi = u == 3;
                        lo = s < dj && u < 2;
                    }
                }
                inj = __any_sync(FULL, hi);
                lowj = lowj || __any_sync(FULL, lo);
            }
            if ((int)lane == j) {
                in = in || inj;
                low = low || lowj;
            }
        }
        bool rec = false;
        if (act && !heavy) {
            const uint8_t nwv = in ? 2 : ((old == 1 && low) ? 0 : old);
            if (nwv != old) st[d] = nwv;
            rec = nwv == 0 && A.record == GG_RECORD_EQ_ZERO;
            sc += end - beg;
        }
        if (A.out_bits) {
            const unsigned bits = __ballot_sync(FULL, rec);
            if (lane == 0) A.out_bits[w] = bits;
            emit_out(A, rec, d, nv, ne);
        }
    }
    if (A.out_cnt) flush_counts<kBlock>(A, nv, ne, sc);
}

// The MIS relation over the long rows: a warp per chunk of a heavy row ORs
// "some source is in" (bit 0) and "some lower source is undecided or
// conditionally in" (bit 1) into the row's flag word; then a thread per heavy
// row applies the relation and records it.
__global__ void __launch_bounds__(256) k_mis_heavy_chunks(EmapArgs A, const uint8_t *__restrict__ st,
                                                          const uint32_t *__restrict__ dst_bits, HeavyRows H,
                                                          uint32_t *__restrict__ flags) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < H.nchunks; c += nw) {
        const uint32_t lo = H.crow[c];
        const uint32_t d = H.v[lo];
        if (dst_bits && !dev::bit_test(dst_bits, d)) continue;  // the same row for the whole warp
        const uint64_t rb = A.in_off[d], re = A.in_off[d + 1];
        const uint64_t e0 = rb + (c - H.first[lo]) * H.CH;
        const uint64_t e1 = min(e0 + H.CH, re);
        uint32_t f = 0;
        for (uint64_t base = e0; base < e1; base += 128) {
            uint32_t sv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint64_t e = base + j * 32 + lane;
                sv[j] = e < e1 ? __ldg(A.in_adj + e) : d;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (sv[j] == d) continue;
                const uint8_t u = __ldcg(st + sv[j]);
                f |= (u == 3 ? 1u : 0u) | ((sv[j] < d && u < 2) ? 2u : 0u);
            }
        }
        f = __reduce_or_sync(FULL, f);
        if (lane == 0 && f) atomicOr(flags + lo, f);
    }
}

__global__ void __launch_bounds__(256) k_mis_heavy_finalize(EmapArgs A, uint8_t *__restrict__ st,
                                                            const uint32_t *__restrict__ dst_bits, HeavyRows H,
                                                            const uint32_t *__restrict__ flags) {
    unsigned long long nv = 0, ne = 0;
    const uint32_t nth = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < H.nheavy; i0 += nth) {
        const uint32_t i = i0 + threadIdx.x;
        bool rec = false;
        uint32_t d = 0;
        if (i < H.nheavy) {
            d = H.v[i];
            if (!dst_bits || dev::bit_test(dst_bits, d)) {
                const uint8_t old = st[d];
                const uint32_t f = flags[i];
                const uint8_t nwv = (f & 1u) ? 2 : ((old == 1 && (f & 2u)) ? 0 : old);
                if (nwv != old) st[d] = nwv;
                rec = nwv == 0 && A.record == GG_RECORD_EQ_ZERO;
            }
        }
        if (rec && A.out_bits) atomicOr(A.out_bits + (d >> 5), 1u << (d & 31));
        if (A.out_b0) emit_out(A, rec, d, nv, ne);
    }
    if (A.out_cnt) flush_counts<256>(A, nv, ne, 0);
}

static gg_status mis_relax(gg_graph *g, const gg_emap_desc *d, gg_frontier *in, gg_frontier *out) {
    gg_ctx *ctx = g->ctx;
    if (d->a->t != GG_U8) return set_error(ctx, GG_ERR_ARG, "MIS relax: uint8 states");
    if (d->dst_filter != GG_FILTER_NONE && d->dst_filter != GG_FILTER_IN_FRONTIER)
        return set_error(ctx, GG_ERR_UNSUPPORTED, "MIS relax: dst filter NONE or IN_FRONTIER");
    if (d->record != GG_RECORD_NONE && d->record != GG_RECORD_EQ_ZERO)
        return set_error(ctx, GG_ERR_UNSUPPORTED, "MIS relax: record NONE or EQ_ZERO");
    if (d->dst_filter == GG_FILTER_NONE && in && !in->all)
        return set_error(ctx, GG_ERR_UNSUPPORTED, "MIS relax: the frontier filters destinations (IN_FRONTIER)");
    EmapArgs A;
    memset(&A, 0, sizeof(A));
    A.off = g->off;
    A.in_off = g->in_off;
    A.in_adj = g->in_adj;
    A.n = g->n;
    A.record = out ? d->record : GG_RECORD_NONE;
    const Tuning &t = tuning();
    A.smax = t.bin_small_max;
    A.mmax = t.bin_medium_max;
    const uint32_t *dst_bits = nullptr;
    if (d->dst_filter == GG_FILTER_IN_FRONTIER && in && !in->all) {
        GG_CHECK(frontier_ensure_bitmap(in));
        dst_bits = in->bitmap;
    }
    if (out) {
        GG_CHECK(frontier_alloc_bins(out));
        GG_CHECK(frontier_alloc_bitmap(out));
        GG_CHECK(frontier_reset_counts(out));
        A.out_bits = out->bitmap;
        A.out_b0 = out->bins[0];
        A.out_b1 = out->bins[1];
        A.out_b2 = out->bins[2];
        A.out_cnt = (unsigned long long *)out->d_cnt;
    }
    const HeavyRows &H = g->heavy;
    uint32_t *flags = nullptr;
    if (H.nchunks) {
        void *scr = nullptr;
        GG_CHECK(graph_scratch(g, ((size_t)H.nheavy + 1) * 4, &scr));
        flags = (uint32_t *)scr;
        GG_CUDA(ctx, cudaMemsetAsync(flags, 0, ((size_t)H.nheavy + 1) * 4, ctx->stream));
        A.heavy_T = H.T;
    }
    const uint64_t words = ((uint64_t)g->n + 31) / 32;
    k_mis<<<persistent_grid(ctx, words), kBlock, 0, ctx->stream>>>(A, (uint8_t *)d->a->d, dst_bits);
    GG_LAUNCHED(ctx);
    if (flags) {
        const unsigned cap = (unsigned)(ctx->sm_count * 8);
        const unsigned cb = (unsigned)std::min<uint64_t>((H.nchunks * 32 + 255) / 256, cap);
        k_mis_heavy_chunks<<<cb ? cb : 1, 256, 0, ctx->stream>>>(A, (const uint8_t *)d->a->d, dst_bits, H, flags);
        GG_LAUNCHED(ctx);
        const unsigned fb = (unsigned)std::min<uint64_t>((H.nheavy + 255) / 256, cap);
        k_mis_heavy_finalize<<<fb ? fb : 1, 256, 0, ctx->stream>>>(A, (uint8_t *)d->a->d, dst_bits, H, flags);
        GG_LAUNCHED(ctx);
    }
    if (out) {
        out->all = false;
        out->has_list = true;
        out->has_bitmap = true;
        out->host_valid = false;
    }
    return GG_OK;
}

gg_status edgemap_impl(gg_graph *g, const gg_emap_desc *d, gg_frontier *in, gg_frontier *out,
                       gg_emap_stats *stats) {
    gg_ctx *ctx = g->ctx;
    if (!d->a || d->a->g != g) return set_error(ctx, GG_ERR_ARG, "edgemap: relaxed property missing or of another graph");
    if (in && in->g != g) return set_error(ctx, GG_ERR_ARG, "edgemap: input frontier of another graph");
    if (out && out->g != g) return set_error(ctx, GG_ERR_ARG, "edgemap: output frontier of another graph");
    if (out && out == in) return set_error(ctx, GG_ERR_ARG, "edgemap: input and output frontier must differ");
    if (d->relax == GG_RELAX_ADD_GATHER) {
        if (d->record != GG_RECORD_NONE) return set_error(ctx, GG_ERR_UNSUPPORTED, "ADD_GATHER records no frontier");
        GG_CHECK(pr_edgemap_gather(g, d, in));
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            stats->variant = GG_VAR_PULL_DENSE;
            stats->nactv_in = g->n;
            stats->nacte_in = g->m;
            stats->scanned = g->m;
        }
        return GG_OK;
    }
    if (d->relax == GG_RELAX_MIS_U8) {
        GG_CHECK(mis_relax(g, d, in, out));
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            stats->variant = GG_VAR_PULL_DENSE;
        }
        return GG_OK;
    }
    if (d->relax >= GG_RELAX_NE_CHECK && d->relax <= GG_RELAX_AHEAD_CHECK) {
        if (d->record != GG_RECORD_REDUCTION && out)
            return set_error(ctx, GG_ERR_UNSUPPORTED, "check relaxes record by reduction");
        GG_CHECK(check_relax(g, d, in, out));
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            stats->variant = GG_VAR_PULL_DENSE;
        }
        return GG_OK;
    }
    const gg_dtype want = d->relax == GG_RELAX_MIN_PLUS1_I32 ? GG_I32 : GG_U32;
    if (d->relax < 0 ||
        (d->relax > GG_RELAX_SETIF_U32 && d->relax != GG_RELAX_OR_U32 && d->relax != GG_RELAX_COUNT_DOWN_U32))
        return set_error(ctx, GG_ERR_ARG, "unknown relax kind");
    if (d->relax == GG_RELAX_COUNT_DOWN_U32) {
        if (d->dst_filter != GG_FILTER_GT_CONST || d->dst_filter_k < 0 || d->dst_filter_k > 0xFFFFFFFFll)
            return set_error(ctx, GG_ERR_ARG, "COUNT_DOWN takes dst filter GT_CONST with the floor k");
        if (d->record != GG_RECORD_NONE && d->record != GG_RECORD_REDUCTION && d->record != GG_RECORD_AT_FLOOR)
            return set_error(ctx, GG_ERR_UNSUPPORTED, "COUNT_DOWN records NONE, REDUCTION or AT_FLOOR");
    } else if (d->record == GG_RECORD_AT_FLOOR) {
        return set_error(ctx, GG_ERR_UNSUPPORTED, "record AT_FLOOR belongs to COUNT_DOWN");
    }
    if (d->relax == GG_RELAX_OR_U32 && (!d->src || d->src->g != g || d->src->t != GG_U32))
        return set_error(ctx, GG_ERR_ARG, "OR_U32 needs a uint32 source property of g");
    if (d->a->t != want) return set_error(ctx, GG_ERR_ARG, "relaxed property has the wrong dtype");
    if (d->prev && (d->prev->t != want || d->prev->g != g)) return set_error(ctx, GG_ERR_ARG, "prev property mismatch");
    if (d->record == GG_RECORD_NE_PREV && !d->prev) return set_error(ctx, GG_ERR_ARG, "NE_PREV record needs prev");
    if (d->dst_filter < GG_FILTER_NONE || d->dst_filter > GG_FILTER_NE_CONST) return set_error(ctx, GG_ERR_ARG, "unknown dst filter");
    if (d->dst_filter != GG_FILTER_NONE && d->dst_filter_prop && d->dst_filter_prop != d->a)
        return set_error(ctx, GG_ERR_UNSUPPORTED, "dst filter on a property other than the relaxed one");
    if (d->threshold == GG_THRESH_FRAC && d->threshold_k <= 0) return set_error(ctx, GG_ERR_ARG, "frac threshold needs k > 0");

    uint64_t nactv = g->n, nacte = g->m;
    const bool all_in = in == nullptr || in->all;
    if (!all_in) {
        GG_CHECK(frontier_fetch_counts(in));
        nactv = in->h_cnt[FC_NACTV];
        nacte = in->h_cnt[FC_NACTE];
    }
    int variant = d->variant;
    if (variant == GG_VAR_AUTO) {
        bool can_exit = d->dst_filter != GG_FILTER_NONE;
        if (all_in) {
            variant = GG_VAR_PULL_DENSE;
        } else if (d->threshold == GG_THRESH_LEARNED) {
            variant = learned_select(g, nactv, nacte, 0, can_exit);
        } else {
            variant = threshold_sparse(d->threshold, d->threshold_k, nactv, nacte, g->m)
                          ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
        }
    }
    if (all_in && (variant == GG_VAR_PUSH_SPARSE || variant == GG_VAR_PUSH_MERGE) && !in)
        variant = GG_VAR_PUSH_DENSE;
    if (!all_in && nactv == 0) {
        // empty input: empty output, nothing to launch
        if (out) GG_CHECK(gg_frontier_clear(out));
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            stats->variant = variant;
        }
        return GG_OK;
    }
    gg_status s;
    ctx->time_kernels = stats != nullptr;
    if (stats) cudaEventRecord(ctx->evk0, ctx->stream);  // defined start even if nothing launches
    switch (d->relax) {
    case GG_RELAX_MIN_PLUS1_I32: s = launch_variant<GG_RELAX_MIN_PLUS1_I32>(g, d, in, out, variant); break;
    case GG_RELAX_MIN_U32: s = launch_variant<GG_RELAX_MIN_U32>(g, d, in, out, variant); break;
    case GG_RELAX_OR_U32: s = launch_variant<GG_RELAX_OR_U32>(g, d, in, out, variant); break;
    case GG_RELAX_COUNT_DOWN_U32: s = launch_variant<GG_RELAX_COUNT_DOWN_U32>(g, d, in, out, variant); break;
    default: s = launch_variant<GG_RELAX_SETIF_U32>(g, d, in, out, variant); break;
    }
    if (stats && s == GG_OK) cudaEventRecord(ctx->evk1, ctx->stream);
    ctx->time_kernels = false;
    GG_CHECK(s);
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        GG_CUDA(ctx, cudaEventSynchronize(ctx->evk1));
        float kms = 0;
        cudaEventElapsedTime(&kms, ctx->evk0, ctx->evk1);
        stats->kernel_ms = kms;
        stats->variant = variant;
        stats->nactv_in = nactv;
        stats->nacte_in = nacte;
        if (out && d->record != GG_RECORD_NONE) {
            GG_CHECK(frontier_fetch_counts(out));
            stats->scanned = out->h_cnt[FC_SCANNED];
            stats->nactv_out = out->h_cnt[FC_NACTV];
            stats->nacte_out = out->h_cnt[FC_NACTE];
        }
    }
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Drivers
// ---------------------------------------------------------------------------
struct RunTimer {
    gg_ctx *ctx;
    explicit RunTimer(gg_ctx *c) : ctx(c) { cudaEventRecord(ctx->ev0, ctx->stream); }
    double stop() {
        cudaEventRecord(ctx->ev1, ctx->stream);
        cudaEventSynchronize(ctx->ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        return ms;
    }
};

static gg_status get_tmp_frontiers(gg_graph *g, gg_frontier **a, gg_frontier **b) {
    for (auto &f : g->tmp_front)
        if (!f) GG_CHECK(gg_frontier_create(g, &f));
    *a = g->tmp_front[0];
    *b = g->tmp_front[1];
    return GG_OK;
}

// Per-graph cached temporaries (prev copies, default outputs): created on
// first use, reused by later runs, freed with the graph.
static gg_status tmp_prop(gg_graph *g, int slot, gg_dtype t, gg_prop **out) {
    gg_prop *&p = g->tmp_prop[slot];
    if (p && p->t != t) {
        gg_prop_destroy(p);
        p = nullptr;
    }
    if (!p) GG_CHECK(gg_prop_create(g, t, &p));
    *out = p;
    return GG_OK;
}

static void record_iter(gg_run_stats *st, int it, const gg_emap_stats &es) {
    if (!st || it >= GG_MAX_ITERS) return;
    st->variant[it] = es.variant;
    st->nactv[it] = es.nactv_in;
    st->nacte[it] = es.nacte_in;
    st->scanned[it] = es.scanned;
    st->iter_ms[it] = es.kernel_ms;
    st->kernel_ms[it] = es.kernel_ms;
    st->scanned_edges += es.scanned;
}

static void default_opts(const gg_run_opts *o, gg_run_opts *r, int thresh, int k) {
    if (o) {
        *r = *o;
    } else {
        r->threshold = thresh;
        r->threshold_k = k;
        r->variant = GG_VAR_AUTO;
        r->collect_stats = 0;
    }
}

// Candidate lists live for one driver run.
struct CandScope {
    gg_graph *g;
    explicit CandScope(gg_graph *gr) : g(gr) {}
    gg_status open() {
        CandLists &c = g->cand;
        if (!c.list[0]) {
            for (auto &l : c.list) GG_CUDA(g->ctx, cudaMalloc(&l, ((size_t)g->n + 1) * 4));
            GG_CUDA(g->ctx, cudaMalloc(&c.cnt, 2 * sizeof(uint64_t)));
        }
        c.cur = 0;
        c.valid = false;
        c.host_n = UINT64_MAX;
        g->cand_active = true;
        return GG_OK;
    }
    ~CandScope() { g->cand_active = false; }
};

// Device-driven loop (analytic bit set in the `persistent` knob) unless a
// variant only the host loop provides is asked for.
// The learned selector and timing collection run device-driven always.
static bool use_persistent(const gg_graph *g, const gg_run_opts &opt, int analytic_bit) {
    if (opt.threshold == GG_THRESH_LEARNED || g->force_iter >= 0) return true;
    return (tuning().persistent & analytic_bit) != 0;
}

// Generic frontier loop shared by the three analytics.
static gg_status frontier_loop(gg_graph *g, gg_emap_desc &desc, gg_frontier *F, gg_frontier *O,
                               const gg_run_opts &opt, gg_run_stats *st, bool level_k,
                               int *iters_out) {
    CandScope cs(g);
    GG_CHECK(cs.open());
    int iter = 0;
    for (;;) {
        GG_CHECK(frontier_fetch_counts(F));
        if (F->h_cnt[FC_NACTV] == 0 && !F->all) break;
        if (st) {
            st->vertices_reached += F->h_cnt[FC_NACTV];
            st->edges_reached += F->h_cnt[FC_NACTE];
        }
        if (level_k) desc.dst_filter_k = iter + 1;
        gg_emap_stats es;
        GG_CHECK(edgemap_impl(g, &desc, F, O, opt.collect_stats ? &es : nullptr));
        if (opt.collect_stats) record_iter(st, iter, es);
        std::swap(F, O);
        ++iter;
        if (iter > (int)g->n + 2) return set_error(g->ctx, GG_ERR_STATE, "frontier loop did not converge");
    }
    *iters_out = iter;
    return GG_OK;
}

// ---------------------------------------------------------------------------
// Graph-driven BFS levels: the host loop's kernels, decided on the device
// ---------------------------------------------------------------------------
// The host-driven loop waits for every iteration's frontier counts before it
// picks push or pull and launches the next kernels; on R-MAT scale 24 those
// round trips are about a third of a BFS.  Here one CUDA graph holds a whole
// run: a WHILE conditional node repeats
//     decide -> IF(push){list, push} , IF(pull){pull} -> post
// The one-warp decide kernel reads the frontier counts on the device, applies
// the threshold (api.h:130-222) and writes the step's arguments to device
// memory; the step kernels run the same bodies as the host-launched kernels
// on fixed grids and read their arguments there; post recycles the consumed
// frontier and sets the loop condition.  Every kernel keeps the normal L1
// path (no grid-wide waits), and the host waits once, at the end.
struct GFront {
    uint32_t *bins[NBINS];
    uint32_t *bitmap;
    unsigned long long *cnt;
};

struct GCtl {
    EmapArgs A;  // this step's traversal arguments
    Op<GG_RELAX_MIN_PLUS1_I32> op;
    int variant;  // GG_VAR_PUSH_SPARSE / GG_VAR_PULL_DENSE, -1: finished
    int need_list, need_bitmap, use_first;
    int cur, iter, max_iters, iterations;
    int has_list[2], has_bitmap[2];
    GFront f[2];
    // per-run configuration
    int32_t *level, *prev;
    uint32_t root, n;
    uint64_t m;
    int threshold, threshold_k;
    int handoff_iter;  // > 0: after this many iterations the run leaves the graph (handed_off = 1)
    int handed_off;
    int clr;  // written by the step kernel: 1 + the frontier whose bitmap `next` clears, or 0
    const __nv_bfloat16 *sel_w;  // learned selector weights (bfloat16), or null: the threshold decides
    float gini;
    float sel_x4, sel_x9;  // the selector's per-graph features (average degree, size)
    // last network evaluation: reused while the frontier counts stay within 1/16
    unsigned long long sel_nactv, sel_nacte, sel_unr;
    int sel_iter, sel_push, sel_valid;
    uint32_t smax, mmax, large_ch, sm_count;
    int pull_k, push_k;
    const uint64_t *off, *in_off, *word_prefix;
    const uint32_t *adj, *in_adj;
    const uint4 *first_in;
    const uint2 *first1;
    int rec_n;
    int lazy_off;
    int fresh_ok;                     // a pull after a pull skips its candidates' level loads (knob pull_fresh)
    uint32_t stage_words;             // bitmap words each pull CTA stages in shared memory (knob pull_stage)
    int split;                        // pulls in two passes (pull_body PASS 1 / 2)
    int flat;                         // the loop body is one chain of kernels (no step conditionals)
    int need_chunks;                  // this push step needs k_g_chunks
    uint32_t *rest;                   // split pull: the second pass's rows
    unsigned long long rest_n;
    const uint32_t *nonisolated;
    const unsigned long long *nonisolated_n;
    uint32_t *cand[2];
    uint64_t *chunk_first;  // large-bin chunk prefix (k_g_chunks), chunk_cap entries
    uint64_t chunk_cap;
    unsigned long long *cand_n;  // [2]
    int cand_cur, cand_valid;
    // records
    unsigned long long reached_v, reached_e;
    unsigned stage_timeouts;  // pull CTAs whose bitmap staging did not complete in time (probes went to L2)
    cudaGraphConditionalHandle h_while, h_push, h_pull, h_list, h_bits, h_chunks;
    // per-iteration records (after the head: `next` works on a shared-memory
    // copy of everything before them)
    alignas(16) int variants[GG_MAX_ITERS];
    unsigned long long nactv[GG_MAX_ITERS], nacte[GG_MAX_ITERS], scanned[GG_MAX_ITERS];
    unsigned long long t_ns[GG_MAX_ITERS + 1];
    // span of each step's traversal kernel (first CTA start, last CTA end)
    unsigned long long kt0[GG_MAX_ITERS], kt1[GG_MAX_ITERS];
};
constexpr size_t kCtlHead = offsetof(GCtl, variants);
static_assert(kCtlHead % 16 == 0 && kCtlHead <= 4096, "control block head: whole 16-byte words, small");

__device__ __forceinline__ unsigned long long g_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool d_threshold_sparse(int kind, int k, uint64_t nactv, uint64_t nacte, uint64_t m) {
    switch (kind) {
    case GG_THRESH_ALWAYS_SPARSE: return true;
    case GG_THRESH_ALWAYS_DENSE: return false;
    case GG_THRESH_FRAC: return (float)(nactv + nacte) <= (float)m / (float)(100.0 / (float)k);
    default: return (nactv + nacte) <= (m / 20);
    }
}

__device__ void decide_step(GCtl *c, GCtl *h, const mlp::LaneWeights *lw = nullptr);

// Programmatic dependent launch (knob graph_pdl): the loop body's kernels
// are joined by programmatic edges, so each is launched while its
// predecessor still runs; it lets its own successor launch at once and waits
// here for its predecessor's completion (and memory) before it reads the
// control block.  Without such an edge both instructions do nothing.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__global__ void k_g_init(GCtl *c) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < GG_MAX_ITERS; i += nth) {
        c->kt0[i] = ~0ull;
        c->kt1[i] = 0ull;
    }
    const int32_t inf = (int32_t)c->n + 1;
    // (prev is not used by level-synchronous steps: only level is filled)
    for (uint64_t v = tid; v < c->n; v += nth) c->level[v] = v == c->root ? 0 : inf;
    const uint64_t words = ((uint64_t)c->n + 31) / 32;
    for (uint64_t w = tid; w < words; w += nth) {
        c->f[0].bitmap[w] = w == (c->root >> 5) ? 1u << (c->root & 31) : 0u;
        c->f[1].bitmap[w] = 0u;
    }
    if (tid == 0) {
        for (int i = 0; i < FC_WORDS; ++i) {
            c->f[0].cnt[i] = 0;
            c->f[1].cnt[i] = 0;
        }
        const uint64_t deg = c->off[c->root + 1] - c->off[c->root];
        const int b = deg <= c->smax ? 0 : (deg <= c->mmax ? 1 : 2);
        c->f[0].bins[b][0] = c->root;
        c->f[0].cnt[FC_BIN0 + b] = 1;
        c->f[0].cnt[FC_NACTV] = 1;
        c->f[0].cnt[FC_NACTE] = deg;
        c->has_list[0] = 1;
        c->has_list[1] = 0;
        c->has_bitmap[0] = 1;
        c->has_bitmap[1] = 0;
        c->cur = 0;
        c->iter = 0;
        c->iterations = 0;
        c->cand_valid = 0;
        c->cand_cur = 0;
        c->sel_valid = 0;
        c->handed_off = 0;
        c->clr = 0;
        c->reached_v = 0;
        c->reached_e = 0;
        c->stage_timeouts = 0;
        c->variant = -1;
        c->t_ns[0] = g_now();
    }
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        __syncwarp();
        decide_step(c, c);  // the first step's decision (warp 0 of CTA 0)
    }
}

// the decision of the step about to run (one thread): reads the frontier
// counts, writes the step's arguments, sets the branch and loop conditions
// Called by the 32 lanes of one warp (the network is evaluated by a warp);
// lane 0 writes the decision.
__device__ void decide_step(GCtl *c, GCtl *h, const mlp::LaneWeights *lw) {
    const uint32_t lane = threadIdx.x & 31u;
    const GFront F = h->f[h->cur], O = h->f[h->cur ^ 1];
    const unsigned long long nactv = F.cnt[FC_NACTV], nacte = F.cnt[FC_NACTE];
    const int iter = h->iter;
    const bool handoff = h->handoff_iter > 0 && iter >= h->handoff_iter;
    if (nactv == 0 || iter >= h->max_iters || handoff) {
        if (lane != 0) return;
        // a long run of small steps continues in the device-driven traversal
        h->handed_off = nactv != 0 && iter < h->max_iters;
        h->variant = -1;
        h->iterations = iter;
        // kernels of the loop body still to run (an unrolled body) do nothing
        h->need_list = 0;
        h->need_bitmap = 0;
        h->need_chunks = 0;
        if (!h->flat) {
            cudaGraphSetConditional(h->h_push, 2u);  // the step switch: no body
            cudaGraphSetConditional(h->h_list, 0);
            cudaGraphSetConditional(h->h_bits, 0);
            cudaGraphSetConditional(h->h_chunks, 0);
        }
        cudaGraphSetConditional(h->h_while, 0);
        return;
    }
    bool push = d_threshold_sparse(h->threshold, h->threshold_k, nactv, nacte, h->m);
    const unsigned long long unr_c = h->reached_v < h->n ? h->n - h->reached_v : 0ull;
    const auto close = [](unsigned long long a, unsigned long long b) {
        const unsigned long long d = a > b ? a - b : b - a, mx = a > b ? a : b;
        return d * 16 <= mx;
    };
    if (h->sel_w && h->sel_valid && close(nactv, h->sel_nactv) && close(nacte, h->sel_nacte) &&
        close(unr_c, h->sel_unr) && min(iter, 255) - h->sel_iter < 8) {
        push = h->sel_push != 0;  // the last evaluation still applies
    } else if (h->sel_w) {
        // learned choice between the two variants this driver runs: the
        // threshold's stands unless the network predicts a clear gain.
        // Features in single precision (the graph's constant ones come from
        // the host): the network's inputs are floats either way.
        const float n = (float)h->n, m = (float)h->m, fv = (float)nactv, fe = (float)nacte;
        float x[GG_SEL_FEATURES];
        x[0] = log2f(1.0f + fv) / 32;
        x[1] = log2f(1.0f + fe) / 40;
        x[2] = log2f(1.0f + (float)unr_c) / 32;
        x[3] = log2f(1.0f + (float)min(iter, 255)) / 8;
        x[4] = h->sel_x4;
        x[5] = h->gini;
        x[6] = n > 0 ? fv / n : 0.0f;
        x[7] = m > 0 ? fe / m : 0.0f;
        x[8] = fminf(4.0f, m > 0 ? (fv + fe) / m : 0.0f);
        x[9] = h->sel_x9;
        float o[GG_SEL_VARIANTS];
        if (lw) {
            mlp::warp_forward_regs(*lw, x, o);
        } else {
            float z1, a1, z2, a2;
            mlp::warp_forward(h->sel_w, x, o, z1, a1, z2, a2);
        }
        const int tv = push ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
        const int best = o[GG_VAR_PUSH_SPARSE] < o[GG_VAR_PULL_DENSE] ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
        if (o[best] < o[tv] - mlp::kSelMargin) push = best == GG_VAR_PUSH_SPARSE;
        __syncwarp();
        if (lane == 0) {
            h->sel_nactv = nactv;
            h->sel_nacte = nacte;
            h->sel_unr = unr_c;
            h->sel_iter = min(iter, 255);
            h->sel_push = push;
            h->sel_valid = 1;
        }
    }
    if (lane != 0) return;
    if (iter < GG_MAX_ITERS) {
        c->variants[iter] = push ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
        c->nactv[iter] = nactv;
        c->nacte[iter] = nacte;
    }
    h->reached_v += nactv;
    h->reached_e += nacte;
    EmapArgs A;
    memset(&A, 0, sizeof(A));
    A.off = h->off;
    A.adj = h->adj;
    A.in_off = h->in_off;
    A.in_adj = h->in_adj;
    A.n = h->n;
    A.record = GG_RECORD_NE_PREV;
    A.smax = h->smax;
    A.mmax = h->mmax;
    A.K = push ? h->push_k : h->pull_k;
    A.word_prefix = h->word_prefix;
    A.first_in = push ? nullptr : h->first_in;
    A.first1 = push ? nullptr : h->first1;
    A.rec_n = h->rec_n;
    A.lazy_off = h->lazy_off;
    // candidates left unsettled by the pull just run are all unvisited
    A.fresh = !push && h->fresh_ok && h->cand_valid && h->variant == GG_VAR_PULL_DENSE;
    A.out_b0 = O.bins[0];
    A.out_b1 = O.bins[1];
    A.out_b2 = O.bins[2];
    A.out_cnt = O.cnt;
    A.in_bits = F.bitmap;
    A.in_b0 = F.bins[0];
    A.in_b1 = F.bins[1];
    A.in_b2 = F.bins[2];
    A.large_ch = h->large_ch;
    if (!push) {
        const int cc = h->cand_cur;
        A.cand = h->cand_valid ? h->cand[cc] : h->nonisolated;
        A.cand_n = h->cand_valid ? h->cand_n + cc : h->nonisolated_n;
        A.cand_out = h->cand[cc ^ 1];
        A.cand_out_n = h->cand_n + (cc ^ 1);
        h->cand_n[cc ^ 1] = 0;
        A.out_bits = O.bitmap;  // cleared by the post kernel of the step that consumed it
        // split when the frontier holds less than half the edges: then most
        // candidates' first two in-edges leave them open, and a warp of the
        // single pass waits for its lanes' long rows
        if (h->split && 2 * nacte < h->m) {
            A.rest_out = h->rest;
            A.rest_out_n = &c->rest_n;
            h->rest_n = 0;
        }
    }
    h->A = A;
    Op<GG_RELAX_MIN_PLUS1_I32> op;
    op.a = h->level;
    op.prev = h->prev;
    op.filter = GG_FILTER_GT_CONST;
    op.fk = iter + 1;
    op.level_sync = 1;
    h->op = op;
    h->variant = push ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
    h->need_list = push && !h->has_list[h->cur];
    h->use_first = 0;
    // a large bin too big for a CTA's shared table gets its chunk prefix from
    // k_g_chunks (its size is known here unless the list is still to be built)
    const bool chunks = push && (h->need_list || F.cnt[FC_BIN2] > kLargeLocal);
    h->need_chunks = chunks;
    h->need_bitmap = !push && !h->has_bitmap[h->cur];
    if (!h->flat) {
        cudaGraphSetConditional(h->h_chunks, chunks ? 1u : 0u);
        cudaGraphSetConditional(h->h_push, push ? 0u : 1u);  // the step switch: push or pull body
        cudaGraphSetConditional(h->h_list, h->need_list ? 1u : 0u);
        cudaGraphSetConditional(h->h_bits, h->need_bitmap ? 1u : 0u);
    }
    cudaGraphSetConditional(h->h_while, 1u);
}

// a frontier held as a bitmap only (after a pull) gets its binned list
__global__ void __launch_bounds__(256) k_g_tolist(GCtl *c) {
    chain_enter();
    if (!c->need_list) return;
    const GFront F = c->f[c->cur];
    __shared__ uint32_t sb[3][8][256];
    const uint32_t wib = threadIdx.x >> 5;
    dev::WarpAppender<256> ap0{sb[0][wib], 0, F.bins[0], F.cnt + FC_BIN0};
    dev::WarpAppender<256> ap1{sb[1][wib], 0, F.bins[1], F.cnt + FC_BIN1};
    dev::WarpAppender<256> ap2{sb[2][wib], 0, F.bins[2], F.cnt + FC_BIN2};
    unsigned long long nv = 0, ne = 0;  // the counts are known already
    dev::bitmap_to_bins(F.bitmap, c->n, c->off, c->smax, c->mmax, ap0, ap1, ap2, nv, ne);
    ap0.flush();
    ap1.flush();
    ap2.flush();
}

// the push step: the partition of the fixed grid over the three bins is
// derived by every CTA from the same device counts
// The step's arguments are copied once per CTA into shared memory: the
// bodies then read them like kernel parameters (cheap broadcast loads), with
// no register copy to spill and no global reloads after the kernel's stores.
__device__ __noinline__ void g_push_setup(GCtl *c, uint32_t cap, EmapArgs *sA, Op<GG_RELAX_MIN_PLUS1_I32> *sOp,
                                          uint32_t *s_nl, uint32_t *s_nm);

// Span of a step's traversal kernel: the first CTA to start and the last to
// finish (the last warp of each CTA records its end) stamp the step's record.
__device__ __forceinline__ void kspan_start(GCtl *c, int it) {
    if (it < GG_MAX_ITERS) atomicMin(&c->kt0[it], g_now());
}
__device__ __forceinline__ void kspan_end(GCtl *c, int it, unsigned *s_done) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0 && atomicAdd(s_done, 1u) == blockDim.x / 32 - 1 && it < GG_MAX_ITERS)
        atomicMax(&c->kt1[it], g_now());
}

template <int MINB>  // resident CTAs per SM it is compiled for (knob push_ctas)
__global__ void __launch_bounds__(kBlock, MINB) k_g_push(GCtl *c) {
    chain_enter();
    if (c->variant != GG_VAR_PUSH_SPARSE) return;
    __shared__ EmapArgs sA;
    __shared__ Op<GG_RELAX_MIN_PLUS1_I32> sOp;
    __shared__ uint32_t s_nl, s_nm;
    __shared__ int s_it;
    __shared__ unsigned s_done;
    if (threadIdx.x == 0) {
        s_it = c->iter;
        s_done = 0;
        kspan_start(c, s_it);
        g_push_setup(c, gridDim.x, &sA, &sOp, &s_nl, &s_nm);
        // the pushed frontier's bitmap, if a pull made it, is cleared after
        if (blockIdx.x == 0) c->clr = c->has_bitmap[c->cur] ? c->cur + 1 : 0;
    }
    __syncthreads();
    push_binned_body<GG_RELAX_MIN_PLUS1_I32, kBlock>(sA, sOp, s_nl, s_nm);
    kspan_end(c, s_it, &s_done);
}

// one thread per CTA: the push arguments and the partition of the grid
__device__ __noinline__ void g_push_setup(GCtl *c, uint32_t cap, EmapArgs *sA, Op<GG_RELAX_MIN_PLUS1_I32> *sOp,
                                          uint32_t *s_nl, uint32_t *s_nm) {
    {
        EmapArgs A = c->A;
        const GFront F = c->f[c->cur];
        A.c0 = (uint32_t)F.cnt[FC_BIN0];
        A.c1 = (uint32_t)F.cnt[FC_BIN1];
        A.c2 = (uint32_t)F.cnt[FC_BIN2];
        A.merge_med = A.c1 && A.c1 + A.c2 <= kLargeLocal && A.c1 < c->sm_count;
        A.large_as_med = !A.merge_med && A.c2 > kLargeLocal;
        if (A.c2 > kLargeLocal && c->use_first) {  // chunk prefix built by k_g_chunks
            A.large_first = c->chunk_first;
            A.large_as_med = 0;
        }
        const uint64_t nacte = F.cnt[FC_NACTE];
        uint32_t nl = 0;
        if ((A.c2 && !A.large_as_med) || A.merge_med)
            nl = (uint32_t)min((uint64_t)cap, nacte / A.large_ch + A.c2 + (A.merge_med ? A.c1 : 0u));
        const uint32_t cmed = A.merge_med ? 0u : A.c1 + (A.large_as_med ? A.c2 : 0u);
        uint32_t nm = (uint32_t)min((uint64_t)cap, ((uint64_t)cmed + kBlock / 32 - 1) / (kBlock / 32));
        const uint32_t ns = (uint32_t)min((uint64_t)cap, ((uint64_t)A.c0 + kBlock - 1) / kBlock);
        // demands above the grid: every path keeps a share in proportion, at
        // least one CTA each, the small bin takes what the others leave
        const uint64_t tot = (uint64_t)nl + nm + ns;
        if (tot > cap) {
            nl = nl ? max(1u, (uint32_t)((uint64_t)nl * cap / tot)) : 0u;
            nm = nm ? max(1u, (uint32_t)((uint64_t)nm * cap / tot)) : 0u;
            while (ns && nl + nm >= cap) {  // leave one CTA at least for the small bin
                if (nl > 1) --nl; else if (nm > 1) --nm; else break;
            }
        }
        *sA = A;
        *sOp = c->op;
        *s_nl = nl;
        *s_nm = nm;
    }
}

// a frontier held as a list only (after a push) gets its bitmap (clear since
// the frontier's buffer was last consumed)
__global__ void k_g_tobitmap(GCtl *c) {
    chain_enter();
    if (!c->need_bitmap) return;
    const GFront F = c->f[c->cur];
    const unsigned long long c0 = F.cnt[FC_BIN0], c1 = F.cnt[FC_BIN1], c2 = F.cnt[FC_BIN2];
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < c0 + c1 + c2; i += nth) {
        const uint32_t v = i < c0 ? F.bins[0][i] : (i < c0 + c1 ? F.bins[1][i - c0] : F.bins[2][i - c0 - c1]);
        atomicOr(F.bitmap + (v >> 5), 1u << (v & 31));
    }
}

// Frontier bitmap staging (knob pull_stage): thread 0 copies the bitmap's
// first `words` words (rounded down to 16-byte units) into the CTA's dynamic
// shared memory with one bulk copy (cp.async.bulk, completion counted on an
// mbarrier); every thread waits on the barrier at most kStageSpin polls.
// Returns the number of vertex ids the copy covers, the same for every
// thread; 0 when nothing was staged or the wait ran out (then every probe
// goes to L2 and the copy is waited for again before the CTA exits).
constexpr uint32_t kStageSpin = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool stage_poll(uint32_t bar, uint32_t limit) {
    uint32_t ok = 0;
    for (uint32_t i = 0; i < limit && !ok; ++i)
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(bar)
                     : "memory");
    return ok != 0;
}

__device__ uint32_t stage_bitmap(const uint32_t *src, uint64_t src_words, uint32_t words, uint32_t *dst,
                                 unsigned long long *bar, bool *pending) {
    words = (uint32_t)min((uint64_t)words, src_words) & ~3u;
    *pending = false;
    if (words == 0 || ((uintptr_t)src & 15u) != 0) return 0;
    const uint32_t b = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(words * 4u) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32(dst)),
                     "l"(src), "r"(words * 4u), "r"(b)
                     : "memory");
    }
    __syncthreads();  // the barrier is initialised before any thread polls it
    const bool ok = __syncthreads_and(stage_poll(b, kStageSpin)) != 0;
    *pending = !ok;
    return ok ? words * 32u : 0u;
}

// a CTA whose staging wait ran out waits (bounded) for the copy before it
// exits, and counts the event
__device__ __forceinline__ void stage_finish(GCtl *c, unsigned long long *bar, bool pending) {
    if (!pending) return;
    if (threadIdx.x == 0) {
        atomicAdd(&c->stage_timeouts, 1u);
        stage_poll(smem_u32(bar), kStageSpin);
    }
    __syncthreads();
}

// MINB: resident CTAs per SM the kernel is compiled for (knob pull_ctas):
// 6 caps it at 40 registers, with spills in the row loop; 4 gives 64, none
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_g_pull(GCtl *c) {
    chain_enter();
    if (c->variant != GG_VAR_PULL_DENSE) return;
    extern __shared__ __align__(128) uint32_t s_stage[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ EmapArgs sA;
    __shared__ Op<GG_RELAX_MIN_PLUS1_I32> sOp;
    __shared__ int s_it;
    __shared__ unsigned s_done;
    if (threadIdx.x == 0) {
        s_it = c->iter;
        s_done = 0;
        kspan_start(c, s_it);
        sA = c->A;
        sOp = c->op;
        if (blockIdx.x == 0) c->clr = c->cur + 1;  // a pulled frontier has a bitmap to clear after
    }
    __syncthreads();
    __shared__ PullSmem<kBlock, true> sm;
    if (c->stage_words) {
        bool pending;
        const uint32_t sn = stage_bitmap(sA.in_bits, ((uint64_t)sA.n + 31) / 32, c->stage_words, s_stage, &s_bar,
                                         &pending);
        if (sA.rest_out) pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock, 1, true>(sA, sOp, sm, s_stage, sn);
        else pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock, 0, true>(sA, sOp, sm, s_stage, sn);
        stage_finish(c, &s_bar, pending);
    } else if (sA.rest_out) {
        pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock, 1>(sA, sOp, sm);
    } else {
        pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock>(sA, sOp, sm);
    }
    kspan_end(c, s_it, &s_done);
}

// second pass of a split pull: the rows the first pass left open, from
// their third in-edge
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_g_pull2(GCtl *c) {
    chain_enter();
    if (c->variant != GG_VAR_PULL_DENSE || !c->A.rest_out) return;
    extern __shared__ __align__(128) uint32_t s_stage[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ EmapArgs sA;
    __shared__ Op<GG_RELAX_MIN_PLUS1_I32> sOp;
    __shared__ int s_it;
    __shared__ unsigned s_done;
    if (threadIdx.x == 0) {
        s_it = c->iter;
        s_done = 0;
        kspan_start(c, s_it);
        sA = c->A;
        sA.cand = c->rest;
        sA.cand_n = &c->rest_n;
        sA.first_in = nullptr;
        sA.first1 = nullptr;
        sA.rest_out = nullptr;
        sA.fresh = c->fresh_ok;  // rows the first pass left open are unvisited
        sOp = c->op;
    }
    __syncthreads();
    __shared__ PullSmem<kBlock, false> sm;
    if (c->stage_words) {
        bool pending;
        const uint32_t sn = stage_bitmap(sA.in_bits, ((uint64_t)sA.n + 31) / 32, c->stage_words, s_stage, &s_bar,
                                         &pending);
        pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock, 2, true>(sA, sOp, sm, s_stage, sn);
        stage_finish(c, &s_bar, pending);
    } else {
        pull_body<GG_RELAX_MIN_PLUS1_I32, true, true, kBlock, 2>(sA, sOp, sm);
    }
    kspan_end(c, s_it, &s_done);
}

__device__ void g_bookkeep(GCtl *c, GCtl *h);

// After a step: every CTA clears the consumed frontier's bitmap for its next
// use as an output (when the step, or the conversion for a pull, set one:
// the step kernel names it in `clr`, a field nothing here writes); warp 0 of
// CTA 0 meanwhile does the step's bookkeeping (thread 0) and the next step's
// decision, which touch no bitmap.
__global__ void __launch_bounds__(256) k_g_next(GCtl *c) {
    chain_enter();
    const int clr = c->clr;
    if (clr) {
        uint32_t *bm = c->f[clr - 1].bitmap;
        const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
        const uint64_t words = ((uint64_t)c->n + 31) / 32;
        for (uint64_t w = tid; w < words; w += nth) bm[w] = 0u;
    }
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    if (c->variant < 0) {
        if (threadIdx.x == 0) cudaGraphSetConditional(c->h_while, 0);
        return;
    }
    // the control block's head (everything but the per-iteration records)
    // is read into shared memory in one round of 16-byte loads, the
    // bookkeeping and the decision work on that copy, and it is written
    // back: one global round trip instead of one per dependent field
    __shared__ __align__(16) unsigned char s_head[kCtlHead];
    const uint32_t lane = threadIdx.x;
    const __nv_bfloat16 *sel_w = c->sel_w;
    for (uint32_t i = lane; i < kCtlHead / 16; i += 32) ((uint4 *)s_head)[i] = ((const uint4 *)c)[i];
    // the selector's weights, if any, are loaded now and arrive while the
    // bookkeeping and the frontier counts are read
    mlp::LaneWeights lw;
    if (sel_w) mlp::load_lane(sel_w, lw);
    __syncwarp();
    GCtl *h = (GCtl *)s_head;
    if (lane == 0) g_bookkeep(c, h);
    __syncwarp();
    decide_step(c, h, sel_w ? &lw : nullptr);  // an empty frontier or the iteration bound ends the loop
    __syncwarp();
    for (uint32_t i = lane; i < kCtlHead / 16; i += 32) ((uint4 *)c)[i] = ((const uint4 *)s_head)[i];
}

// bookkeeping of the step that ran (one thread)
__device__ void g_bookkeep(GCtl *c, GCtl *h) {
    {
    const int cur = h->cur;
    const GFront F = h->f[cur], O = h->f[cur ^ 1];
    const int iter = h->iter;
    if (iter < GG_MAX_ITERS) c->scanned[iter] = O.cnt[FC_SCANNED];
    for (int i = 0; i < FC_WORDS; ++i) F.cnt[i] = 0;
    h->has_list[cur ^ 1] = h->variant == GG_VAR_PUSH_SPARSE;
    h->has_list[cur] = 0;
    h->has_bitmap[cur ^ 1] = h->variant == GG_VAR_PULL_DENSE;
    h->has_bitmap[cur] = 0;
    if (h->variant == GG_VAR_PULL_DENSE) {
        h->cand_valid = 1;
        h->cand_cur ^= 1;
    }
    h->cur = cur ^ 1;
    h->iter = iter + 1;
    if (iter + 1 <= GG_MAX_ITERS) c->t_ns[iter + 1] = g_now();
    }
}

// Chunk prefix of a large bin of more than kLargeLocal rows (one CTA of
// 1024 threads, tiles of 1024 rows): first[i] = chunks of rows before i.
__global__ void __launch_bounds__(1024) k_g_chunks(GCtl *c) {
    __shared__ unsigned long long s_warp[32];
    __shared__ unsigned long long s_base;
    chain_enter();
    if (c->variant != GG_VAR_PUSH_SPARSE || !c->need_chunks) return;
    const GFront F = c->f[c->cur];
    const uint64_t c2 = F.cnt[FC_BIN2];
    if (c2 <= kLargeLocal || c2 + 1 > c->chunk_cap) return;  // use_first stays 0: warp rows
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const uint64_t *off = c->off;
    const uint32_t ch = c->large_ch;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (uint64_t base = 0; base < c2; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        unsigned long long x = 0;
        if (i < c2) {
            const uint32_t v = F.bins[2][i];
            x = (off[v + 1] - off[v] + ch - 1) / ch;
        }
        unsigned long long inc = x;  // inclusive scan within the warp
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, d);
            if ((int)lane >= d) inc += t;
        }
        if (lane == 31) s_warp[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            unsigned long long w = s_warp[lane], wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, d);
                if ((int)lane >= d) wi += t;
            }
            s_warp[lane] = wi - w;  // exclusive prefix of the warp totals
        }
        __syncthreads();
        const unsigned long long b = s_base;
        if (i < c2) c->chunk_first[i] = b + s_warp[wid] + inc - x;
        __syncthreads();
        if (threadIdx.x == 1023) s_base = b + s_warp[wid] + inc;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c->chunk_first[c2] = s_base;
        c->use_first = 1;
    }
}

const void *selector_weights(gg_graph *g);

struct GraphBfs {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    GCtl *ctl = nullptr;
    uint64_t *chunk_first = nullptr;
    uint64_t chunk_cap = 0;
    uint32_t *rest = nullptr;  // split pull: second-pass rows (n entries)
    uint64_t rest_cap = 0;
    unsigned push_grid = 0, pull_grid = 0, vgrid = 0;
    int flat = 0;  // built as one chain of kernels per step (knob graph_flat)
    int stage_kb = 0;  // pull kernels built with this much dynamic shared memory (knob pull_stage)
    int pdl = 0;       // the flat loop body's kernels joined by programmatic edges (knob graph_pdl)
    int pdl_refused = 0;  // the runtime refused programmatic edges here: built without them
    int unroll = 1;       // copies of the flat chain per loop iteration (knob graph_unroll)
    int pull_ctas = 6;    // the pull kernels' compiled residency (knob pull_ctas)
    int push_ctas = 6;    // the push kernel's (knob push_ctas)
    // page-locked host copies of the control block: the configuration sent
    // before a run, and the records a kernel writes back after it through the
    // mapping (no copy-engine transfer: a run's records do not queue behind
    // a caller's large device-to-host copy on another stream)
    GCtl *h_up = nullptr;
    GCtl *h_rec = nullptr, *d_rec = nullptr;
};

// 16-byte words: whole-line writes over the host link (byte stores would
// each be a transaction of their own)
__global__ void k_copy_words16(const uint4 *__restrict__ src, uint4 *__restrict__ dst, size_t nw) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

static gg_status add_kernel(gg_ctx *ctx, cudaGraph_t g, cudaGraphNode_t *node, const cudaGraphNode_t *deps, size_t nd,
                            const void *fn, unsigned grid, unsigned block, GCtl **arg, unsigned smem = 0) {
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.func = (void *)fn;
    kp.gridDim = dim3(grid);
    kp.blockDim = dim3(block);
    kp.sharedMemBytes = smem;
    void *args[] = {arg};
    kp.kernelParams = args;
    GG_CUDA(ctx, cudaGraphAddKernelNode(node, g, deps, nd, &kp));
    return GG_OK;
}

static gg_status add_cond(gg_ctx *ctx, cudaGraph_t g, cudaGraphNode_t *node, const cudaGraphNode_t *deps, size_t nd,
                          cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaGraph_t *body,
                          unsigned nbodies = 1) {
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = nbodies;
    GG_CUDA(ctx, cudaGraphAddNode(node, g, deps, nd, &np));
    for (unsigned i = 0; i < nbodies; ++i) body[i] = np.conditional.phGraph_out[i];
    return GG_OK;
}

void graph_bfs_free(gg_graph *g) {
    GraphBfs *gb = (GraphBfs *)g->gbfs;
    if (!gb) return;
    if (gb->exec) cudaGraphExecDestroy(gb->exec);
    if (gb->graph) cudaGraphDestroy(gb->graph);
    cudaFree(gb->ctl);
    cudaFree(gb->chunk_first);
    cudaFree(gb->rest);
    cudaFreeHost(gb->h_up);
    cudaFreeHost(gb->h_rec);
    delete gb;
    g->gbfs = nullptr;
}

static gg_status graph_bfs_build(gg_graph *g, GraphBfs *gb, int pdl) {
    gg_ctx *ctx = g->ctx;
    // (16 bytes of slack: the records' copy moves whole 16-byte words)
    GG_CUDA(ctx, cudaMalloc(&gb->ctl, sizeof(GCtl) + 16));
    GG_CUDA(ctx, cudaHostAlloc(&gb->h_up, sizeof(GCtl), cudaHostAllocDefault));
    GG_CUDA(ctx, cudaHostAlloc(&gb->h_rec, sizeof(GCtl) + 16, cudaHostAllocMapped));
    GG_CUDA(ctx, cudaHostGetDevicePointer((void **)&gb->d_rec, gb->h_rec, 0));
    gb->push_ctas = tuning().push_ctas;
    const void *fpush = gb->push_ctas == 4   ? (const void *)k_g_push<4>
                        : gb->push_ctas == 5 ? (const void *)k_g_push<5>
                        : gb->push_ctas == 7 ? (const void *)k_g_push<7>
                        : gb->push_ctas == 8 ? (const void *)k_g_push<8>
                                             : (const void *)k_g_push<6>;
    gb->push_grid = (unsigned)(ctx->sm_count * resident_ctas(fpush, kBlock));
    // pulls that stage the frontier bitmap's first words take that much
    // dynamic shared memory per CTA (fewer CTAs may then fit on an SM)
    gb->stage_kb = tuning().pull_stage;
    const unsigned stage_bytes = (unsigned)gb->stage_kb * 1024u;
    gb->pull_ctas = tuning().pull_ctas;
    const void *fpull = gb->pull_ctas == 4   ? (const void *)k_g_pull<4>
                        : gb->pull_ctas == 5 ? (const void *)k_g_pull<5>
                        : gb->pull_ctas == 7 ? (const void *)k_g_pull<7>
                        : gb->pull_ctas == 8 ? (const void *)k_g_pull<8>
                                             : (const void *)k_g_pull<6>;
    const void *fpull2 = gb->pull_ctas == 4   ? (const void *)k_g_pull2<4>
                         : gb->pull_ctas == 5 ? (const void *)k_g_pull2<5>
                         : gb->pull_ctas == 7 ? (const void *)k_g_pull2<7>
                         : gb->pull_ctas == 8 ? (const void *)k_g_pull2<8>
                                              : (const void *)k_g_pull2<6>;
    int pull_occ = 0;
    for (const void *fn : {fpull, fpull2})
        GG_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes));
    GG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pull_occ, fpull, kBlock, stage_bytes));
    gb->pull_grid = (unsigned)(ctx->sm_count * std::max(pull_occ, 1));
    gb->vgrid = (unsigned)(ctx->sm_count * 8);
    GG_CUDA(ctx, cudaGraphCreate(&gb->graph, 0));
    cudaGraph_t G = gb->graph;
    GCtl *ctl = gb->ctl;
    GCtl **arg = &gb->ctl;
    // init (+ first decision) -> WHILE { SWITCH { push: IF list {tolist} -> IF chunks {chunks} -> push,
    //                                           pull: IF bits {tobitmap} -> pull } -> next (clear + decision) }
    // The branch handles keep the value the decision set (no default
    // assignment); the loop handle starts at 1 on every launch.
    cudaGraphConditionalHandle hw, hp = 0, hq = 0, hl = 0, hb = 0, hc = 0;
    GG_CUDA(ctx, cudaGraphConditionalHandleCreate(&hw, G, 1, cudaGraphCondAssignDefault));
    cudaGraphNode_t n_init, n_while;
    GG_CHECK(add_kernel(ctx, G, &n_init, nullptr, 0, (const void *)k_g_init, gb->vgrid, 256, arg));
    cudaGraph_t body;
    GG_CHECK(add_cond(ctx, G, &n_while, &n_init, 1, hw, cudaGraphCondTypeWhile, &body));
    gb->flat = tuning().graph_flat;
    if (gb->flat) {
        // WHILE { tolist -> chunks -> push -> tobitmap -> pull -> pull2 -> next }: every
        // kernel returns at once when the step does not need it.  A conditional
        // node costs several times an idle kernel's launch inside the loop
        // (measured on B200: SWITCH about 6.7 us, IF about 2.4 us, an idle
        // kernel about 0.9 us per iteration).
        const void *chain[] = {(const void *)k_g_tolist, (const void *)k_g_chunks, fpush,
                               (const void *)k_g_tobitmap, fpull, fpull2,
                               (const void *)k_g_next};
        const unsigned grids[] = {gb->vgrid, 1, gb->push_grid, gb->vgrid, gb->pull_grid, gb->pull_grid,
                                  (unsigned)ctx->sm_count * 2};
        const unsigned blocks[] = {256, 1024, kBlock, 256, kBlock, kBlock, 256};
        const unsigned smem[] = {0, 0, 0, 0, stage_bytes, stage_bytes, 0};
        // with graph_pdl each kernel is launched while its predecessor runs
        // (programmatic edge from the predecessor's trigger port; the kernel
        // waits for the predecessor's completion in chain_enter)
        gb->pdl = pdl;
        cudaGraphEdgeData ed;
        memset(&ed, 0, sizeof(ed));
        ed.from_port = cudaGraphKernelNodePortProgrammatic;
        ed.type = cudaGraphDependencyTypeProgrammatic;
        // graph_unroll copies of the chain per loop iteration: the loop's own
        // cost is paid once per copies steps (a run that ends in an earlier
        // copy leaves the later copies' kernels with nothing to do)
        gb->unroll = tuning().graph_unroll;
        cudaGraphNode_t prev = nullptr;
        for (int i = 0; i < 7 * gb->unroll; ++i) {
            cudaGraphNode_t nd;
            GG_CHECK(add_kernel(ctx, body, &nd, (prev && !gb->pdl) ? &prev : nullptr, (prev && !gb->pdl) ? 1 : 0,
                                chain[i % 7], grids[i % 7], blocks[i % 7], arg, smem[i % 7]));
            if (prev && gb->pdl) GG_CUDA(ctx, cudaGraphAddDependencies_v2(body, &prev, &nd, &ed, 1));
            prev = nd;
        }
        GG_CUDA(ctx, cudaGraphInstantiate(&gb->exec, G, 0));
        cudaGraphConditionalHandle hs[6] = {hw, hp, hq, hl, hb, hc};
        GG_CUDA(ctx, cudaMemcpyAsync(&ctl->h_while, hs, sizeof(hs), cudaMemcpyHostToDevice, ctx->stream));
        return GG_OK;
    }
    // one SWITCH picks the step: body 0 push, body 1 pull, 2 none (h_pull
    // is the same handle)
    GG_CUDA(ctx, cudaGraphConditionalHandleCreate(&hp, body, 0, 0));
    hq = hp;
    cudaGraphNode_t n_sw, n_next;
    cudaGraph_t bsw[2];
    GG_CHECK(add_cond(ctx, body, &n_sw, nullptr, 0, hp, cudaGraphCondTypeSwitch, bsw, 2));
    cudaGraph_t bp = bsw[0], bq = bsw[1];
    GG_CUDA(ctx, cudaGraphConditionalHandleCreate(&hl, bp, 0, 0));
    GG_CUDA(ctx, cudaGraphConditionalHandleCreate(&hc, bp, 0, 0));
    GG_CUDA(ctx, cudaGraphConditionalHandleCreate(&hb, bq, 0, 0));
    cudaGraphNode_t n_ifl, n_ifb, n_list, n_push, n_bits, n_pull;
    cudaGraph_t bl, bb;
    GG_CHECK(add_cond(ctx, bp, &n_ifl, nullptr, 0, hl, cudaGraphCondTypeIf, &bl));
    GG_CHECK(add_kernel(ctx, bl, &n_list, nullptr, 0, (const void *)k_g_tolist, gb->vgrid, 256, arg));
    cudaGraphNode_t n_ifc, n_chunks;
    cudaGraph_t bc;
    GG_CHECK(add_cond(ctx, bp, &n_ifc, &n_ifl, 1, hc, cudaGraphCondTypeIf, &bc));
    GG_CHECK(add_kernel(ctx, bc, &n_chunks, nullptr, 0, (const void *)k_g_chunks, 1, 1024, arg));
    GG_CHECK(add_kernel(ctx, bp, &n_push, &n_ifc, 1, fpush, gb->push_grid, kBlock, arg));
    GG_CHECK(add_cond(ctx, bq, &n_ifb, nullptr, 0, hb, cudaGraphCondTypeIf, &bb));
    GG_CHECK(add_kernel(ctx, bb, &n_bits, nullptr, 0, (const void *)k_g_tobitmap, gb->vgrid, 256, arg));
    GG_CHECK(add_kernel(ctx, bq, &n_pull, &n_ifb, 1, fpull, gb->pull_grid, kBlock, arg, stage_bytes));
    cudaGraphNode_t n_pull2;
    GG_CHECK(add_kernel(ctx, bq, &n_pull2, &n_pull, 1, fpull2, gb->pull_grid, kBlock, arg,
                        stage_bytes));
    GG_CHECK(add_kernel(ctx, body, &n_next, &n_sw, 1, (const void *)k_g_next, (unsigned)ctx->sm_count * 2, 256, arg));
    GG_CUDA(ctx, cudaGraphInstantiate(&gb->exec, G, 0));
    // the handles live in the control block, set once
    cudaGraphConditionalHandle hs[6] = {hw, hp, hq, hl, hb, hc};
    GG_CUDA(ctx, cudaMemcpyAsync(&ctl->h_while, hs, sizeof(hs), cudaMemcpyHostToDevice, ctx->stream));
    return GG_OK;
}

// BFS levels as one graph launch (host-driven kernels, device decisions)
gg_status graph_bfs_level(gg_graph *g, uint32_t root, const gg_run_opts &opt, gg_prop *level, gg_prop *prev,
                          gg_run_stats *st, int *iters_out) {
    gg_ctx *ctx = g->ctx;
    if (!g->gbfs) {
        GraphBfs *gb = new (std::nothrow) GraphBfs;
        if (!gb) return GG_ERR_OOM;
        g->gbfs = gb;
        const int pdl = tuning().graph_flat && tuning().graph_pdl;
        gg_status s = graph_bfs_build(g, gb, pdl);
        if (s != GG_OK && pdl) {
            // programmatic edges refused (in a conditional body, say): the
            // plain chain, and no retry while the knobs stay as they are
            graph_bfs_free(g);
            cudaGetLastError();
            gb = new (std::nothrow) GraphBfs;
            if (!gb) return GG_ERR_OOM;
            g->gbfs = gb;
            s = graph_bfs_build(g, gb, 0);
            gb->pdl_refused = 1;
        }
        if (s != GG_OK) {
            graph_bfs_free(g);
            return s;
        }
    }
    GraphBfs *gb = (GraphBfs *)g->gbfs;
    if (gb->flat != tuning().graph_flat || gb->stage_kb != tuning().pull_stage ||
        (gb->flat && !gb->pdl_refused && gb->pdl != tuning().graph_pdl) ||
        (gb->flat && gb->unroll != tuning().graph_unroll) || gb->pull_ctas != tuning().pull_ctas ||
        gb->push_ctas != tuning().push_ctas) {  // built for another shape
        graph_bfs_free(g);
        return graph_bfs_level(g, root, opt, level, prev, st, iters_out);
    }
    for (auto &f : g->tmp_front)
        if (!f) GG_CHECK(gg_frontier_create(g, &f));
    for (auto *f : g->tmp_front) {
        GG_CHECK(frontier_alloc_bins(f));
        GG_CHECK(frontier_alloc_bitmap(f));
        f->host_valid = false;
        f->has_list = f->has_bitmap = f->all = false;
    }
    CandLists &cl = g->cand;
    if (!cl.list[0]) {
        for (auto &l : cl.list) GG_CUDA(ctx, cudaMalloc(&l, ((size_t)g->n + 1) * 4));
        GG_CUDA(ctx, cudaMalloc(&cl.cnt, 2 * sizeof(uint64_t)));
    }
    const Tuning &t = tuning();
    // configuration part of the control block (everything before the records)
    GCtl &h = *gb->h_up;  // the previous run's upload finished before it returned
    memset(&h, 0, offsetof(GCtl, reached_v));
    for (int i = 0; i < 2; ++i) {
        gg_frontier *f = g->tmp_front[i];
        for (int b = 0; b < NBINS; ++b) h.f[i].bins[b] = f->bins[b];
        h.f[i].bitmap = f->bitmap;
        h.f[i].cnt = (unsigned long long *)f->d_cnt;
    }
    h.level = (int32_t *)level->d;
    h.prev = (int32_t *)prev->d;
    h.root = root;
    h.n = g->n;
    h.m = g->m;
    h.max_iters = (int)std::min<uint64_t>((uint64_t)g->n + 2, (uint64_t)INT_MAX / 2);
    h.threshold = opt.threshold;
    h.threshold_k = opt.threshold_k;
    h.handoff_iter = t.graph_handoff;
    h.sel_w = nullptr;
    if (opt.threshold == GG_THRESH_LEARNED && selector_weights(g)) {
        if (g->gini < 0) {
            float gi;
            GG_CHECK(graph_gini(g, &gi));
        }
        h.sel_w = (const __nv_bfloat16 *)selector_weights(g);
        h.gini = g->gini < 0 ? 0.0f : g->gini;
        float xs[GG_SEL_FEATURES];
        selector_features(xs, 0, 0, 0, 0, (double)g->n, (double)g->m, h.gini);
        h.sel_x4 = xs[4];
        h.sel_x9 = xs[9];
    }
    h.smax = t.bin_small_max;
    h.mmax = t.bin_medium_max;
    h.large_ch = t.large_chunk;
    h.sm_count = (uint32_t)ctx->sm_count;
    h.pull_k = t.pull_k;
    h.push_k = t.push_k;
    h.off = g->off;
    h.in_off = g->in_off;
    h.word_prefix = g->heavy.pull_prefix;
    h.adj = g->adj;
    h.in_adj = g->in_adj;
    GG_CHECK(pull_records(g, t, &h.first_in, &h.first1, &h.rec_n, &h.lazy_off));
    h.fresh_ok = t.pull_fresh;
    h.stage_words = (uint32_t)gb->stage_kb * 256u;
    // the split pull's second pass starts past the record's edges: it needs
    // the first pass to have taken them from the records
    h.split = t.pull_split && (h.first_in || h.first1);
    h.flat = gb->flat;
    if (h.split && gb->rest_cap < (uint64_t)g->n) {
        cudaFree(gb->rest);
        gb->rest = nullptr;
        gb->rest_cap = 0;
        GG_CUDA(ctx, cudaMalloc(&gb->rest, ((uint64_t)g->n + 1) * 4));
        gb->rest_cap = g->n;
    }
    h.rest = gb->rest;
    h.rest_n = 0;
    h.nonisolated = g->nonisolated;
    h.nonisolated_n = (const unsigned long long *)g->nonisolated_n;
    // chunk prefix room: rows above bin_medium_max edges, at most m / (max + 1)
    const uint64_t need = g->m / ((uint64_t)t.bin_medium_max + 1) + 2;
    if (gb->chunk_cap < need) {
        cudaFree(gb->chunk_first);
        gb->chunk_first = nullptr;
        gb->chunk_cap = 0;
        GG_CUDA(ctx, cudaMalloc(&gb->chunk_first, need * 8));
        gb->chunk_cap = need;
    }
    h.chunk_first = gb->chunk_first;
    h.chunk_cap = gb->chunk_cap;
    h.cand[0] = cl.list[0];
    h.cand[1] = cl.list[1];
    h.cand_n = (unsigned long long *)cl.cnt;
    GG_CUDA(ctx, cudaMemcpyAsync(gb->ctl, &h, offsetof(GCtl, reached_v), cudaMemcpyHostToDevice, ctx->stream));
    GG_CUDA(ctx, cudaGraphLaunch(gb->exec, ctx->stream));
    // state and records back (one wait per run)
    const size_t rec0 = offsetof(GCtl, variant), rec1 = sizeof(GCtl);
    GCtl *hr = gb->h_rec;
    const size_t w0 = rec0 / 16, w1 = (rec1 + 15) / 16;  // both bases are 16-byte aligned
    k_copy_words16<<<8, 256, 0, ctx->stream>>>((const uint4 *)gb->ctl + w0, (uint4 *)gb->d_rec + w0, w1 - w0);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "graph BFS");
    if (hr->stage_timeouts)
        return set_error(ctx, GG_ERR_TIMEOUT, "graph BFS: frontier bitmap staging copy did not complete in time");
    const int T = hr->iterations;
    *iters_out = T;
    // kernels the graph ran: init, then per iteration the step kernel and
    // next, a pull's second-pass kernel (plus a list or bitmap conversion
    // where the variant changes); then the records' copy
    uint64_t npull = 0;
    for (int i = 0; i < T && i < GG_MAX_ITERS; ++i) npull += hr->variants[i] == GG_VAR_PULL_DENSE;
    // (an unrolled chain: every copy of a started loop iteration)
    const uint64_t per_loop = 7 * (uint64_t)gb->unroll;
    ctx->launches += gb->flat ? 2 + per_loop * (((uint64_t)T + gb->unroll) / gb->unroll) : 2 + 2 * (uint64_t)T + npull;
    if (hr->handed_off) {
        // the rest of the run as one device-driven launch from the current
        // frontier (a push leaves it as a list only: add its bitmap)
        const int cur = hr->cur;
        gg_frontier *f = g->tmp_front[cur];
        gg_status s = GG_OK;
        if (!hr->has_bitmap[cur]) {
            f->has_list = true;
            f->has_bitmap = f->all = f->host_valid = false;
            s = frontier_ensure_bitmap(f);
        }
        gg_emap_desc desc;
        memset(&desc, 0, sizeof(desc));
        desc.relax = GG_RELAX_MIN_PLUS1_I32;
        desc.a = level;
        desc.dst_filter = GG_FILTER_GT_CONST;
        desc.src_level_sync = 1;
        desc.record = GG_RECORD_NE_PREV;
        desc.prev = prev;
        const PersistResume rs{T, cur, hr->has_list[cur], hr->reached_v, hr->reached_e};
        int iters = 0;
        if (s == GG_OK) s = persistent_traverse(g, desc, 1, false, root, opt, st, &iters, -1, -1, nullptr, 0, &rs);
        if (s != GG_OK) return s;
        *iters_out = iters;
    } else if (st) {
        st->vertices_reached = hr->reached_v;
        st->edges_reached = hr->reached_e;
    }
    if (st) {
        for (int i = 0; i < std::min(T, GG_MAX_ITERS); ++i) {
            st->variant[i] = hr->variants[i];
            st->nactv[i] = hr->nactv[i];
            st->nacte[i] = hr->nacte[i];
            st->scanned[i] = hr->scanned[i];
            st->scanned_edges += hr->scanned[i];
            st->iter_ms[i] = i + 1 <= GG_MAX_ITERS ? (double)(hr->t_ns[i + 1] - hr->t_ns[i]) * 1e-6 : 0.0;
            st->kernel_ms[i] = hr->kt1[i] > hr->kt0[i] && hr->kt0[i] != ~0ull
                                   ? (double)(hr->kt1[i] - hr->kt0[i]) * 1e-6 : st->iter_ms[i];
        }
    }
    for (auto *f : g->tmp_front) f->host_valid = false;
    g->cand.valid = false;
    return GG_OK;
}

// Starts of the batch traversals, enqueued on the context's stream (kernel
// launches only, so a graph capture can record them).
// BFS levels from many roots: level = n+1, 0 at each root.
gg_status enqueue_bfs_start(gg_graph *g, gg_prop *level, gg_prop *prev, const uint32_t *d_roots, uint32_t k) {
    gg_ctx *ctx = g->ctx;
    int32_t inf = (int32_t)g->n + 1;
    GG_CHECK(gg_prop_fill(level, &inf));  // (prev: unused by level-synchronous steps)
    if (k) {
        k_scatter_zero_i32<<<(k + 255) / 256, 256, 0, ctx->stream>>>((int32_t *)level->d, (int32_t *)prev->d,
                                                                     d_roots, k);
        GG_LAUNCHED(ctx);
    }
    return GG_OK;
}

// CC: IDs[v] = v, prevIDs = IDs (CCv.C:246-248), PRESET_ZERO on a symmetric graph.
gg_status enqueue_cc_start(gg_graph *g, gg_prop *label, gg_prop *prev) {
    gg_ctx *ctx = g->ctx;
    if (!g->n) return GG_OK;
    k_iota_u32<<<persistent_grid(ctx, (g->n + 31) / 32), kBlock, 0, ctx->stream>>>((uint32_t *)label->d, g->n);
    GG_LAUNCHED(ctx);
    k_iota_u32<<<persistent_grid(ctx, (g->n + 31) / 32), kBlock, 0, ctx->stream>>>((uint32_t *)prev->d, g->n);
    GG_LAUNCHED(ctx);
    if (g->symmetric) {
        k_preset_zero<<<ctx->sm_count, kBlock, 0, ctx->stream>>>(g->off, g->adj, 0, (uint32_t *)label->d,
                                                                 (uint32_t *)prev->d);
        GG_LAUNCHED(ctx);
    }
    return GG_OK;
}

gg_status run_tmp_prop(gg_graph *g, int slot, gg_dtype t, gg_prop **out) { return tmp_prop(g, slot, t, out); }

}  // namespace gg

using namespace gg;

extern "C" {

gg_status gg_edgemap(gg_graph *g, const gg_emap_desc *d, gg_frontier *in, gg_frontier *out,
                     gg_emap_stats *stats) {
    if (!g || !d) return GG_ERR_ARG;
    return edgemap_impl(g, d, in, out, stats);
}

gg_status gg_bfs_level(gg_graph *g, uint32_t root, const gg_run_opts *o, gg_prop *level,
                       int32_t *host_level, gg_run_stats *st) {
    if (!g || root >= g->n) return GG_ERR_ARG;
    if (level && (level->g != g || level->t != GG_I32)) return set_error(g->ctx, GG_ERR_ARG, "level must be an I32 property of g");
    gg_run_opts opt;
    default_opts(o, &opt, GG_THRESH_DEFAULT, 0);
    if (!level) GG_CHECK(tmp_prop(g, 0, GG_I32, &level));
    gg_prop *prev;
    GG_CHECK(tmp_prop(g, 1, GG_I32, &prev));
    if (st) memset(st, 0, sizeof(*st));
    uint64_t k0 = g->ctx->launches;
    // one CUDA graph per run (device decisions) unless another driver is asked for
    // (the learned selector runs inside the graph too, choosing between its
    // push and pull; timing collection forces variants device-driven)
    const bool graph_mode = (tuning().graph & 1) && !(tuning().persistent & 1) && g->force_iter < 0 &&
                            opt.variant == GG_VAR_AUTO;
    if (graph_mode) {
        RunTimer tm(g->ctx);
        int iters = 0;
        GG_CHECK(graph_bfs_level(g, root, opt, level, prev, st, &iters));
        const double ms = tm.stop();
        if (st) {
            st->iterations = iters;
            st->total_ms = ms;
            st->kernels = g->ctx->launches - k0;
        }
        if (host_level) GG_CHECK(gg_prop_download(level, host_level));
        return gg_ctx_sync(g->ctx);
    }
    RunTimer tm(g->ctx);
    // BFSLVLv.C:117-129: level = prev = n+1, level[start] = prev[start] = 0;
    // the level-synchronous steps below never read or write prev (an
    // unvisited vertex's prev would equal its level), so only level is set
    int32_t inf = (int32_t)g->n + 1, zero = 0;
    GG_CHECK(gg_prop_fill(level, &inf));
    GG_CHECK(gg_prop_set(level, root, &zero));
    gg_frontier *F, *O;
    GG_CHECK(get_tmp_frontiers(g, &F, &O));
    GG_CHECK(gg_frontier_set_single(F, root));
    gg_emap_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.relax = GG_RELAX_MIN_PLUS1_I32;
    desc.a = level;
    desc.dst_filter = GG_FILTER_GT_CONST;  // level[d] > iter+1   (BFSLVLv.C:190-194)
    desc.src_level_sync = 1;               // frontier of iteration i holds level i
    desc.record = GG_RECORD_NE_PREV;       // level[d] != prev[d]  (BFSLVLv.C:168-172)
    desc.prev = prev;
    desc.threshold = opt.threshold;
    desc.threshold_k = opt.threshold_k;
    desc.variant = opt.variant;
    int iters = 0;
    if (use_persistent(g, opt, 1)) GG_CHECK(persistent_traverse(g, desc, 1, false, root, opt, st, &iters));
    else GG_CHECK(frontier_loop(g, desc, F, O, opt, st, true, &iters));
    double ms = tm.stop();
    if (st) {
        st->iterations = iters;
        st->total_ms = ms;
        st->kernels = g->ctx->launches - k0;
    }
    if (host_level) GG_CHECK(gg_prop_download(level, host_level));
    return gg_ctx_sync(g->ctx);
}

// BFS levels of one root into host memory, the copy overlapping the caller's
// next call: the run writes one of two level buffers in turn, its copy to
// host_level runs on the graph's copy stream, and the call returns once its
// BFS is done and the previous call's copy has landed.
gg_status gg_bfs_level_host_async(gg_graph *g, uint32_t root, const gg_run_opts *o, int32_t *host_level,
                                  gg_run_stats *st) {
    if (!g || !host_level || root >= g->n) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    if (!g->copy_stream) {
        GG_CUDA(ctx, cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            GG_CUDA(ctx, cudaEventCreateWithFlags(&g->copy_done[i], cudaEventDisableTiming));
            GG_CHECK(gg_prop_create(g, GG_I32, &g->async_level[i]));
        }
    }
    const int slot = g->async_next;
    // the buffer's last copy (two calls ago) finished before the previous call returned
    GG_CHECK(gg_bfs_level(g, root, o, g->async_level[slot], nullptr, st));
    GG_CUDA(ctx, cudaMemcpyAsync(host_level, g->async_level[slot]->d, (size_t)g->n * 4, cudaMemcpyDeviceToHost,
                                 g->copy_stream));
    GG_CUDA(ctx, cudaEventRecord(g->copy_done[slot], g->copy_stream));
    g->copy_pending[slot] = true;
    g->async_next = slot ^ 1;
    if (g->copy_pending[slot ^ 1]) {
        GG_CUDA(ctx, cudaEventSynchronize(g->copy_done[slot ^ 1]));
        g->copy_pending[slot ^ 1] = false;
    }
    return GG_OK;
}

gg_status gg_bfs_level_host_wait(gg_graph *g) {
    if (!g) return GG_ERR_ARG;
    for (int i = 0; i < 2; ++i)
        if (g->copy_pending[i]) {
            GG_CUDA(g->ctx, cudaEventSynchronize(g->copy_done[i]));
            g->copy_pending[i] = false;
        }
    return GG_OK;
}


gg_status gg_bfs_level_multi(gg_graph *g, const uint32_t *roots, uint32_t k, const gg_run_opts *o, gg_prop *level,
                             int32_t *host_level, gg_run_stats *st) {
    if (!g || (k && !roots)) return GG_ERR_ARG;
    if (level && (level->g != g || level->t != GG_I32)) return set_error(g->ctx, GG_ERR_ARG, "level must be an I32 property of g");
    gg_ctx *ctx = g->ctx;
    // distinct, in-range roots
    std::vector<uint32_t> r(roots, roots + k);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    if (!r.empty() && r.back() >= g->n) return set_error(ctx, GG_ERR_ARG, "gg_bfs_level_multi: root out of range");
    gg_run_opts opt;
    default_opts(o, &opt, GG_THRESH_DEFAULT, 0);
    if (!level) GG_CHECK(tmp_prop(g, 0, GG_I32, &level));
    gg_prop *prev;
    GG_CHECK(tmp_prop(g, 1, GG_I32, &prev));
    if (st) memset(st, 0, sizeof(*st));
    uint64_t k0 = ctx->launches;
    // roots staged in the graph scratch space past the traversal's merge
    // scratch (n + grid + 1 words, grid <= 16 CTAs per SM), so that the
    // traversal never regrows the buffer under them
    const size_t roots_at = ((size_t)g->n + (size_t)ctx->sm_count * 16 + 64) * 8;
    void *scr;
    GG_CHECK(graph_scratch(g, roots_at + r.size() * 4 + 256, &scr));
    uint32_t *d_roots = (uint32_t *)((char *)scr + roots_at);
    if (!r.empty())
        GG_CUDA(ctx, cudaMemcpyAsync(d_roots, r.data(), r.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    RunTimer tm(ctx);
    int32_t inf = (int32_t)g->n + 1;
    GG_CHECK(gg_prop_fill(level, &inf));  // (prev: unused by level-synchronous steps)
    if (!r.empty()) {
        k_scatter_zero_i32<<<((unsigned)r.size() + 255) / 256, 256, 0, ctx->stream>>>(
            (int32_t *)level->d, (int32_t *)prev->d, d_roots, (uint32_t)r.size());
        GG_LAUNCHED(ctx);
    }
    gg_emap_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.relax = GG_RELAX_MIN_PLUS1_I32;
    desc.a = level;
    desc.dst_filter = GG_FILTER_GT_CONST;
    desc.src_level_sync = 1;
    desc.record = GG_RECORD_NE_PREV;
    desc.prev = prev;
    desc.threshold = opt.threshold;
    desc.threshold_k = opt.threshold_k;
    desc.variant = opt.variant;
    // one device-driven launch for all roots
    int iters = 0;
    GG_CHECK(persistent_traverse(g, desc, 1, false, 0, opt, st, &iters, -1, -1, d_roots, (uint32_t)r.size()));
    double ms = tm.stop();
    if (st) {
        st->iterations = iters;
        st->total_ms = ms;
        st->kernels = ctx->launches - k0;
    }
    if (host_level) GG_CHECK(gg_prop_download(level, host_level));
    return gg_ctx_sync(ctx);
}

gg_status gg_bfs_parent(gg_graph *g, uint32_t root, const gg_run_opts *o, gg_prop *parent,
                        uint32_t *host_parent, gg_run_stats *st) {
    if (!g || root >= g->n) return GG_ERR_ARG;
    if (parent && (parent->g != g || parent->t != GG_U32)) return set_error(g->ctx, GG_ERR_ARG, "parent must be a U32 property of g");
    gg_run_opts opt;
    default_opts(o, &opt, GG_THRESH_DEFAULT, 0);
    if (!parent) GG_CHECK(tmp_prop(g, 2, GG_U32, &parent));
    gg_prop *prev;
    GG_CHECK(tmp_prop(g, 3, GG_U32, &prev));
    if (st) memset(st, 0, sizeof(*st));
    uint64_t k0 = g->ctx->launches;
    RunTimer tm(g->ctx);
    // BFSv.C:105-113: parent = prev = ~0, parent[start] = prev[start] = start
    uint32_t unset = 0xFFFFFFFFu;
    GG_CHECK(gg_prop_fill(parent, &unset));
    GG_CHECK(gg_prop_fill(prev, &unset));
    GG_CHECK(gg_prop_set(parent, root, &root));
    GG_CHECK(gg_prop_set(prev, root, &root));
    gg_frontier *F, *O;
    GG_CHECK(get_tmp_frontiers(g, &F, &O));
    GG_CHECK(gg_frontier_set_single(F, root));
    gg_emap_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.relax = GG_RELAX_SETIF_U32;       // parent[d].setif(s)   (BFSv.C:144-146)
    desc.a = parent;
    desc.dst_filter = GG_FILTER_MSB_SET;   // msbset(parent[d])    (BFSv.C:139-142)
    desc.src_strong = 1;
    desc.record = GG_RECORD_NE_PREV;
    desc.prev = prev;
    desc.threshold = opt.threshold;
    desc.threshold_k = opt.threshold_k;
    desc.variant = opt.variant;
    int iters = 0;
    if (use_persistent(g, opt, 2)) GG_CHECK(persistent_traverse(g, desc, 0, false, root, opt, st, &iters));
    else GG_CHECK(frontier_loop(g, desc, F, O, opt, st, false, &iters));
    double ms = tm.stop();
    if (st) {
        st->iterations = iters;
        st->total_ms = ms;
        st->kernels = g->ctx->launches - k0;
    }
    if (host_parent) GG_CHECK(gg_prop_download(parent, host_parent));
    return gg_ctx_sync(g->ctx);
}

gg_status gg_cc(gg_graph *g, const gg_run_opts *o, gg_prop *label, uint32_t *host_label,
                gg_run_stats *st) {
    if (!g) return GG_ERR_ARG;
    if (label && (label->g != g || label->t != GG_U32)) return set_error(g->ctx, GG_ERR_ARG, "label must be a U32 property of g");
    gg_run_opts opt;
    default_opts(o, &opt, GG_THRESH_FRAC, 5);  // CCv.C:309 emap_step(F, 5)
    if (!label) GG_CHECK(tmp_prop(g, 2, GG_U32, &label));
    gg_prop *prev;
    GG_CHECK(tmp_prop(g, 3, GG_U32, &prev));
    if (st) memset(st, 0, sizeof(*st));
    gg_ctx *ctx = g->ctx;
    uint64_t k0 = ctx->launches;
    RunTimer tm(ctx);
    if (g->n) {
        // IDs[v] = v (CCv.C:246-248), prevIDs = IDs
        k_iota_u32<<<persistent_grid(ctx, (g->n + 31) / 32), kBlock, 0, ctx->stream>>>((uint32_t *)label->d, g->n);
        GG_LAUNCHED(ctx);
        k_iota_u32<<<persistent_grid(ctx, (g->n + 31) / 32), kBlock, 0, ctx->stream>>>((uint32_t *)prev->d, g->n);
        GG_LAUNCHED(ctx);
        if (g->symmetric) {
            k_preset_zero<<<ctx->sm_count, kBlock, 0, ctx->stream>>>(g->off, g->adj, 0, (uint32_t *)label->d,
                                                                     (uint32_t *)prev->d);
            GG_LAUNCHED(ctx);
        }
    }
    gg_frontier *F, *O;
    GG_CHECK(get_tmp_frontiers(g, &F, &O));
    GG_CHECK(gg_frontier_set_all(F));
    gg_emap_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.relax = GG_RELAX_MIN_U32;         // IDs[d].min(IDs[s])   (CCv.C:575-581)
    desc.a = label;
    desc.dst_filter = GG_FILTER_NE_ZERO;   // IDs[d] != 0          (CCv.C:566-570)
    desc.record = GG_RECORD_NE_PREV;       // IDs[d] != prevIDs[d] (CCv.C:546-551)
    desc.prev = prev;
    desc.threshold = opt.threshold;
    desc.threshold_k = opt.threshold_k;
    desc.variant = opt.variant;
    int iters = 0;
    if (use_persistent(g, opt, 4)) GG_CHECK(persistent_traverse(g, desc, 0, true, 0, opt, st, &iters));
    else GG_CHECK(frontier_loop(g, desc, F, O, opt, st, false, &iters));
    double ms = tm.stop();
    if (st) {
        st->iterations = iters;
        st->total_ms = ms;
        st->kernels = ctx->launches - k0;
    }
    if (host_label) GG_CHECK(gg_prop_download(label, host_label));
    return gg_ctx_sync(ctx);
}

// ---------------------------------------------------------------------------
// k-core decomposition (KC_bucket, bench/KC_bucket.C:107-420)
// ---------------------------------------------------------------------------
// count[v] starts at v's degree (KC_bucket.C:125-133: coreness = degree).
// For floors L = 0, 1, 2, ... the alive list (vertices not peeled yet, all
// vertices before the first floor) is scanned once: vertices whose count is
// L form the peel frontier F (degree-binned, with its counts), vertices above
// L stay alive, and the smallest count among those is kept.  F's vertices
// have coreness L; each peel step counts their alive neighbours down towards
// L (edgemap: COUNT_DOWN with floor L, record AT_FLOOR) and the vertices that
// reach L form the next step's F, until none does (the reference's bucket for
// K and its fused re-insertions, KC_bucket.C:290-420).  A floor whose scan
// finds no vertex jumps to the smallest count left.  Where the reference
// keeps 127 buckets of vertex lists and moves vertices between them, this
// keeps one alive list that every floor compacts.
// count = degree; ngt1 counts the vertices of degree above one
__global__ void __launch_bounds__(256) k_kc_init(const uint64_t *__restrict__ off, uint32_t n,
                                                 uint32_t *__restrict__ count, unsigned long long *ngt1) {
    unsigned long long k = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t deg = off[v + 1] - off[v];
        count[v] = deg > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)deg;
        k += deg > 1;
    }
    k = dev::block_sum<unsigned long long, 256>(k);
    if (threadIdx.x == 0 && k) atomicAdd(ngt1, k);
}

// The reference's degree-one preprocessing (KC_bucket.C:131-160), taken
// when fewer than n/2 vertices have a degree above one, raises every count
// to at least 1 and leaves isolated vertices (in no bucket) at that 1: its
// output reports coreness 1 for them then, as this does.
__global__ void __launch_bounds__(256) k_kc_isolated(const uint64_t *__restrict__ off, uint32_t n,
                                                     uint32_t *__restrict__ count) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        if (off[v + 1] == off[v]) count[v] = 1u;
}

// alive == nullptr: every vertex (the first floor)
__global__ void __launch_bounds__(256) k_kc_scan(const uint32_t *__restrict__ alive, uint64_t nall,
                                                 const unsigned long long *__restrict__ alive_n,
                                                 const uint32_t *__restrict__ count, uint32_t L,
                                                 const uint64_t *__restrict__ off, uint32_t smax, uint32_t mmax,
                                                 uint32_t *b0, uint32_t *b1, uint32_t *b2,
                                                 unsigned long long *fcnt, uint32_t *alive_out,
                                                 unsigned long long *alive_out_n, unsigned long long *min_left) {
    __shared__ uint32_t sb[4][8][256];
    const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    dev::WarpAppender<256> ap0{sb[0][wib], 0, b0, fcnt + FC_BIN0};
    dev::WarpAppender<256> ap1{sb[1][wib], 0, b1, fcnt + FC_BIN1};
    dev::WarpAppender<256> ap2{sb[2][wib], 0, b2, fcnt + FC_BIN2};
    dev::WarpAppender<256> keep{sb[3][wib], 0, alive_out, alive_out_n};
    const uint64_t na = alive ? (uint64_t)*alive_n : nall;
    unsigned long long nv = 0, ne = 0;
    uint32_t mn = 0xFFFFFFFFu;
    const uint64_t step = (uint64_t)gridDim.x * 256;
    for (uint64_t base = ((uint64_t)blockIdx.x * 8 + wib) * 32; base < na; base += step) {
        const uint64_t i = base + lane;
        uint32_t v = 0;
        bool at = false, above = false;
        uint64_t deg = 0;
        if (i < na) {
            v = alive ? alive[i] : (uint32_t)i;
            const uint32_t c = count[v];
            at = c == L;
            above = c > L;
            if (at) deg = off[v + 1] - off[v];
            if (above) mn = min(mn, c);
        }
        ap0.push(at && deg <= smax, v);
        ap1.push(at && deg > smax && deg <= mmax, v);
        ap2.push(at && deg > mmax, v);
        keep.push(above, v);
        if (at) {
            nv++;
            ne += deg;
        }
    }
    ap0.flush();
    ap1.flush();
    ap2.flush();
    keep.flush();
    mn = __reduce_min_sync(FULL, mn);
    if (lane == 0 && mn != 0xFFFFFFFFu) atomicMin(min_left, (unsigned long long)mn);
    nv = dev::block_sum<unsigned long long, 256>(nv);
    ne = dev::block_sum<unsigned long long, 256>(ne);
    if (threadIdx.x == 0) {
        if (nv) atomicAdd(fcnt + FC_NACTV, nv);
        if (ne) atomicAdd(fcnt + FC_NACTE, ne);
    }
}

gg_status gg_kcore(gg_graph *g, const gg_run_opts *o, gg_prop *coreness, uint32_t *host_coreness,
                   uint32_t *largest_core, gg_run_stats *st) {
    if (!g) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    if (!g->symmetric) return set_error(ctx, GG_ERR_UNSUPPORTED, "gg_kcore: symmetric graphs only");
    if (coreness && (coreness->g != g || coreness->t != GG_U32))
        return set_error(ctx, GG_ERR_ARG, "coreness must be a U32 property of g");
    // Sparse push by default: a count-down pull has no early exit, so one warp
    // walks each high-degree row whole (measured at R-MAT 22: 34.5 ms with
    // every step a push against 218 ms with the m/20 threshold, whose few
    // pulls took most of it)
    gg_run_opts opt;
    default_opts(o, &opt, GG_THRESH_ALWAYS_SPARSE, 0);
    if (opt.threshold == GG_THRESH_LEARNED) opt.threshold = GG_THRESH_ALWAYS_SPARSE;  // no network for this relax
    if (!coreness) GG_CHECK(tmp_prop(g, 2, GG_U32, &coreness));
    if (st) memset(st, 0, sizeof(*st));
    if (!g->kc_cnt) {
        for (auto &a : g->kc_alive) GG_CUDA(ctx, cudaMalloc(&a, ((size_t)g->n + 1) * 4));
        GG_CUDA(ctx, cudaMalloc(&g->kc_cnt, 4 * sizeof(unsigned long long)));
    }
    const Tuning &t = tuning();
    cudaStream_t sm = ctx->stream;
    uint64_t k0 = ctx->launches;
    RunTimer tm(ctx);
    uint32_t *count = (uint32_t *)coreness->d;
    GG_CUDA(ctx, cudaMemsetAsync(g->kc_cnt + 3, 0, 8, sm));
    if (g->n) {
        k_kc_init<<<persistent_grid(ctx, ((uint64_t)g->n + 31) / 32), 256, 0, sm>>>(g->off, g->n, count,
                                                                                    g->kc_cnt + 3);
        GG_LAUNCHED(ctx);
    }
    gg_frontier *F, *O;
    GG_CHECK(get_tmp_frontiers(g, &F, &O));
    gg_emap_desc desc;
    memset(&desc, 0, sizeof(desc));
    desc.relax = GG_RELAX_COUNT_DOWN_U32;  // coreness[d].count_down_value(cK)  (KC_bucket.C:371-380)
    desc.a = coreness;
    desc.dst_filter = GG_FILTER_GT_CONST;  // only counts above the floor move
    desc.record = GG_RECORD_AT_FLOOR;      // old == cK + 1: d reached the floor  (KC_bucket.C:353-369)
    desc.threshold = opt.threshold;
    desc.threshold_k = opt.threshold_k;
    desc.variant = opt.variant;
    const unsigned sgrid = (unsigned)(ctx->sm_count * resident_ctas((const void *)k_kc_scan, 256));
    // {alive A, alive B, min left, vertices of degree above one}, in a part of the pinned staging buffer
    // that the frontier count reads (its first FC_WORDS words) leave alone
    unsigned long long *hc = (unsigned long long *)ctx->h_pinned + 48;
    uint64_t L = 0;
    int cur = 0, steps = 0, floors = 0;
    bool first = true;
    uint32_t largest = 0;
    while (g->n) {
        // the scan at floor L: peel frontier F, the next alive list, the smallest count left
        GG_CHECK(frontier_alloc_bins(F));
        GG_CHECK(frontier_reset_counts(F));
        GG_CUDA(ctx, cudaMemsetAsync(g->kc_cnt + (cur ^ 1), 0, 8, sm));
        GG_CUDA(ctx, cudaMemsetAsync(g->kc_cnt + 2, 0xFF, 8, sm));
        k_kc_scan<<<sgrid, 256, 0, sm>>>(first ? nullptr : g->kc_alive[cur], g->n, g->kc_cnt + cur, count,
                                         (uint32_t)L, g->off, t.bin_small_max, t.bin_medium_max, F->bins[0],
                                         F->bins[1], F->bins[2], (unsigned long long *)F->d_cnt,
                                         g->kc_alive[cur ^ 1], g->kc_cnt + (cur ^ 1), g->kc_cnt + 2);
        GG_LAUNCHED(ctx);
        F->all = false;
        F->has_list = true;
        F->has_bitmap = false;
        F->host_valid = false;
        GG_CUDA(ctx, cudaMemcpyAsync(hc, g->kc_cnt, 4 * 8, cudaMemcpyDeviceToHost, sm));
        GG_CHECK(frontier_fetch_counts(F));  // (synchronises: hc is current too)
        cur ^= 1;
        first = false;
        ++floors;
        const uint64_t left = hc[cur], min_left = hc[2];
        if (F->h_cnt[FC_NACTV] == 0) {
            if (left == 0) break;
            L = min_left;  // no vertex at this floor: the next count that exists
            continue;
        }
        largest = (uint32_t)L;
        // peel steps at floor L: F's vertices have coreness L
        desc.dst_filter_k = (int64_t)L;
        while (F->h_cnt[FC_NACTV] != 0 && F->h_cnt[FC_NACTE] != 0) {
            gg_emap_stats es;
            GG_CHECK(edgemap_impl(g, &desc, F, O, opt.collect_stats ? &es : nullptr));
            if (opt.collect_stats) record_iter(st, steps, es);
            ++steps;
            std::swap(F, O);
            GG_CHECK(frontier_fetch_counts(F));
        }
        if (left == 0) break;
        L = L + 1;
    }
    if (g->n && hc[3] < (unsigned long long)(g->n / 2)) {  // (hc[3]: vertices of degree above one)
        k_kc_isolated<<<persistent_grid(ctx, ((uint64_t)g->n + 31) / 32), 256, 0, sm>>>(g->off, g->n, count);
        GG_LAUNCHED(ctx);
        largest = std::max(largest, 1u);
    }
    double ms = tm.stop();
    if (st) {
        st->iterations = steps;
        st->total_ms = ms;
        st->kernels = ctx->launches - k0;
        st->vertices_reached = (uint64_t)floors;  // floors scanned
    }
    if (largest_core) *largest_core = largest;
    if (host_coreness) GG_CHECK(gg_prop_download(coreness, host_coreness));
    return gg_ctx_sync(ctx);
}

}  // extern "C"
