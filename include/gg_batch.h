/*
 * gg_batch.h -- batched traversals of libgg.so.
 *
 * Graptor runs one analytic instance per invocation (bench/BFSLVLv.C runs
 * its roots one after another, bench/PRv.C has no seed vector).  None of
 * these entry points replaces a reference interface; they batch the same
 * relax rules over many instances so that one launch serves them all:
 *
 *  - gg_msbfs: BFS levels from up to 64 roots at once.  Each vertex holds a
 *    64-bit word per state (frontier, next, visited), bit i for root i; an
 *    iteration pushes or pulls whole words, so one edge visit serves every
 *    root.  Levels equal gg_bfs_level's for each root (BFSLVLv.C:165-216
 *    semantics: level[root] = 0, unreached = n+1).  One cooperative launch.
 *  - gg_ppr: personalized PageRank for up to 128 seeds,
 *        x_s = alpha * e_s + (1 - alpha) * A^T D^-1 x_s,
 *    D = out-degree (vertices without out-edges pass nothing on), x_s(0) =
 *    e_s, `iters` iterations.  Ranks and contributions are stored in
 *    bfloat16 (a 256-byte row of 128 seeds per vertex), sums in float32.
 *    The iteration loop is captured once into a CUDA graph.
 *  - gg_graph_union + gg_bfs_level_multi + gg_cc: many independent graphs
 *    are laid side by side as one graph (part i's vertex v becomes
 *    vertex_base[i] + v); BFS from one root per part is a multi-root BFS on
 *    the union (one device-driven launch), CC of every part is CC of the
 *    union (label - vertex_base[i] = part-local label).
 */
#ifndef GG_BATCH_H
#define GG_BATCH_H
#include "gg.h"
#ifdef __cplusplus
extern "C" {
#endif

#define GG_MSBFS_MAX_ROOTS 64
#define GG_PPR_MAX_SEEDS 128

/* Multi-source BFS levels.  host_levels (may be NULL): [n][k] int32,
 * host_levels[v*k + i] = level of v from roots[i].  Roots may repeat.
 * stats: iterations, total_ms, edges_reached (sum over roots of the
 * out-degrees of reached vertices, the GTEPS numerator), variant[] /
 * iter_ms[] per iteration (GG_VAR_PUSH_DENSE or GG_VAR_PULL_DENSE). */
GG_API gg_status gg_msbfs(gg_graph *g, const uint32_t *roots, int k, int32_t *host_levels, gg_run_stats *stats);

/* Personalized PageRank.  host_x (may be NULL): [n][k] float32, the
 * bfloat16-stored ranks widened.  stats: total_ms, iterations. */
GG_API gg_status gg_ppr(gg_graph *g, const uint32_t *seeds, int k, float alpha, int iters, float *host_x,
                        gg_run_stats *stats);

/* Disjoint union of k graphs of the same context into a new graph.
 * vertex_base (may be NULL) receives k+1 entries: the first union vertex of
 * each part and the total.  Symmetric iff every part is. */
GG_API gg_status gg_graph_union(gg_ctx *ctx, gg_graph *const *parts, int k, gg_graph **out, uint32_t *vertex_base);

/* BFS levels from several roots at once (all at level 0), run as one
 * device-driven launch.  Duplicate roots are ignored. */
GG_API gg_status gg_bfs_level_multi(gg_graph *g, const uint32_t *roots, uint32_t k, const gg_run_opts *o,
                                    gg_prop *level, int32_t *host_level, gg_run_stats *st);

/* BFS levels from several roots and CC labels of one graph -- a disjoint
 * union of many small graphs (gg_graph_union), each part's BFS from its own
 * root and its components -- submitted as ONE CUDA graph launch (the BFS
 * start, the device-driven multi-root BFS, the CC start and the
 * device-driven CC; the host waits once).  The reference runs BFSLVLv.C and
 * CCv.C once per graph (bench/BFSLVLv.C:110-254, bench/CCv.C:221-471); this
 * batch has no counterpart there.  level (I32) / label (U32) may be NULL
 * (library temporaries).  bfs_stats / cc_stats receive each run's records
 * and the batch's device time in total_ms; *graph_launches is 1 when the
 * work went out as one graph launch (0 if the runtime refused the capture
 * and the launches went out one by one) and *kernel_launches the kernels
 * the batch holds.  Duplicate roots are ignored. */
GG_API gg_status gg_batch_bfs_cc(gg_graph *g, const uint32_t *roots, uint32_t k, gg_prop *level, gg_prop *label,
                                 int32_t *host_level, uint32_t *host_label, gg_run_stats *bfs_stats,
                                 gg_run_stats *cc_stats, int *graph_launches, uint64_t *kernel_launches);

#ifdef __cplusplus
}
#endif
#endif
