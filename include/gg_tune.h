/*
 * gg_tune.h -- tuning knobs of libgg.so (degree-bin thresholds, chunk sizes,
 * per-lane scan depths, grid sizes, kernel variants) and the autotuner that
 * picks them.  Values are process-wide.
 *
 * No reference counterpart: Graptor fixes its equivalents at compile time
 * (EMAP_BLOCK_SIZE, include/graptor/dsl/edgemap.h:29-31; the edge-chunk
 * granularity of dsl/emap/edgechunk.h:315-440; MAX_VL).
 *
 * Names: bin_small_max, bin_medium_max (sparse-push degree bins),
 * pull_k, push_k (edges a lane scans alone before its warp helps),
 * heavy_deg, heavy_chunk (CSC rows chunked for gathers; apply to graphs
 * created afterwards or after gg_graph_retune), large_chunk (push: edges
 * per chunk of a hub row), blocks_per_sm (CTAs per SM of the grid-stride
 * kernels), pr_stream (1: warp-streamed segmented PageRank gather, 0:
 * per-row), pr_blocks_per_sm (the PageRank kernels' grid cap, 16), persistent (bit mask: 1 BFS levels, 2 BFS parents, 4 CC run as
 * one device-driven cooperative launch; otherwise one launch per iteration
 * from the host), graph (1, the default: BFS levels run as one CUDA graph
 * whose conditional nodes take each step's push/pull decision on the
 * device; 0: one host round trip per iteration), graph_handoff (32, the
 * default: a graph-driven BFS still running after that many iterations
 * continues as one device-driven cooperative launch from its current
 * frontier; 0: never), handoff_ctas (CTAs of that launch, 148 by default,
 * 0 = all that fit), small_frontier (1, the default: from level
 * graph_handoff on (32 when that knob is 0), a device-driven BFS whose
 * listed frontier is at most 8192 vertices and 65536 edges runs its levels
 * in one cluster of 8 CTAs with the frontier in shared memory until the
 * frontier outgrows a CTA's 4096-entry queue or 262144 edges; 0: never),
 * cc_hook (1: a
 * device-driven CC run of a symmetric graph
 * that passes CCv's road-network test after its first step finishes by
 * min-id hooking; 0: label propagation throughout), fusion (4: the sparse
 * push steps of a device-driven CC run fused, as CCv with api::fusion: a
 * lowered label is propagated at once through a device work queue; 0, the
 * default: level by level), fusion_queue (entries of
 * that queue, 0 = 2n + 65536; entries beyond it spill into the next
 * frontier), barrier_timeout_ns (how long a CTA of a persistent run waits
 * at a grid barrier, or a warp on the work queue without progress, before
 * it reports GG_ERR_TIMEOUT).
 */
#ifndef GG_TUNE_H
#define GG_TUNE_H
#include "gg.h"
#ifdef __cplusplus
extern "C" {
#endif
GG_API gg_status gg_tuning_set(const char *name, int64_t value);
GG_API gg_status gg_tuning_get(const char *name, int64_t *value);

/* Rebuild the graph's tuning-dependent tables (chunked heavy rows, per-word
 * cost prefixes) with the current heavy_deg / heavy_chunk. */
GG_API gg_status gg_graph_retune(gg_graph *g);

/* Autotuner.  Coordinate descent over the knobs above on graph g: each knob
 * in turn takes each of its candidate values while the others stay at their
 * best so far; a candidate is kept when the objective (the sum of the
 * analytics' device times, each the minimum of `reps` runs) drops by more
 * than 1%.  `passes` sweeps over all knobs.  Every candidate's BFS levels
 * and CC labels are compared with the first run's and must be identical
 * (GG_ERR_STATE otherwise).  On return the best values are set. */
enum { GG_TUNE_BFS = 1, GG_TUNE_CC = 2, GG_TUNE_PR = 4 };
typedef struct gg_tune_result {
    double initial_ms;   /* objective with the values on entry */
    double best_ms;      /* objective with the chosen values */
    int evaluations;     /* objective evaluations */
    char best[512];      /* "name=value,..." of every knob tuned */
} gg_tune_result;
GG_API gg_status gg_autotune(gg_graph *g, int analytics, const uint32_t *roots, int nroots, int passes, int reps,
                             gg_tune_result *out);
#ifdef __cplusplus
}
#endif
#endif
