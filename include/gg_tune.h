/*
 * gg_tune.h -- tuning knobs of libgg.so (degree-bin thresholds, chunk sizes,
 * per-lane scan depths, kernel variants).  Set by the project's autotuner
 * (graptor_b200/autotune.py) or by hand; values are process-wide.
 *
 * No reference counterpart: Graptor fixes its equivalents at compile time
 * (EMAP_BLOCK_SIZE, include/graptor/dsl/edgemap.h:29-31; the edge-chunk
 * granularity of dsl/emap/edgechunk.h:315-440; MAX_VL).
 *
 * Names: bin_small_max, bin_medium_max (sparse-push degree bins),
 * pull_k, push_k (edges a lane scans alone before its warp helps),
 * heavy_deg, heavy_chunk (CSC rows chunked for gathers; applies to graphs
 * created afterwards), large_chunk (push: edges per chunk of a hub row),
 * pr_stream (1: warp-streamed segmented PageRank gather, 0: per-row),
 * persistent (bit mask: 1 BFS levels, 2 BFS parents, 4 CC run as one
 * device-driven cooperative launch; otherwise one launch per iteration from
 * the host), barrier_timeout_ns
 * (how long a CTA of a persistent run waits at a grid barrier before it
 * reports GG_ERR_TIMEOUT).
 */
#ifndef GG_TUNE_H
#define GG_TUNE_H
#include "gg.h"
#ifdef __cplusplus
extern "C" {
#endif
GG_API gg_status gg_tuning_set(const char *name, int64_t value);
GG_API gg_status gg_tuning_get(const char *name, int64_t *value);
#ifdef __cplusplus
}
#endif
#endif
