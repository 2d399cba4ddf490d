/*
 * gg_select.h -- the learned traversal-variant selector of libgg.so.
 *
 * Graptor picks sparse push or dense pull per edgemap call by a fixed
 * density threshold (include/graptor/api.h:130-222; CCv.C:309,408 vary its
 * fraction).  The selector replaces that rule by a small network that, at
 * every iteration of a device-driven traversal, predicts the time of each
 * traversal variant from frontier statistics already on the device and runs
 * the fastest; the threshold stays the fallback (no selector attached, or
 * GG_THRESH_DEFAULT/FRAC), and its choice stands unless the network
 * predicts the other variant at least 13% faster.  Every variant computes
 * the same result, so the choice changes time only.
 *
 * Network: 10 -> 32 -> 32 -> 4, ReLU, output = predicted log2 of the
 * variant's iteration time in microseconds (push_sparse, push_merge,
 * pull_dense, push_dense).  Inference uses bfloat16 weights with float32
 * accumulation; training keeps float32 master weights (Adam, full batch).
 * Parameters are packed as W1[32][10], b1[32], W2[32][32], b2[32],
 * W3[4][32], b3[4] (GG_SEL_NPARAMS floats).
 *
 * Features of an iteration (all computed on the device):
 *   0 log2(1+|F|)/32          1 log2(1+sum outdeg F)/40   2 log2(1+unreached)/32
 *   3 log2(1+min(iter,255))/8 4 log2(1+m/n)/8             5 degree Gini of the graph
 *   6 |F|/n                   7 outdeg(F)/m               8 min((|F|+outdeg F)/m, 4)
 *   9 log2(n)/32
 * (the iteration enters by its logarithm: a linear count let the network
 * fit bumps between the sampled iterations of long runs)
 */
#ifndef GG_SELECT_H
#define GG_SELECT_H
#include "gg.h"
#ifdef __cplusplus
extern "C" {
#endif

#define GG_SEL_FEATURES 10
#define GG_SEL_VARIANTS 4
#define GG_SEL_NPARAMS (32 * 10 + 32 + 32 * 32 + 32 + 4 * 32 + 4)

typedef struct gg_selector gg_selector;

GG_API gg_status gg_selector_create(gg_ctx *ctx, gg_selector **out);
GG_API gg_status gg_selector_destroy(gg_selector *s);
GG_API gg_status gg_selector_set_params(gg_selector *s, const float *params, int nparams);
GG_API gg_status gg_selector_get_params(gg_selector *s, float *params, int nparams);
/* Inference (bfloat16 weights): out[n][4] = predicted log2 us, X host [n][10]. */
GG_API gg_status gg_selector_forward(gg_selector *s, const float *X, int n, float *out);
/* Masked MSE loss and its gradient w.r.t. the float32 parameters (host arrays). */
GG_API gg_status gg_selector_loss_grad(gg_selector *s, const float *X, const float *Y, const float *M,
                                       int n, float *loss, float *grad);
/* Full-batch Adam training on the GPU for `epochs` steps; final loss out. */
GG_API gg_status gg_selector_train(gg_selector *s, const float *X, const float *Y, const float *M, int n,
                                   int epochs, float lr, float *final_loss);

/* Timing collection.  Runs the analytic (0 = BFS levels from root, 1 = CC)
 * device-driven, once per (sampled iteration, variant), every iteration
 * using the threshold's choice except the sampled one, and records per
 * sampled iteration its features X[k][10] and, per variant, the log2 us of
 * the sampled iteration (BFS: every variant leaves the same next frontier)
 * or of the rest of the run from that iteration on (CC: a fused push step
 * finishes the run) in Y[k][4] (NaN where the forced run ended before that
 * iteration, which CC's racing push steps can cause).  Any iteration of the
 * run can be sampled.  At most `max_samples` iterations are sampled,
 * alternately spread evenly and geometrically over the run (duplicates
 * dropped); *nrec receives the record count (<= cap). */
GG_API gg_status gg_selector_collect(gg_graph *g, int analytic, uint32_t root, int max_samples,
                                     float *X, float *Y, int cap, int *nrec);

/* Attach a selector to a graph (NULL detaches): runs with GG_THRESH_LEARNED
 * consult its network.  The graph keeps its own copy of the weights as they
 * are at this call, so the selector may be retrained or destroyed afterwards
 * (attach again to use retrained weights). */
GG_API gg_status gg_graph_set_selector(gg_graph *g, gg_selector *s);

#ifdef __cplusplus
}
#endif
#endif
