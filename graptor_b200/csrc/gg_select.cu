// gg_select.cu -- traversal-variant selection for the LEARNED threshold.
//
// Until a trained network is loaded, the selector is the reference's default
// density threshold (include/graptor/api.h:151-157: sparse iff
// nactv + nacte <= m/20).
#include "gg_internal.cuh"

namespace gg {

int learned_select(gg_graph *g, uint64_t nactv, uint64_t nacte, int iter, bool can_early_exit) {
    (void)iter;
    (void)can_early_exit;
    return (nactv + nacte) <= (g->m / 20) ? GG_VAR_PUSH_SPARSE : GG_VAR_PULL_DENSE;
}

}  // namespace gg
