// gg_tune.cu -- the autotuner: coordinate descent over the tuning knobs,
// timing the analytics on the graph they will run on.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gg_internal.cuh"

namespace gg {

namespace {

struct Knob {
    const char *name;
    std::vector<int64_t> values;
    bool rebuild;  // changes the graph's heavy-row tables
};

std::vector<Knob> knob_space(int analytics) {
    std::vector<Knob> k = {
        {"bin_small_max", {8, 16, 32, 64, 128}, false},
        {"bin_medium_max", {512, 1024, 2048, 4096, 8192}, false},
        {"pull_k", {2, 4, 8, 16}, false},
        {"push_k", {4, 8, 16}, false},
        {"large_chunk", {256, 512, 1024, 2048}, false},
        {"blocks_per_sm", {2, 4, 8, 16}, false},
        {"heavy_deg", {128, 256, 512, 1024}, true},
        {"heavy_chunk", {512, 1024, 2048, 4096}, true},
    };
    if (analytics & (GG_TUNE_BFS | GG_TUNE_CC)) k.push_back({"persistent", {0, 1, 4, 5}, false});
    if (analytics & GG_TUNE_BFS) k.push_back({"pull_split", {0, 1}, false});
    if (analytics & GG_TUNE_PR) {
        k.push_back({"pr_stream", {0, 1}, false});
        k.push_back({"pr_blocks_per_sm", {4, 8, 16, 32}, false});
    }
    return k;
}

struct Objective {
    gg_graph *g;
    int analytics;
    std::vector<uint32_t> roots;
    int reps;
    std::vector<int32_t> lv0, lv;
    std::vector<uint32_t> cc0, cc;
    bool have_ref = false;
    int evals = 0;

    // sum over analytics of the fastest of `reps` runs; false on a result mismatch
    gg_status eval(double *ms_out) {
        ++evals;
        double total = 0;
        gg_run_stats st;
        if (analytics & GG_TUNE_BFS) {
            for (size_t i = 0; i < roots.size(); ++i) {
                double best = 1e30;
                for (int r = 0; r < reps; ++r) {
                    const bool check = r == 0 && i == 0;
                    GG_CHECK(gg_bfs_level(g, roots[i], nullptr, nullptr, check ? lv.data() : nullptr, &st));
                    best = std::min(best, st.total_ms);
                }
                total += best;
            }
        }
        if (analytics & GG_TUNE_CC) {
            double best = 1e30;
            for (int r = 0; r < reps; ++r) {
                GG_CHECK(gg_cc(g, nullptr, nullptr, r == 0 ? cc.data() : nullptr, &st));
                best = std::min(best, st.total_ms);
            }
            total += best;
        }
        if (analytics & GG_TUNE_PR) {
            gg_pr_params p;
            std::memset(&p, 0, sizeof(p));
            p.maxiter = 5;
            p.tol = 0;
            p.damping = 0.85f;
            p.contrib_dtype = GG_F32;
            p.accum_f64 = 0;
            double best = 1e30;
            for (int r = 0; r < reps; ++r) {
                GG_CHECK(gg_pagerank(g, &p, nullptr, nullptr, &st));
                best = std::min(best, st.total_ms);
            }
            total += best;
        }
        if (!have_ref) {
            lv0 = lv;
            cc0 = cc;
            have_ref = true;
        } else if (lv != lv0 || cc != cc0) {
            return set_error(g->ctx, GG_ERR_STATE, "autotune: results changed with the tuning knobs");
        }
        *ms_out = total;
        return GG_OK;
    }
};

gg_status set_knob(gg_graph *g, const Knob &k, int64_t v) {
    GG_CHECK(gg_tuning_set(k.name, v));
    if (k.rebuild) GG_CHECK(gg_graph_retune(g));
    return GG_OK;
}

}  // namespace
}  // namespace gg

using namespace gg;

extern "C" {

gg_status gg_graph_retune(gg_graph *g) {
    if (!g) return GG_ERR_ARG;
    GG_CUDA(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    HeavyRows &H = g->heavy;
    cudaFree(H.v);
    cudaFree(H.first);
    cudaFree(H.crow);
    cudaFree(H.light_prefix);
    cudaFree(H.pull_prefix);
    H = HeavyRows();
    cudaFree(g->nonisolated);
    cudaFree(g->nonisolated_n);
    g->nonisolated = nullptr;
    g->nonisolated_n = nullptr;
    return build_heavy_rows(g);
}

gg_status gg_autotune(gg_graph *g, int analytics, const uint32_t *roots, int nroots, int passes, int reps,
                      gg_tune_result *out) {
    if (!g || !out || passes < 1 || reps < 1 || !(analytics & 7)) return GG_ERR_ARG;
    if ((analytics & GG_TUNE_BFS) && (nroots < 1 || !roots)) return GG_ERR_ARG;
    for (int i = 0; i < nroots; ++i)
        if (roots[i] >= g->n) return set_error(g->ctx, GG_ERR_ARG, "gg_autotune: root out of range");
    std::memset(out, 0, sizeof(*out));
    Objective obj;
    obj.g = g;
    obj.analytics = analytics;
    if (analytics & GG_TUNE_BFS) obj.roots.assign(roots, roots + nroots);
    obj.reps = reps;
    obj.lv.assign((analytics & GG_TUNE_BFS) ? g->n : 0, 0);
    obj.cc.assign((analytics & GG_TUNE_CC) ? g->n : 0, 0);
    std::vector<Knob> space = knob_space(analytics);
    std::vector<int64_t> cur(space.size());
    for (size_t i = 0; i < space.size(); ++i) GG_CHECK(gg_tuning_get(space[i].name, &cur[i]));
    // a warm-up evaluation (first-use allocations), then the reference one
    double best;
    GG_CHECK(obj.eval(&best));
    GG_CHECK(obj.eval(&best));
    out->initial_ms = best;
    for (int pass = 0; pass < passes; ++pass) {
        bool changed = false;
        for (size_t i = 0; i < space.size(); ++i) {
            const Knob &k = space[i];
            int64_t keep = cur[i];
            for (int64_t v : k.values) {
                if (v == cur[i]) continue;
                // bin_small_max <= bin_medium_max must hold
                int64_t lo = 0, hi = 0;
                gg_tuning_get("bin_small_max", &lo);
                gg_tuning_get("bin_medium_max", &hi);
                if ((!std::strcmp(k.name, "bin_small_max") && v > hi) ||
                    (!std::strcmp(k.name, "bin_medium_max") && v < lo))
                    continue;
                GG_CHECK(set_knob(g, k, v));
                double ms;
                gg_status s = obj.eval(&ms);
                if (s != GG_OK) {
                    set_knob(g, k, keep);
                    return s;
                }
                if (ms < best * 0.99) {
                    best = ms;
                    keep = v;
                    changed = true;
                }
            }
            GG_CHECK(set_knob(g, k, keep));
            cur[i] = keep;
        }
        if (!changed) break;
    }
    out->best_ms = best;
    out->evaluations = obj.evals;
    std::string s;
    for (size_t i = 0; i < space.size(); ++i) {
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%s%s=%lld", i ? "," : "", space[i].name, (long long)cur[i]);
        s += buf;
    }
    std::snprintf(out->best, sizeof(out->best), "%s", s.c_str());
    return GG_OK;
}

}  // extern "C"
