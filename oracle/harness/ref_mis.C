// ref_mis.C -- TEST HARNESS around the reference's own MISv analytic.
//
// Compiled (by oracle/Makefile) together with the UNMODIFIED reference source
// bench/MISv.C (VARIANT 13, its default: 2-bit states) with NOBENCH defined,
// so its driver.C main() is left out.  MISv prints only a validation summary;
// the harness builds the GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)> layout
// the reference driver builds (bench/driver.C:70-75, 110-116), runs
// MISv::run() and validate(), and writes the final state of every vertex
// (0 undecided, 1 conditionally in, 2 out, 3 in; MISv.C:118-123) in ORIGINAL
// vertex order as uint8 to <out>, and the layout id of every vertex (MISv's
// priorities are layout ids: s < d, MISv.C:240-243) as uint32 to <out>.remap.
// Prints "n <n> padded <n'> iters <k> in <c> time_s <run() seconds>".
// Usage: ref_mis <graph.bin> <out>
#include "graptor/graptor.h"
#include "graptor/api.h"
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#define NOBENCH 1
#define private public  // expose the analytic's state array to the harness
#include "MISv.C"
#undef private

using HarnessGraph = GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)>;

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s graph.bin out\n", argv[0]);
        return 2;
    }
    GraphCSx G(argv[1], -1, true, nullptr);
    const VID n = G.numVertices();
    HarnessGraph PG(G, 256, MAX_VL / 2, MAX_VL, 4);
    G.del();
    char a0[] = "ref_mis";
    char *cargv[] = {a0, nullptr};
    commandLine P(1, cargv, "");
    MISv<HarnessGraph> problem(PG, P);
    auto t0 = std::chrono::steady_clock::now();
    problem.run();
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    MISv<HarnessGraph>::stat st;
    problem.validate(st, false);
    std::vector<uint8_t> state(n);
    std::vector<uint32_t> remap(n);
    VID in = 0;
    for (VID v = 0; v < n; ++v) {
        remap[v] = (uint32_t)PG.remapID(v);
        state[v] = (uint8_t)Enc::get(problem.m_flags, remap[v]);
        in += state[v] == 3;
    }
    std::printf("n %u padded %u iters %d in %u time_s %.6f\n", (unsigned)n, (unsigned)PG.numVertices(), problem.iter,
                (unsigned)in, sec);
    FILE *f = std::fopen(argv[2], "wb");
    if (!f || std::fwrite(state.data(), 1, n, f) != n) return 3;
    std::fclose(f);
    f = std::fopen((std::string(argv[2]) + ".remap").c_str(), "wb");
    if (!f || std::fwrite(remap.data(), 4, n, f) != n) return 3;
    std::fclose(f);
    PG.del();
    return 0;
}
