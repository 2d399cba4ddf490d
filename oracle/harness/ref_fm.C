// ref_fm.C -- TEST HARNESS around the reference's own FMv analytic.
//
// Compiled (by oracle/Makefile) together with the UNMODIFIED reference source
// bench/FMv.C, which includes bench/driver.C unconditionally: the driver's
// main() is renamed while it is included and never called.  It
// exists because FMv prints only the effective diameter: the harness builds
// the same GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)> layout the reference
// driver builds (bench/driver.C:70-75, 110-116), runs FMv::run() once with
// -itimes, and reports
//   * "n <file n> padded <layout n> iters <k> deffG <x> time_s <run() seconds>";
//   * "nactv <|F| of iteration 0> <|F| of iteration 1> ..." (FMv.C:416-425);
//   * <prefix>.mask: the final bit mask per vertex, in ORIGINAL order (uint32);
//   * <prefix>.remap: the layout id of each original vertex (uint32): FMv
//     draws its initial masks in layout order (FMv.C:291-298), so vertex v
//     starts with draw number remap[v].
// Usage: ref_fm <graph.bin> <out_prefix>
#include "graptor/graptor.h"
#include "graptor/api.h"
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#define private public  // expose the analytic's result arrays to the harness
#define main ref_fm_driver_main_unused
#include "FMv.C"
#undef main
#undef private

using HarnessGraph = GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)>;

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s graph.bin out_prefix\n", argv[0]);
        return 2;
    }
    const std::string out = argv[2];
    GraphCSx G(argv[1], -1, true, nullptr);
    const VID n = G.numVertices();
    HarnessGraph PG(G, 256, MAX_VL / 2, MAX_VL, 4);
    G.del();
    char a0[] = "ref_fm", a1[] = "-itimes";
    char *cargv[] = {a0, a1, nullptr};
    commandLine P(2, cargv, "");
    FMv<HarnessGraph> problem(PG, P);
    auto t0 = std::chrono::steady_clock::now();
    problem.run();
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("n %u padded %u iters %d deffG %.9g time_s %.6f\n", (unsigned)n, (unsigned)PG.numVertices(),
                problem.iter, (double)problem.deffG, sec);
    std::printf("nactv");
    for (int i = 0; i < problem.iter; ++i) std::printf(" %llu", (unsigned long long)problem.info_buf[i].nactv);
    std::printf("\n");
    std::vector<uint32_t> mask(n), remap(n);
    for (VID v = 0; v < n; ++v) {
        remap[v] = (uint32_t)PG.remapID(v);
        mask[v] = (uint32_t)problem.new_mask[remap[v]];
    }
    FILE *f = std::fopen((out + ".mask").c_str(), "wb");
    if (!f || std::fwrite(mask.data(), 4, n, f) != n) return 3;
    std::fclose(f);
    f = std::fopen((out + ".remap").c_str(), "wb");
    if (!f || std::fwrite(remap.data(), 4, n, f) != n) return 3;
    std::fclose(f);
    PG.del();
    return 0;
}
