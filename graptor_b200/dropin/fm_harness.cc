// Drives the reference's FMv analytic (bench/FMv.C), compiled unchanged
// against this library's Graptor-compatible headers, on the GPU and reports
// what FMv computes but does not print: the final bit mask of every vertex.
// FMv.C includes its driver unconditionally; the driver's main() is renamed
// while it is included and never called.
//
// Usage: fm graph.bin out_prefix
//   prints "n <n> padded <n> iters <k> deffG <x>" and "nactv <|F| per
//   iteration>", writes out_prefix.mask (uint32 per vertex).
#include "graptor/graptor.h"
#include "graptor/api.h"

#include <cstdio>

#define private public  // the harness reads the analytic's result arrays
#define main fmv_driver_main_unused
#include "FMv.C"
#undef main
#undef private

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s graph.bin out_prefix\n", argv[0]);
        return 2;
    }
    try {
        GraphGPU GA = GraphGPU::read_bin(argv[1], true);
        const std::string out = argv[2];
        const VID n = GA.numVertices();
        char a0[] = "fm", a1[] = "-itimes";
        char *cargv[] = {a0, a1, nullptr};
        commandLine P(2, cargv);
        {
            FMv<GraphGPU> problem(GA, P);
            timer tm;
            problem.run();
            const double t = tm.next();
            std::printf("n %u padded %u iters %d deffG %.9g time_s %.6f\n", (unsigned)n, (unsigned)n, problem.iter,
                        (double)problem.deffG, t);
            std::printf("nactv");
            for (int i = 0; i < problem.iter; ++i)
                std::printf(" %llu", (unsigned long long)problem.info_buf[i].nactv);
            std::printf("\n");
            std::vector<uint32_t> mask(n);
            for (VID v = 0; v < n; ++v) mask[v] = problem.new_mask[v];
            FILE *f = std::fopen((out + ".mask").c_str(), "wb");
            if (!f || std::fwrite(mask.data(), 4, n, f) != n) return 3;
            std::fclose(f);
        }
        GA.del();
    } catch (const graptor_b200::error &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
