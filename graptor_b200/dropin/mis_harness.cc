// Drives the reference's MISv analytic (bench/MISv.C, VARIANT 13), compiled
// unchanged against this library's Graptor-compatible headers with NOBENCH
// defined, on the GPU; runs it, its own validate(), and writes the final
// state of every vertex (0 undecided, 1 conditionally in, 2 out, 3 in) as
// uint8 to <out>, which MISv itself does not print.
//
// Usage: mis graph.bin out
//   prints "n <n> iters <k> in <c> time_s <t>".
#include "graptor/graptor.h"
#include "graptor/api.h"

#include <cstdio>

#define NOBENCH 1
#define private public  // the harness reads the analytic's state array
#include "MISv.C"
#undef private

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s graph.bin out\n", argv[0]);
        return 2;
    }
    try {
        GraphGPU GA = GraphGPU::read_bin(argv[1], true);
        const VID n = GA.numVertices();
        char a0[] = "mis";
        char *cargv[] = {a0, nullptr};
        commandLine P(1, cargv);
        {
            MISv<GraphGPU> problem(GA, P);
            timer tm;
            problem.run();
            const double t = tm.next();
            MISv<GraphGPU>::stat st;
            problem.validate(st, false);
            std::vector<uint8_t> state(n);
            VID in = 0;
            for (VID v = 0; v < n; ++v) {
                state[v] = (uint8_t)Enc::get(problem.m_flags, v);
                in += state[v] == 3;
            }
            std::printf("n %u iters %d in %u time_s %.6f\n", (unsigned)n, problem.iter, (unsigned)in, t);
            FILE *f = std::fopen(argv[2], "wb");
            if (!f || std::fwrite(state.data(), 1, n, f) != n) return 3;
            std::fclose(f);
        }
        GA.del();
    } catch (const graptor_b200::error &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
