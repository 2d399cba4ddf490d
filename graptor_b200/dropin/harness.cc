// Drives an analytic class written against Graptor's operator surface and
// compiled unchanged against this library (graptor/graptor.h from
// include/graptor_b200/compat).  Built by graptor_b200/dropin/Makefile from
// the analytic's own source file with NOBENCH defined, so its driver main()
// is left out and this one is used.
//
// Usage: <prog> graph.bin out_prefix|- root...
//   loads the Graptor .bin graph onto the GPU, runs the analytic from each
//   root and writes the per-vertex result (int32 per vertex) to
//   out_prefix.<root>.i32; prints "root <r> time_s <t>".
#include "graptor/graptor.h"
#include "graptor/api.h"

#include <cstdio>

#define NOBENCH 1
#define private public  // the harness reads the analytic's result arrays
#ifdef DROPIN_BFSV
#include "BFSv.C"
#else
#include "BFSLVLv.C"
#endif
#undef private

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s graph.bin out_prefix|- root...\n", argv[0]);
        return 2;
    }
    try {
        GraphGPU GA = GraphGPU::read_bin(argv[1], true);
        const std::string out = argv[2];
        const VID n = GA.numVertices();
        for (int a = 3; a < argc; ++a) {
            char arg0[] = "dropin", arg1[] = "-start";
            char *cargv[] = {arg0, arg1, argv[a], nullptr};
            commandLine P(3, cargv);
#ifdef DROPIN_BFSV
            BFSv<GraphGPU> problem(GA, P);
#else
            BFSLVLv<GraphGPU> problem(GA, P);
#endif
            timer tm;
            problem.run();
            double t = tm.next();
            std::printf("root %s time_s %.6f\n", argv[a], t);
            if (out != "-") {
                std::vector<int32_t> dump(n);
                for (VID v = 0; v < n; ++v) {
#ifdef DROPIN_BFSV
                    dump[v] = (int32_t)problem.parent[v];
#else
                    dump[v] = (int32_t)problem.a_level[v];
#endif
                }
                std::string path = out + "." + argv[a] + ".i32";
                FILE *f = std::fopen(path.c_str(), "wb");
                if (!f || std::fwrite(dump.data(), 4, n, f) != n) return 3;
                std::fclose(f);
            }
        }
        GA.del();
    } catch (const graptor_b200::error &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
