// ref_bfs.C -- TEST/BASELINE HARNESS around the reference's own BFS analytics.
//
// Compiled (by oracle/Makefile) together with the UNMODIFIED reference
// sources bench/BFSLVLv.C or bench/BFSv.C (selected by -DREF_BFSV) with
// NOBENCH defined, so the reference's driver.C main() is left out and this
// file drives the analytic instead.  It exists because the reference's
// BFS programs print no per-vertex output (only validate() summaries):
//   * loads a Graptor v2 .bin graph once and builds the same
//     GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)> (PullDataParCached)
//     layout the reference driver builds (bench/driver.C:70-75, 110-116);
//   * runs BFS from each requested root, timing only run() exactly like the
//     driver's startTime()/nextTime("Running") bracket (driver.C:245-255);
//   * optionally dumps per-vertex levels (or parents) in ORIGINAL vertex
//     order to a binary file (int32 per vertex).
// VEBO pads every partition to a multiple of the vector length
// (graph/VEBOReorder.h:700-712), so the reordered graph can hold more vertices
// than the file; BFSLVLv's "unreached" level is then (padded n)+1.  The dump
// covers the file's vertices only and writes unreached levels as n+1 of the
// file's n; the padded count is printed so callers can reject padded graphs
// where a comparison depends on it.
//
// With out_prefix "+" nothing is written; each root's line instead ends
// with two 64-bit checksums of the per-vertex result, sum over v of
// (uint32)value[v] * w_k(v) modulo 2^64 with w_k(v) = splitmix64 finaliser of
// (v + k * 0x9E3779B97F4A7C15), k = 1, 2, so that a caller can compare the
// result of a large graph without reading it.
//
// Usage: ref_bfs <graph.bin> <out_prefix|-|+> <root> [root ...]
//   prints one line per root:  "root <r> time_s <t> reached <k> [check <h1> <h2>]"
#include "graptor/graptor.h"
#include "graptor/api.h"
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#define NOBENCH 1
#define private public   // expose the analytic's result arrays to the harness
#ifdef REF_BFSV
#include "BFSv.C"
#else
#include "BFSLVLv.C"
#endif
#undef private

using HarnessGraph = GraphVEBOGraptor<GRAPTOR_MODE_MACRO(1,0,1)>;

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s graph.bin out_prefix|- root...\n", argv[0]);
        return 2;
    }
    const std::string file = argv[1];
    const std::string out = argv[2];
    GraphCSx G(file, -1, true, nullptr);
    const VID n = G.numVertices();
    const int npart = 256;
    HarnessGraph PG(G, npart, MAX_VL / 2, MAX_VL, 4);
    G.del();
    const VID npad = PG.numVertices();
    std::printf("n %u padded %u\n", (unsigned)n, (unsigned)npad);
    for (int a = 3; a < argc; ++a) {
        std::string root = argv[a];
        char arg0[] = "ref_bfs", arg1[] = "-start";
        std::vector<char> rbuf(root.begin(), root.end());
        rbuf.push_back('\0');
        char *cargv[] = {arg0, arg1, rbuf.data(), nullptr};
        commandLine P(3, cargv, "");
#ifdef REF_BFSV
        BFSv<HarnessGraph> problem(PG, P);
#else
        BFSLVLv<HarnessGraph> problem(PG, P);
#endif
        auto t0 = std::chrono::steady_clock::now();
        problem.run();
        auto t1 = std::chrono::steady_clock::now();
        double sec = std::chrono::duration<double>(t1 - t0).count();
        VID reached = 0;
        const bool check = out == "+";
        uint64_t h1 = 0, h2 = 0;
        std::vector<int32_t> dump(out == "-" || check ? 0 : n);
        for (VID v = 0; v < n; ++v) {
            VID rv = PG.remapID(v);
#ifdef REF_BFSV
            VID p = problem.parent[rv];
            int32_t val = (~p == 0) ? -1 : (int32_t)PG.originalID(p);
            reached += (~p != 0);
#else
            int32_t val = (int32_t)problem.a_level[rv];
            if (val < 0 || (VID)val > npad) val = (int32_t)(n + 1);  // unreached
            reached += ((VID)val <= n);
#endif
            if (!dump.empty()) dump[v] = val;
            if (check) {
                h1 += (uint64_t)(uint32_t)val * mix64((uint64_t)v + 0x9E3779B97F4A7C15ull);
                h2 += (uint64_t)(uint32_t)val * mix64((uint64_t)v + 2 * 0x9E3779B97F4A7C15ull);
            }
        }
        if (check)
            std::printf("root %s time_s %.9f reached %u check %016llx %016llx\n", root.c_str(), sec,
                        (unsigned)reached, (unsigned long long)h1, (unsigned long long)h2);
        else
            std::printf("root %s time_s %.9f reached %u\n", root.c_str(), sec, (unsigned)reached);
        std::fflush(stdout);
        if (!dump.empty()) {
            std::string path = out + "." + root + ".i32";
            FILE *f = std::fopen(path.c_str(), "wb");
            if (!f || std::fwrite(dump.data(), 4, n, f) != n) return 3;
            std::fclose(f);
        }
    }
    PG.del();
    return 0;
}
