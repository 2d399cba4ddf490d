// graptor/graptor.h for sources written against Graptor: maps the include
// onto the B200 library's operator surface (graptor_b200/api.h) and adds the
// host-side pieces the analytics and the reference's own bench/driver.C use:
// the host CSR file reader (GraphCSx), the graph layout names the driver's
// createGraph() helpers construct, the PBBS-style timing macros, the option
// parser, and the host utilities of the validation code (map_vertexL,
// vertexFilter with a C++ functor, sequence::pack, ...).
//
// Put include/graptor_b200/compat first on the include path; the analytics'
// own sources (bench/BFSLVLv.C, BFSv.C, CCv.C, PRv.C, PR_vary.C) then compile
// unchanged, with their driver, and run their edgemap / vertexmap steps on
// the GPU.  Every layout name (GRAPHTYPE) builds the same device CSR/CSC.
#ifndef GRAPTOR_B200_COMPAT_GRAPTOR_H
#define GRAPTOR_B200_COMPAT_GRAPTOR_H

#include <algorithm>
#include <cassert>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#include "graptor_b200/api.h"

// Command-line options with Graptor's accessors (legacy/parseCommandLine.h):
// getOption(flag) = flag present, getOptionValue(flag) = next argument,
// getOptionLongValue(flag, default), getArgument(i) = i-th argument from the end.
struct commandLine {
    int argc;
    char **argv;
    std::string usage;
    commandLine(int c, char **v, std::string u = "") : argc(c), argv(v), usage(std::move(u)) {}
    int find(const std::string &flag) const {
        for (int i = 1; i < argc; ++i)
            if (flag == argv[i]) return i;
        return -1;
    }
    bool getOption(const std::string &flag) const { return find(flag) >= 0; }
    // a flag with no value that ends the line still counts as given ("-s <file>"
    // is read as -s followed by a value, which is how the reference treats it)
    char *getOptionValue(const std::string &flag) const {
        int i = find(flag);
        return (i >= 0 && i + 1 < argc) ? argv[i + 1] : nullptr;
    }
    std::string getOptionValue(const std::string &flag, const std::string &dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::string(v) : dflt;
    }
    long getOptionLongValue(const std::string &flag, long dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::atol(v) : dflt;
    }
    double getOptionDoubleValue(const std::string &flag, double dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::atof(v) : dflt;
    }
    char *getArgument(int i) const { return argv[argc - 1 - i]; }
};

// Wall-clock interval timer with Graptor's interface (timer.h): start(),
// next() = seconds since the previous start/next, total().
class timer {
public:
    timer() { start(); }
    void start() { last_ = now(); }
    double next() {
        double t = now(), d = t - last_;
        last_ = t;
        total_ += d;
        return d;
    }
    double stop() { next(); return total_; }
    double total() const { return total_; }

private:
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
    double last_ = 0, total_ = 0;
};

namespace graptor_b200 {
// The driver's round timer (legacy/gettime.h startTime/nextTime/reportAvg):
// nextTime waits for the device work of the round before it reads the clock
// and prints "<name> : <seconds>".
struct round_timer {
    timer t;
    double sum = 0;
    void start() {
        if (ctx_slot()) check(gg_ctx_sync(ctx_slot()), "gg_ctx_sync");
        t.start();
    }
    void report(const char *name) {
        if (ctx_slot()) check(gg_ctx_sync(ctx_slot()), "gg_ctx_sync");
        double d = t.next();
        sum += d;
        std::cout << name << " : " << std::setprecision(6) << d << std::endl;
    }
    void avg(long rounds) {
        std::cout << "Average time : " << std::setprecision(6) << (rounds ? sum / rounds : 0.0) << std::endl;
    }
};
inline round_timer &the_round_timer() {
    static round_timer r;
    return r;
}
}  // namespace graptor_b200

#define startTime() graptor_b200::the_round_timer().start()
#define nextTime(_name) graptor_b200::the_round_timer().report(_name)
#define reportAvg(_rounds) graptor_b200::the_round_timer().avg(_rounds)

inline unsigned ilog2(uint64_t x) { return x ? 63u - (unsigned)__builtin_clzll(x) : 0u; }

// Host CSR read from a Graptor version-2/3 binary file
// (GraphCSx::readFromBinaryFile, graph/GraphCSx.h:2137-2262): header of 8
// words {version, _, n, m, sizeof(VID), sizeof(EID), ...}, n offsets, (v3:
// the n+1-th offset), m edge targets.  Weighted graphs are not on the path.
class GraphCSx {
public:
    GraphCSx(const char *file, int /*allocation*/, bool symmetric, const char *weights = nullptr)
        : sym_(symmetric) {
        if (weights) throw graptor_b200::error(GG_ERR_UNSUPPORTED, "edge weights are not on the edgemap path");
        FILE *f = std::fopen(file, "rb");
        if (!f) throw graptor_b200::error(GG_ERR_IO, std::string("cannot open ") + file);
        uint64_t h[8];
        bool ok = std::fread(h, sizeof h, 1, f) == 1 && (h[0] == 2 || h[0] == 3) && h[4] == 4 && h[5] == 8 &&
                  h[2] < 0xFFFFFFFFull;
        if (ok) {
            n_ = (VID)h[2];
            m_ = h[3];
            off_.resize((size_t)n_ + 1);
            adj_.resize(m_ ? m_ : 1);
            ok = n_ == 0 || std::fread(off_.data(), 8, n_, f) == n_;
            if (ok && h[0] == 3) {
                uint64_t last = 0;
                ok = std::fread(&last, 8, 1, f) == 1 && last == m_;
            }
            ok = ok && (m_ == 0 || std::fread(adj_.data(), 4, m_, f) == m_);
            off_[n_] = m_;
        }
        std::fclose(f);
        if (!ok) throw graptor_b200::error(GG_ERR_IO, std::string("not a Graptor v2/v3 graph file: ") + file);
    }
    VID numVertices() const { return n_; }
    EID numEdges() const { return m_; }
    const EID *getIndex() const { return off_.data(); }
    const VID *getEdges() const { return adj_.data(); }
    VID getDegree(VID v) const { return (VID)(off_[v + 1] - off_[v]); }
    bool isSymmetric() const { return sym_; }
    void del() {
        std::vector<EID>().swap(off_);
        std::vector<VID>().swap(adj_);
    }

private:
    VID n_ = 0;
    EID m_ = 0;
    bool sym_ = false;
    std::vector<EID> off_;
    std::vector<VID> adj_;
};

// The graph layouts bench/driver.C names (its createGraph() helpers).  They
// are the reference's CPU layouts (VEBO, SlimSell, Graptor SIMD slabs, ...);
// on the GPU every one of them is the device CSR/CSC of GraphGPU.
#define GG_COMPAT_LAYOUT(Name)                                                   \
    struct Name : GraphGPU {                                                     \
        Name(const GraphCSx &G, int npart = 0, int a = 0, int b = 0, int c = 0)  \
            : GraphGPU(G, npart) { (void)a; (void)b; (void)c; }                  \
        Name(const GraphCSx &G, int npart, bool balance) : GraphGPU(G, npart) {  \
            (void)balance;                                                       \
        }                                                                        \
    };
GG_COMPAT_LAYOUT(GraphGGVEBO)
GG_COMPAT_LAYOUT(GraphGG)
GG_COMPAT_LAYOUT(GraphVEBOSlimSell)
GG_COMPAT_LAYOUT(GraphSlimSell)
GG_COMPAT_LAYOUT(GraphVEBOPartCSR)
GG_COMPAT_LAYOUT(GraphVEBOPartCCSR)
GG_COMPAT_LAYOUT(GraphCSR)
#undef GG_COMPAT_LAYOUT

using graptor_mode_t = unsigned;
// (cached, push, single-vector) flags of the Graptor layouts
#define GRAPTOR_MODE_MACRO(c, p, s) ((graptor_mode_t)(((c) << 2) | ((p) << 1) | (s)))
#ifndef GRAPTOR_MODE
#define GRAPTOR_MODE GRAPTOR_MODE_MACRO(1, 0, 1)
#endif
template <graptor_mode_t Mode> struct GraphVEBOGraptor : GraphGPU {
    GraphVEBOGraptor(const GraphCSx &G, int npart = 0, int a = 0, int b = 0, int c = 0) : GraphGPU(G, npart) {
        (void)a; (void)b; (void)c;
    }
};

// Host loops over the vertices (map_vertexL, legacy/parallel loops); the
// functors are host code, as in the reference, and run on the host's threads
// where the program is built with OpenMP (the reference runs them in
// parallel too).
template <typename Fn> void map_vertexL(const partitioner &part, Fn fn) {
    graptor_b200::host_sync();
    const int64_t n = part.get_num_vertices();
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; ++v) fn((VID)v);
}
// map_vertex_serialL: the same loop, in vertex order (the reference runs it
// serially for repeatable random draws, FMv.C:291-298)
template <typename Fn> void map_vertex_serialL(const partitioner &part, Fn fn) {
    graptor_b200::host_sync();
    for (VID v = 0, n = part.get_num_vertices(); v < n; ++v) fn(v);
}
// map_partitionL(part, fn(k)): fn per partition (one partition on the device)
template <typename Fn> void map_partitionL(const partitioner &part, Fn fn) {
    graptor_b200::host_sync();
    const int p = part.get_num_partitions();
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < p; ++k) fn((unsigned)k);
}
// vertexMap(part, F, functor): a host functor over the vertices of F
// (legacy vertexMap with a C++ functor, APRv.C:500)
template <typename F> void vertexMap(const partitioner &part, const frontier &Fr, F fn) {
    graptor_b200::host_sync();
    if (Fr.all()) {
        const int64_t n = part.get_num_vertices();
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < n; ++v) fn((VID)v);
    } else {
        const VID *l = Fr.getSparse();
        const int64_t k = Fr.nActiveVertices();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < k; ++i) fn(l[i]);
    }
}
template <typename I, typename Fn> void parallel_loop(I lo, I hi, Fn fn) {
    graptor_b200::host_sync();
#pragma omp parallel for schedule(static)
    for (int64_t i = (int64_t)lo; i < (int64_t)hi; ++i) fn((I)i);
}

// vertexFilter(GA, V, functor) (dsl/vmap_utils.h:62-72): the vertices of V
// for which a C++ functor holds.  The functor is host code (it reads host
// arrays), so it runs on the host over the managed arrays; the edgemap
// analytics' expression filters (lazy_executor::vertex_filter) run on the GPU.
template <typename GraphType, typename F> frontier vertexFilter(const GraphType &GA, frontier V, F filter) {
    graptor_b200::host_sync();
    const VID n = GA.numVertices();
    std::vector<VID> keep;
    if (V.all()) {
        for (VID v = 0; v < n; ++v)
            if (filter(v)) keep.push_back(v);
    } else {
        const VID *l = V.getSparse();
        for (VID i = 0, k = V.nActiveVertices(); i < k; ++i)
            if (filter(l[i])) keep.push_back(l[i]);
        std::sort(keep.begin(), keep.end());
    }
    return frontier::sparse(n, (VID)keep.size(), keep.data());
}

// gtraits<G>::createValidFrontier<W>(G) (graph/gtraits.h): every vertex of the
// file; the device layout has no padding vertices.
template <typename GraphType> struct gtraits {
    template <unsigned short W> static frontier createValidFrontier(const GraphType &G) {
        return frontier::all_true(G.numVertices(), G.numEdges());
    }
};

// sequence::pack (legacy/sequence.h): the indices in [s, e) whose flag is set.
template <typename T> struct _seq {
    T *A = nullptr;
    long n = 0;
    _seq() = default;
    _seq(T *a, long k) : A(a), n(k) {}
};
template <typename T> struct identityF {
    T operator()(T i) const { return i; }
};
namespace sequence {
template <typename T, typename Flag, typename F>
_seq<T> pack(T *out, const Flag *flags, T s, T e, F f) {
    graptor_b200::host_sync();
    long k = 0;
    for (T i = s; i < e; ++i) k += flags[i] != 0;
    T *a = out ? out : new T[k ? k : 1];
    long j = 0;
    for (T i = s; i < e; ++i)
        if (flags[i] != 0) a[j++] = f(i);
    return _seq<T>(a, k);
}
}  // namespace sequence

#endif
