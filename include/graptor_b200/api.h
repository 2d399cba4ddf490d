// graptor_b200/api.h -- Graptor's edgemap/vertexmap operator surface over the
// B200 library (libgg.so, C ABI in gg.h).  Header-only C++17.
//
// The reference's analytics are written against include/graptor/api.h:
//   api::edgemap(GA, api::record(...), api::filter(...), api::relax(λ))  (api.h:2143-2415)
//   make_lazy_executor(part).vertex_map(λ).vertex_scan(λ).materialize() (dsl/vertexmap.h:2120-2446)
//   api::vertexprop<T,VID,AID,Enc>                                      (api/vertexprop.h:30-140)
//   frontier::create / all_true / del / nActiveVertices / ...            (frontier/frontier.h:58-716)
// and the lambdas return expression trees built from expr::_c, _0, _1, cast,
// iif, min, setif, ... (dsl/ast).  As in the reference the lambdas run once,
// on placeholder arguments, to build the tree; here the tree is a run-time
// object that is lowered to a gg_emap_desc (the enumerated relax/filter/record
// kinds of the hot path) or compiled to a gg_vmap_desc stack program.  A tree
// outside the lowering table throws graptor_b200::error(GG_ERR_UNSUPPORTED)
// naming the expression.
#ifndef GRAPTOR_B200_API_H
#define GRAPTOR_B200_API_H

#include <cmath>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "gg.h"

using VID = uint32_t;
using EID = uint64_t;

namespace graptor_b200 {

struct error : std::runtime_error {
    gg_status status;
    error(gg_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline gg_ctx *&ctx_slot() {
    static gg_ctx *c = nullptr;
    return c;
}

// Process-wide context on device GG_DEVICE (default 0), created on first use.
inline gg_ctx *context() {
    gg_ctx *&c = ctx_slot();
    if (!c) {
        const char *dv = std::getenv("GG_DEVICE");
        gg_status s = gg_ctx_create(dv ? std::atoi(dv) : 0, &c);
        if (s != GG_OK) throw error(s, std::string("gg_ctx_create: ") + gg_status_string(s));
    }
    return c;
}

inline void check(gg_status s, const char *what) {
    if (s != GG_OK) {
        std::string m = std::string(what) + ": " + gg_status_string(s) + ": " + gg_last_error(ctx_slot());
        throw error(s, m);
    }
}

// Device writes bump this epoch; host mirrors of properties refresh on change.
// (Atomic: the analytics' host loops run on several threads.)
inline std::atomic<uint64_t> &device_epoch() {
    static std::atomic<uint64_t> e{1};
    return e;
}
inline std::mutex &host_mutex() {
    static std::mutex m;
    return m;
}
// an atomic that copies by value (members of copyable host-side handles)
template <typename T> struct catomic {
    std::atomic<T> v;
    catomic(T x = T()) : v(x) {}
    catomic(const catomic &o) : v(o.v.load()) {}
    catomic &operator=(const catomic &o) {
        v.store(o.v.load());
        return *this;
    }
    T load() const { return v.load(); }
    void store(T x) { v.store(x); }
};

template <typename T> struct dtype_of;
template <> struct dtype_of<int32_t> { static constexpr gg_dtype value = GG_I32; };
template <> struct dtype_of<uint32_t> { static constexpr gg_dtype value = GG_U32; };
template <> struct dtype_of<uint8_t> { static constexpr gg_dtype value = GG_U8; };
template <> struct dtype_of<float> { static constexpr gg_dtype value = GG_F32; };
template <> struct dtype_of<double> { static constexpr gg_dtype value = GG_F64; };

// Registry of device arrays by device address, so that expr::array_ro(ptr)
// (PRv.C:125-150) can find the property behind a raw pointer.
inline std::map<const void *, gg_prop *> &registry() {
    static std::map<const void *, gg_prop *> r;
    return r;
}

// Host code reads and writes managed arrays (mmap_ptr) in place; before it
// does, the device work queued since the last wait must have finished.
inline std::atomic<uint64_t> &synced_epoch() {
    static std::atomic<uint64_t> e{0};
    return e;
}
inline void host_sync() {
    const uint64_t d = device_epoch().load();
    if (synced_epoch().load() != d && ctx_slot()) {
        check(gg_ctx_sync(ctx_slot()), "gg_ctx_sync");
        synced_epoch().store(d);
    }
}

// Where a managed array's pages are (mmap_ptr).  Host code that reaches
// for an array the device holds first brings it over in one prefetch;
// arrays the host has reached for since the last device step go back to
// the device in one prefetch before the next step.  Page by page, either
// side would fault them over (or read them across the host link).
struct managed_state {
    gg_prop *p = nullptr;
    std::atomic<bool> on_device{false};
    std::atomic<bool> touched{false};
};
inline std::set<managed_state *> &host_touched() {
    static std::set<managed_state *> s;
    return s;
}
inline void host_access(managed_state *st) {
    std::lock_guard<std::mutex> lock(host_mutex());
    host_sync();
    if (st->on_device) {
        check(gg_prop_prefetch(st->p, 0), "gg_prop_prefetch");
        check(gg_ctx_sync(ctx_slot()), "gg_ctx_sync");
        st->on_device = false;
    }
    if (!st->touched) {
        st->touched = true;
        host_touched().insert(st);
    }
}
inline void before_device() {
    auto &t = host_touched();
    for (managed_state *st : t) {
        check(gg_prop_prefetch(st->p, 1), "gg_prop_prefetch");
        st->on_device = true;
        st->touched = false;
    }
    t.clear();
}

// Dense frontier arrays (frontier::dense) released by one iteration are kept
// for the next one's (an allocation and a free, which waits for the device,
// per iteration otherwise); a graph's are freed with the graph.
inline std::map<std::pair<gg_graph *, int>, std::vector<gg_prop *>> &dense_pool() {
    static std::map<std::pair<gg_graph *, int>, std::vector<gg_prop *>> p;
    return p;
}
inline void dense_pool_release(gg_graph *g) {
    auto &pool = dense_pool();
    for (auto it = pool.begin(); it != pool.end();) {
        if (it->first.first == g) {
            for (gg_prop *q : it->second) gg_prop_destroy(q);
            it = pool.erase(it);
        } else {
            ++it;
        }
    }
}

// The graph that frontiers made from host vertex lists (frontier::sparse)
// belong to: the last graph built, as the analytics use one graph at a time.
inline gg_graph *&default_graph() {
    static gg_graph *g = nullptr;
    return g;
}

}  // namespace graptor_b200

// ---------------------------------------------------------------------------
// Graph and partitioner
// ---------------------------------------------------------------------------
class GraphGPU;

class partitioner {
public:
    partitioner() = default;
    // np: host-side partitions of the vertex range (the driver's -c); the
    // device does not partition
    partitioner(gg_graph *g, VID n, int np = 1) : g_(g), n_(n), np_(np > 0 ? np : 1) {}
    VID get_num_vertices() const { return n_; }
    VID get_num_elements() const { return n_ * scale_; }
    int get_num_partitions() const { return np_; }
    // scale(k): the partitioning of k consecutive elements per vertex
    // (graph/partitioning.h); arrays allocated from it hold n*k elements
    partitioner scale(VID k) const {
        partitioner p(*this);
        p.scale_ *= k;
        return p;
    }
    VID get_scale() const { return scale_; }
    // the vertex range of partition k: [start_of(k), end_of(k))
    VID start_of(int k) const { return k <= 0 ? 0 : (k >= np_ ? n_ : (VID)((uint64_t)k * n_ / np_)); }
    VID end_of(int k) const { return start_of(k + 1); }
    gg_graph *graph() const { return g_; }

private:
    gg_graph *g_ = nullptr;
    VID n_ = 0;
    int np_ = 1;
    VID scale_ = 1;
};

// Host view of the CSR (GraphCSx accessors the analytics call through
// GA.getCSR(), graph/GraphCSx.h:293-420): index and edges in host memory,
// the degree array in managed memory registered as a vertex property, so
// that it serves both host reads and expr::array_ro(getDegree()) operands
// (PRv.C:46,150; the reference's expr::aid_graph_degree).
class GraphCSxView {
public:
    VID numVertices() const { return n_; }
    EID numEdges() const { return m_; }
    const EID *getIndex() const { return off_.data(); }
    const VID *getEdges() const { return adj_.data(); }
    const VID *getDegree() const { graptor_b200::host_sync(); return deg_; }
    VID getDegree(VID v) const { graptor_b200::host_sync(); return deg_[v]; }
    VID getNeighbor(VID v, VID i) const { return adj_[off_[v] + i]; }
    bool isSymmetric() const { return sym_; }

private:
    friend class GraphGPU;
    VID n_ = 0;
    EID m_ = 0;
    bool sym_ = false;
    std::vector<EID> off_;
    std::vector<VID> adj_;
    gg_prop *degp_ = nullptr;
    VID *deg_ = nullptr;
};

class GraphGPU {
public:
    GraphGPU() = default;
    explicit GraphGPU(gg_graph *g) : g_(g) { init(); }
    // From a host CSR with GraphCSx's accessors (the driver's
    // createGraph(G, npart, maxVL), bench/driver.C:12-19,110-116); the
    // partition count and vector length do not apply to the device layout.
    template <typename CSx, typename = decltype(std::declval<const CSx &>().getIndex())>
    explicit GraphGPU(const CSx &G, int npart = 0, int maxVL = 0) {
        (void)maxVL;
        gg_graph *g = nullptr;
        graptor_b200::check(gg_graph_upload(graptor_b200::context(), (uint32_t)G.numVertices(),
                                            (uint64_t)G.numEdges(), (const uint64_t *)G.getIndex(),
                                            (const uint32_t *)G.getEdges(), G.isSymmetric() ? 1 : 0, &g),
                            "gg_graph_upload");
        g_ = g;
        init();
        if (npart > 0) part_ = partitioner(g_, n_, npart);
        // the host CSR the device graph was built from (the same rows in the
        // same order): getCSR() serves it without a download
        make_csr_view((const EID *)G.getIndex(), (const VID *)G.getEdges());
    }
    static GraphGPU read_bin(const std::string &path, bool symmetric) {
        gg_graph *g = nullptr;
        graptor_b200::check(gg_graph_read_bin(graptor_b200::context(), path.c_str(), symmetric, &g),
                            "gg_graph_read_bin");
        return GraphGPU(g);
    }
    static GraphGPU from_csr(VID n, EID m, const EID *off, const VID *adj, bool symmetric) {
        gg_graph *g = nullptr;
        graptor_b200::check(gg_graph_upload(graptor_b200::context(), n, m, off, adj, symmetric, &g),
                            "gg_graph_upload");
        return GraphGPU(g);
    }
    VID numVertices() const { return n_; }
    EID numEdges() const { return m_; }
    bool isSymmetric() const { return sym_ != 0; }
    const partitioner &get_partitioner() const { return part_; }
    // the vector length the layout's pull traversal is built for: the device
    // processes one destination per lane, so analytics see scalar code paths
    static constexpr unsigned short getPullVLBound() { return 1; }
    static constexpr unsigned short getPushVLBound() { return 1; }
    VID getOutDegree(VID v) const { return getCSR().getDegree(v); }
    // The CSR in host memory, fetched once on first use.
    const GraphCSxView &getCSR() const {
        if (!csr_) make_csr_view(nullptr, nullptr);
        return *csr_;
    }
    // host CSR view: copied from off/adj, or downloaded from the device
    void make_csr_view(const EID *off, const VID *adj) const {
        {
            auto c = std::make_shared<GraphCSxView>();
            c->n_ = n_;
            c->m_ = m_;
            c->sym_ = sym_ != 0;
            if (off && adj) {
                c->off_.assign(off, off + (size_t)n_ + 1);
                c->adj_.assign(adj, adj + (size_t)m_);
                if (c->adj_.empty()) c->adj_.resize(1);
            } else {
                c->off_.resize((size_t)n_ + 1);
                c->adj_.resize(m_ ? m_ : 1);
                graptor_b200::check(gg_graph_download(g_, c->off_.data(), c->adj_.data()), "gg_graph_download");
            }
            graptor_b200::check(gg_prop_create_managed(g_, GG_U32, &c->degp_), "gg_prop_create_managed");
            void *d = nullptr;
            gg_prop_device_ptr(c->degp_, &d);
            c->deg_ = (VID *)d;
            for (VID i = 0; i < n_; ++i) c->deg_[i] = (VID)(c->off_[i + 1] - c->off_[i]);
            // never written again: host and device each keep their copy
            graptor_b200::check(gg_prop_prefetch(c->degp_, 2), "gg_prop_prefetch");
            graptor_b200::registry()[d] = c->degp_;
            csr_ = c;
        }
    }
    const GraphCSxView &getCSC() const { return getCSR(); }
    // no vertex renumbering on the device: ids are the file's ids
    VID remapID(VID v) const { return v; }
    VID originalID(VID v) const { return v; }
    gg_graph *handle() const { return g_; }
    // the layout has no partition fragments to report (GraphVEBOGraptor::fragmentation)
    void fragmentation() const {}
    void del() {
        if (g_) graptor_b200::dense_pool_release(g_);
        if (csr_ && csr_->degp_) {
            graptor_b200::registry().erase((const void *)csr_->deg_);
            gg_prop_destroy(csr_->degp_);
            csr_->degp_ = nullptr;
        }
        csr_.reset();
        if (g_) {
            if (graptor_b200::default_graph() == g_) graptor_b200::default_graph() = nullptr;
            gg_graph_destroy(g_);
        }
        g_ = nullptr;
    }

protected:
    void adopt(gg_graph *g) {
        g_ = g;
        init();
    }

private:
    void init() {
        uint64_t m = 0;
        graptor_b200::check(gg_graph_info(g_, &n_, &m, &sym_), "gg_graph_info");
        m_ = m;
        part_ = partitioner(g_, n_);
        graptor_b200::default_graph() = g_;
    }
    gg_graph *g_ = nullptr;
    VID n_ = 0;
    EID m_ = 0;
    int sym_ = 0;
    partitioner part_;
    mutable std::shared_ptr<GraphCSxView> csr_;
};

// A W-byte truth value (Graptor's logical<W>, all bits set = true).
template <unsigned short W> struct logical { unsigned char b[W]; };
// add_logical<T>::type: the logical of T's width (simd/ types)
template <typename T> struct add_logical { using type = logical<sizeof(T)>; };
namespace graptor_b200 {
template <> struct dtype_of<logical<4>> { static constexpr gg_dtype value = GG_U32; };
template <> struct dtype_of<logical<1>> { static constexpr gg_dtype value = GG_U8; };
}  // namespace graptor_b200

// ---------------------------------------------------------------------------
// Frontier (value handle with manual del(), frontier/frontier.h:58-716)
// ---------------------------------------------------------------------------
enum class frontier_type { ft_true = 0, ft_unbacked = 1, ft_bool = 2, ft_bit = 3, ft_logical1 = 4,
                           ft_logical2 = 5, ft_logical4 = 6, ft_logical8 = 7, ft_sparse = 8,
                           ft_bit2 = 9, ft_msb4 = 10, ft_N = 11 };

inline std::ostream &operator<<(std::ostream &os, frontier_type t) {
    static const char *names[] = {"true", "unbacked", "bool", "bit", "logical1", "logical2",
                                  "logical4", "logical8", "sparse", "bit2", "msb4", "N"};
    int i = (int)t;
    return os << names[(i >= 0 && i <= 11) ? i : 11];
}

// How an operator computes its output frontier (frontier/type.h:148-153);
// analytics name it in operator structs.
enum frontier_mode { fm_all_true = 0, fm_reduction = 1, fm_calculate = 2, fm_N = 3 };

class frontier {
public:
    frontier() = default;
    // frontier::create(n, v, deg): one active vertex
    static frontier create(VID n, VID v, VID deg) {
        frontier f;
        f.kind_ = K_SINGLE;
        f.n_ = n;
        f.v_ = v;
        f.nactv_ = 1;
        f.nacte_ = deg;
        return f;
    }
    static frontier all_true(VID n, EID m) {
        frontier f;
        f.kind_ = K_ALL;
        f.n_ = n;
        f.nactv_ = n;
        f.nacte_ = m;
        return f;
    }
    // frontier::sparse(n, k, list): k active vertices from a host array
    // (frontier.h:236-245); the list is copied, the caller keeps its array
    static frontier sparse(VID n, VID k, const VID *list) {
        frontier f;
        f.kind_ = K_LIST;
        f.n_ = n;
        f.list_ = std::make_shared<std::vector<VID>>(list, list + k);
        return f;
    }
    static frontier empty() { return frontier(); }
    // frontier::dense<W>(part) (frontier.h): one W-byte logical per vertex
    // in device memory, all clear, for vertex programs to write (all bits set
    // = active, APRv.C:365-367); calculateActiveCounts() makes it the
    // frontier's active set.  The array lives until del().
    template <unsigned short W> static frontier dense(const partitioner &part) {
        static_assert(W == 1 || W == 4, "dense logical frontiers of 1 or 4 bytes");
        frontier f;
        f.kind_ = K_DENSE;
        f.n_ = part.get_num_vertices();
        // device memory: vertex programs write it, calculateActiveCounts()
        // reads it; host code reads a frontier through getSparse / getDenseL
        const int dt = W == 4 ? GG_U32 : GG_U8;
        auto key = std::make_pair(part.graph(), dt);
        auto &free_list = graptor_b200::dense_pool()[key];
        gg_prop *p = nullptr;
        if (!free_list.empty()) {
            p = free_list.back();
            free_list.pop_back();
        } else {
            graptor_b200::check(gg_prop_create(part.graph(), (gg_dtype)dt, &p), "gg_prop_create");
        }
        const uint32_t zero = 0;
        graptor_b200::check(gg_prop_fill(p, &zero), "gg_prop_fill");
        void *d = nullptr;
        gg_prop_device_ptr(p, &d);
        graptor_b200::registry()[d] = p;
        f.dense_store_ = std::shared_ptr<gg_prop>(p, [d, key](gg_prop *q) {
            graptor_b200::registry().erase(d);
            graptor_b200::dense_pool()[key].push_back(q);
        });
        return f;
    }
    // the dense array of a frontier made by dense<W>()
    template <typename T> T *getDense() const {
        if (!dense_store_) throw graptor_b200::error(GG_ERR_STATE, "getDense() of a frontier without a dense array");
        void *d = nullptr;
        gg_prop_device_ptr(dense_store_.get(), &d);
        return (T *)d;
    }
    // the active set and its counts from the dense array (frontier.h:380-383)
    template <typename GraphType> void calculateActiveCounts(const GraphType &G) {
        if (!dense_store_) throw graptor_b200::error(GG_ERR_STATE, "calculateActiveCounts() without a dense array");
        gg_vmap_desc d;
        std::memset(&d, 0, sizeof(d));
        const uint8_t code[] = {GG_VM_LOAD, GG_VM_CONST, GG_VM_NE, GG_VM_FILTER};
        d.ncode = 4;
        for (int i = 0; i < 4; ++i) d.code[i] = code[i];
        d.props[0] = dense_store_.get();
        double red[GG_VM_MAX_REDUCE] = {0, 0, 0, 0};
        graptor_b200::before_device();
        graptor_b200::check(gg_vertexmap(G.handle(), &d, nullptr, output(G.handle()), red), "gg_vertexmap");
    }
    void del() {
        if (f_) gg_frontier_destroy(f_);
        f_ = nullptr;
        kind_ = K_EMPTY;
        dense_store_.reset();
    }
    bool isEmpty() const {
        if (kind_ == K_LIST) return list_->empty();
        return nActiveVertices() == 0;
    }
    VID nActiveVertices() const {
        if (kind_ == K_LIST) return (VID)list_->size();
        refresh();
        return (VID)nactv_;
    }
    EID nActiveEdges() const {
        if (kind_ == K_LIST) const_cast<frontier *>(this)->bind(graptor_b200::default_graph());
        refresh();
        return nacte_;
    }
    double density(EID m) const { return m ? (double(nActiveVertices()) + double(nActiveEdges())) / double(m) : 0.0; }
    frontier_type getType() const {
        return kind_ == K_ALL ? frontier_type::ft_true : kind_ == K_DEV ? frontier_type::ft_sparse
                                                                       : frontier_type::ft_unbacked;
    }
    bool is_set(VID v) const {
        if (kind_ == K_ALL) return true;
        if (kind_ == K_SINGLE) return v == v_;
        const VID *l = getSparse();
        for (VID i = 0, k = nActiveVertices(); i < k; ++i)
            if (l[i] == v) return true;
        return false;
    }
    // The active vertices as a host list (frontier::getSparse, frontier.h:681),
    // valid until the frontier changes; toSparse() is implied.
    const VID *getSparse() const {
        if (kind_ == K_LIST) return list_->data();
        if (kind_ == K_SINGLE) return &v_;
        auto h = std::make_shared<std::vector<VID>>();
        if (kind_ == K_ALL) {
            h->resize(n_);
            for (VID v = 0; v < n_; ++v) (*h)[v] = v;
        } else if (kind_ == K_DEV) {
            uint64_t k = 0;
            graptor_b200::check(gg_frontier_download(f_, nullptr, 0, &k), "gg_frontier_download");
            h->resize(k ? k : 1);
            graptor_b200::check(gg_frontier_download(f_, h->data(), k, &k), "gg_frontier_download");
            h->resize(k);
        }
        host_ = h;
        return host_->data();
    }
    void toSparse(const partitioner &) const {}
    // Dense host copy, one W-byte logical per vertex (-1 active, 0 not)
    // (frontier::getDenseL<W>, frontier.h:664).
    template <unsigned short W> logical<W> *getDenseL() const {
        const VID nv = n_ ? n_ : (f_ ? frontier_vertices() : 0);
        auto d = std::make_shared<std::vector<int64_t>>((nv * W + 7) / 8 + 1, 0);
        char *b = (char *)d->data();
        auto set = [&](VID v) { std::memset(b + (size_t)v * W, 0xFF, W); };
        if (kind_ == K_ALL) {
            for (VID v = 0; v < nv; ++v) set(v);
        } else {
            const VID *l = getSparse();
            for (VID i = 0, k = nActiveVertices(); i < k; ++i) set(l[i]);
        }
        dense_ = d;
        return (logical<W> *)d->data();
    }

    // --- library side ---
    // Device frontier for graph g (materialises a pending single/all frontier).
    gg_frontier *bind(gg_graph *g) {
        if (kind_ == K_DEV) return f_;
        if (!g) throw graptor_b200::error(GG_ERR_STATE, "frontier used before a graph exists");
        if (!f_) graptor_b200::check(gg_frontier_create(g, &f_), "gg_frontier_create");
        if (kind_ == K_SINGLE) graptor_b200::check(gg_frontier_set_single(f_, v_), "gg_frontier_set_single");
        else if (kind_ == K_ALL) graptor_b200::check(gg_frontier_set_all(f_), "gg_frontier_set_all");
        else if (kind_ == K_LIST)
            graptor_b200::check(gg_frontier_set_list(f_, list_->data(), list_->size()), "gg_frontier_set_list");
        else graptor_b200::check(gg_frontier_clear(f_), "gg_frontier_clear");
        kind_ = K_DEV;
        stale_ = true;
        return f_;
    }
    // An output frontier written by the device.
    gg_frontier *output(gg_graph *g) {
        if (!f_) graptor_b200::check(gg_frontier_create(g, &f_), "gg_frontier_create");
        kind_ = K_DEV;
        stale_ = true;
        return f_;
    }
    bool all() const { return kind_ == K_ALL; }

private:
    enum Kind { K_EMPTY, K_SINGLE, K_ALL, K_DEV, K_LIST, K_DENSE };
    VID frontier_vertices() const {
        uint32_t n = 0;
        graptor_b200::check(gg_graph_info(graptor_b200::default_graph(), &n, nullptr, nullptr), "gg_graph_info");
        return n;
    }
    void refresh() const {
        if (kind_ == K_DEV && stale_) {
            uint64_t v = 0, e = 0;
            graptor_b200::check(gg_frontier_counts(f_, &v, &e), "gg_frontier_counts");
            nactv_ = v;
            nacte_ = e;
            stale_ = false;
        }
    }
    Kind kind_ = K_EMPTY;
    gg_frontier *f_ = nullptr;
    VID n_ = 0, v_ = 0;
    mutable uint64_t nactv_ = 0;
    mutable EID nacte_ = 0;
    mutable bool stale_ = false;
    std::shared_ptr<std::vector<VID>> list_;                 // K_LIST: pending host list
    mutable std::shared_ptr<std::vector<VID>> host_;         // getSparse() copy
    mutable std::shared_ptr<std::vector<int64_t>> dense_;    // getDenseL() copy
    std::shared_ptr<gg_prop> dense_store_;                   // dense<W>() array
};

// ---------------------------------------------------------------------------
// Expression trees (the meaning of dsl/ast for the hot-path operators)
// ---------------------------------------------------------------------------
namespace expr {

enum class NK {
    VarSrc, VarDst, VarV, VarEdge, Const, Ref, Min, SetIf, Assign, AddAssign, MulAssign,
    Add, Sub, Mul, Div, Eq, Ne, Lt, Gt, Le, Ge, LAnd, LOr, Cast, Abs, Iif, MsbSet, Noop,
    OrAssign, BAnd, BOr, BXor, BNot, Let, Tmp, Seq, SetMask, MisOp, Pred, CvtVec
};

struct Node {
    NK k;
    std::vector<std::shared_ptr<Node>> c;
    double cval = 0;       // Const
    gg_dtype dt = GG_F64;  // Const / Ref / Cast: value type
    gg_prop *prop = nullptr;  // Ref: device array
    double *host = nullptr;   // Ref: host scalar accumulator (array_ro over a host variable)
    bool ones = false;        // Const _1s: all bits set in the type of the other operand
};
using NP = std::shared_ptr<Node>;

inline NP mk(NK k, std::vector<NP> c = {}) {
    auto n = std::make_shared<Node>();
    n->k = k;
    n->c = std::move(c);
    return n;
}

inline std::string show(const NP &n) {
    static const char *nm[] = {"s", "d", "v", "e", "const", "ref", "min", "setif", "=", "+=", "*=",
                               "+", "-", "*", "/", "==", "!=", "<", ">", "<=", ">=", "&&", "||",
                               "cast", "abs", "iif", "msbset", "noop", "|=", "&", "|", "^", "~", "let", "tmp",
                               "seq", "setmask", "mis", "pred", "cvtvec"};
    std::ostringstream os;
    if (n->k == NK::Const) return (os << n->cval, os.str());
    os << nm[(int)n->k];
    if (!n->c.empty()) {
        os << "(";
        for (size_t i = 0; i < n->c.size(); ++i) os << (i ? "," : "") << show(n->c[i]);
        os << ")";
    }
    return os.str();
}

class E;
template <typename T> E _c(T v);
inline E make_noop();

// An expression value.  Copying an E copies the handle, not the tree.
class E {
public:
    // one lane per expression value (the reference's vector length)
    static constexpr unsigned short VL = 1;
    E() : n_(mk(NK::Noop)) {}
    explicit E(NP n) : n_(std::move(n)) {}
    template <typename T, typename = std::enable_if_t<std::is_arithmetic<T>::value>>
    E(T v);  // literal operand
    const NP &node() const { return n_; }

    // a[d].min(x): relax to the minimum, "changed" as value
    E min(const E &x) const { return E(mk(NK::Min, {n_, x.n_})); }
    // a[d].setif(x): set when unset (msb set)
    E setif(const E &x) const { return E(mk(NK::SetIf, {n_, x.n_})); }
    E operator+=(const E &x) const { return E(mk(NK::AddAssign, {n_, x.n_})); }
    E operator*=(const E &x) const { return E(mk(NK::MulAssign, {n_, x.n_})); }
    // a[d] |= x: bitwise-or relax, "changed" as value (FMv.C:356-358)
    E operator|=(const E &x) const { return E(mk(NK::OrAssign, {n_, x.n_})); }
    // assignment builds a node (a[v] = x); E values are never re-seated
    E operator=(const E &x) const { return E(mk(NK::Assign, {n_, x.n_})); }
    // _0(vid): the zero index of a scalar accumulator (PRv.C:241)
    E operator()(const E &) const { return *this; }

private:
    NP n_;
};

inline E make_noop() { return E(mk(NK::Noop)); }

inline E cst(double v, gg_dtype dt) {
    auto n = mk(NK::Const);
    n->cval = v;
    n->dt = dt;
    return E(n);
}

template <typename T>
inline gg_dtype literal_dtype() {
    if (std::is_floating_point<T>::value) return sizeof(T) == 4 ? GG_F32 : GG_F64;
    return std::is_signed<T>::value ? GG_I32 : GG_U32;
}

template <typename T, typename>
inline E::E(T v) : n_(cst((double)v, literal_dtype<T>()).node()) {}

template <typename T> inline E _c(T v) { return cst((double)v, literal_dtype<T>()); }

// Result type of an arithmetic node, as C++ promotes: double if either side
// is double, else float if either side is float, else uint32 if either side
// is uint32, else the integer type.
inline gg_dtype promote(gg_dtype a, gg_dtype b) {
    if (a == GG_F64 || b == GG_F64) return GG_F64;
    if (a == GG_F32 || b == GG_F32) return GG_F32;
    if (a == GG_U32 || b == GG_U32) return GG_U32;
    return a;
}
// _1s takes the type of the operand it meets (dsl/ast/value.h: all bits
// set in the element type): 2^32-1 beside a uint32 operand, -1 elsewhere.
inline NP fit_ones(const NP &c, gg_dtype dt) {
    if (c->k != NK::Const || !c->ones) return c;
    auto n = mk(NK::Const);
    n->cval = dt == GG_U32 ? 4294967295.0 : -1.0;
    n->dt = dt;
    return n;
}
inline E binop(NK k, const E &a, const E &b) {
    const NP l = fit_ones(a.node(), b.node()->dt), r = fit_ones(b.node(), a.node()->dt);
    auto n = mk(k, {l, r});
    const bool arith = k == NK::Add || k == NK::Sub || k == NK::Mul || k == NK::Div;
    const bool bits = k == NK::BAnd || k == NK::BOr || k == NK::BXor;
    n->dt = arith || bits ? promote(l->dt, r->dt) : GG_I32;
    return E(n);
}
#define GG_BINOP(op, kind) \
    inline E operator op(const E &a, const E &b) { return binop(NK::kind, a, b); }
GG_BINOP(+, Add)
GG_BINOP(-, Sub)
GG_BINOP(*, Mul)
GG_BINOP(/, Div)
GG_BINOP(==, Eq)
GG_BINOP(!=, Ne)
GG_BINOP(<, Lt)
GG_BINOP(>, Gt)
GG_BINOP(<=, Le)
GG_BINOP(>=, Ge)
GG_BINOP(&&, LAnd)
GG_BINOP(||, LOr)
GG_BINOP(&, BAnd)
GG_BINOP(|, BOr)
GG_BINOP(^, BXor)
#undef GG_BINOP
inline E operator~(const E &a) {
    auto n = mk(NK::BNot, {a.node()});
    n->dt = a.node()->dt == GG_I32 ? GG_I32 : GG_U32;
    return E(n);
}

static const E _0 = cst(0, GG_I32);
static const E _1 = cst(1, GG_I32);
static const E _1s = [] {
    E e = cst(-1, GG_I32);
    e.node()->ones = true;
    return e;
}();
static const E _true = cst(1, GG_I32);
static const E _false = cst(0, GG_I32);

inline E zero_val(const E &) { return cst(0, GG_I32); }
inline E true_val(const E &) { return cst(1, GG_I32); }
// constant_val2(x, v): v in its own type T (dsl/ast/value.h:93-98)
template <typename T> inline E constant_val2(const E &, T v) { return cst((double)v, literal_dtype<T>()); }
// constant_val(x, v): v in the type of x (a float operand rounds v to float)
template <typename T> inline E constant_val(const E &x, T v) {
    const gg_dtype dt = x.node()->k == NK::Ref || x.node()->k == NK::Cast || x.node()->k == NK::Const
                            ? x.node()->dt : literal_dtype<T>();
    return cst(dt == GG_F32 ? (double)(float)v : (double)v, dt);
}
// The array id the reference gives the graph's degree array (PRv.C:46).
constexpr short aid_graph_degree = 127;
template <typename T> inline E cast(const E &a) {
    auto n = mk(NK::Cast, {a.node()});
    n->dt = literal_dtype<T>();
    return E(n);
}
inline E make_unop_abs(const E &a) {
    auto n = mk(NK::Abs, {a.node()});
    n->dt = a.node()->dt;
    return E(n);
}
// iif(c, l, r) selects r where c holds and l elsewhere, as the reference's
// blend (dsl/ast/ternop.h:65-125 -> blendm(m, l, r) = m ? r : l,
// target/scalar_int.h:212-214); the node keeps (c, taken, not taken)
inline E iif(const E &c, const E &l, const E &r) {
    const NP ln = fit_ones(l.node(), r.node()->dt), rn = fit_ones(r.node(), l.node()->dt);
    auto n = mk(NK::Iif, {c.node(), rn, ln});
    n->dt = promote(ln->dt, rn->dt);
    return E(n);
}
// let<AID>(init, cont): cont receives a reference to a temporary holding
// init (dsl/ast/binop.h:1540-1580); the temporary lives for one vertex
template <auto AID, typename Fn> inline E let(const E &init, Fn cont) {
    auto t = mk(NK::Tmp);
    t->dt = init.node()->dt;
    E body = cont(E(t));
    auto n = mk(NK::Let, {init.node(), body.node(), t});
    n->dt = body.node()->dt;
    return E(n);
}
// set_mask(c, x): x where c holds (dsl/ast/ctrl.h); remove_mask(x): x
inline E set_mask(const E &c, const E &x) {
    auto n = mk(NK::SetMask, {c.node(), x.node()});
    n->dt = x.node()->dt;
    return E(n);
}
inline E remove_mask(const E &x) { return x; }
// add_predicate(x, c): x where c holds; an update with it leaves the other
// vertices untouched (APRv.C:455-458)
inline E add_predicate(const E &x, const E &c) {
    auto n = mk(NK::Pred, {x.node(), c.node()});
    n->dt = x.node()->dt;
    return E(n);
}
template <typename Tr> inline E make_unop_cvt_to_mask(const E &x) { return x; }
// The maximal independent set relation (dsl/ast/dfsaop.h:49-230): state
// a[d], update a[s], condition s < d.
struct dfsaop_MIS {
    enum mis_state_t { mis_undecided = 0, mis_conditionally_in = 1, mis_out = 2, mis_in = 3 };
};
inline E make_dfsaop_MIS(const E &state, const E &update, const E &cond) {
    auto n = mk(NK::MisOp, {state.node(), update.node(), cond.node()});
    n->dt = state.node()->dt;
    return E(n);
}
// value<Tr, vk_zero>(): zero in Tr's element type (dsl/ast/value.h)
struct vk_zero {};
template <typename Tr, typename K> inline E value();

// make_seq(a, b, ...): the statements in order (dsl/ast/binop.h:370-395)
inline E make_seq() { return make_noop(); }
template <typename... R> inline E make_seq(const E &a, const R &... r) {
    auto n = mk(NK::Seq, {a.node(), E(r).node()...});
    n->dt = n->c.back()->dt;
    return E(n);
}
inline E msbset(const E &a) { return E(mk(NK::MsbSet, {a.node()})); }

inline E var(NK k) {
    auto n = mk(k);
    n->dt = GG_U32;  // vertex ids
    return E(n);
}

// Reference to element idx of a device array (or of a host scalar).
inline E ref(gg_prop *p, double *host, gg_dtype dt, const E &idx) {
    auto n = mk(NK::Ref, {idx.node()});
    n->prop = p;
    n->host = host;
    n->dt = dt;
    return E(n);
}

}  // namespace expr

// Vector type traits the analytics name in their lambdas (simd/ types):
// one lane on the device.
namespace simd {
template <typename T, unsigned short VL_> struct ty {
    using member_type = T;
    static constexpr unsigned short VL = VL_;
};
namespace detail {
template <typename T, unsigned short VL_> using mask_preferred_traits_type = ty<T, VL_>;
}  // namespace detail
}  // namespace simd

// Storage encodings (encoding.h / customfp.h types): the 16-bit formats are
// two-byte words here, used as storage types and template tags.
template <unsigned short E_, unsigned short M_> struct customfp { uint16_t bits; };
template <bool S_, unsigned short E_, unsigned short M_, bool Z_, int B_> struct scustomfp { uint16_t bits; };
template <typename T> struct array_encoding { using stored_type = T; };
template <typename T, bool = false> struct array_encoding_wide { using stored_type = T; };
// bitfield<B> / array_encoding_bit<B> (encoding.h:453-520): B-bit states.  On
// the device each state takes one byte; host reads give a bitfield value.
template <unsigned short B> struct bitfield {
    uint8_t v;
    uint8_t get() const { return v; }
    operator uint8_t() const { return v; }
};
template <typename T> class mmap_ptr;
struct numa_allocation_partitioned;
template <unsigned short B> struct array_encoding_bit {
    static constexpr unsigned short bits = B;
    using stored_type = uint8_t;
    using storage_type = uint8_t;
    static mmap_ptr<uint8_t> allocate(const numa_allocation_partitioned &a);
    static bitfield<B> get(const uint8_t *base, VID v);
};
template <typename Enc> struct is_bit_encoding : std::false_type { static constexpr unsigned short bits = 0; };
template <unsigned short B> struct is_bit_encoding<array_encoding_bit<B>> : std::true_type {
    static constexpr unsigned short bits = B;
};

namespace graptor_b200 {
template <> struct dtype_of<customfp<6, 10>> { static constexpr gg_dtype value = GG_CFP_6_10; };
template <> struct dtype_of<scustomfp<true, 8, 7, false, 0>> { static constexpr gg_dtype value = GG_BF16_TRUNC; };
template <typename T, typename = void> struct has_dtype : std::false_type {};
template <typename T> struct has_dtype<T, std::void_t<decltype(dtype_of<T>::value)>> : std::true_type {};
template <typename T, typename Enc> struct stored_of { using type = typename Enc::stored_type; };
template <typename T> struct stored_of<T, void> { using type = T; };
}  // namespace graptor_b200

namespace expr {
// expr::array_ro<T,VID,AID,Enc>(ptr) (dsl/ast/memref.h:57-110): a view of
// values of type T over an array stored as Enc::stored_type -- a device
// array registered by mmap_ptr / vertexprop, or a host scalar (reduction
// target).  Indexed with an expression it builds a tree; indexed with a
// VID from host code it reads or writes the (managed) array in place.
template <typename T, typename U = VID, short AID = 0, typename Enc = array_encoding<T>>
class array_ro {
public:
    using storage_type = typename graptor_b200::stored_of<T, Enc>::type;
    array_ro(storage_type *p) : ptr_(p) {
        auto &r = graptor_b200::registry();
        auto it = r.find((const void *)p);
        if (it != r.end()) prop_ = it->second;
        else host_ = reinterpret_cast<double *>(p);
        if (!prop_ && !std::is_same<storage_type, double>::value)
            throw graptor_b200::error(GG_ERR_UNSUPPORTED, "array_ro over host memory must be a double scalar");
    }
    E operator[](const E &i) const { return ref(prop_, host_, graptor_b200::dtype_of<T>::value, i); }
    // host writes need no flush: the next kernel, queued after them, sees them
    // (states of a bit encoding are read on the host as bitfield values)
    using host_ref = std::conditional_t<is_bit_encoding<Enc>::value, bitfield<is_bit_encoding<Enc>::bits>,
                                        storage_type &>;
    using host_cref = std::conditional_t<is_bit_encoding<Enc>::value, bitfield<is_bit_encoding<Enc>::bits>,
                                         const storage_type &>;
    host_ref operator[](VID v) {
        graptor_b200::host_sync();
        if constexpr (is_bit_encoding<Enc>::value) return host_ref{ptr_[v]};
        else return ptr_[v];
    }
    host_cref operator[](VID v) const {
        graptor_b200::host_sync();
        if constexpr (is_bit_encoding<Enc>::value) return host_cref{ptr_[v]};
        else return ptr_[v];
    }
    storage_type *ptr() const { return ptr_; }
    // the same array viewed as its stored type (dsl/ast/memref.h:95-106)
    array_ro<typename Enc::stored_type, U, AID, Enc> observe_stored() const {
        return array_ro<typename Enc::stored_type, U, AID, Enc>(ptr_);
    }

private:
    storage_type *ptr_ = nullptr;
    gg_prop *prop_ = nullptr;
    double *host_ = nullptr;
};

}  // namespace expr

namespace graptor_b200 {
template <typename T, typename Enc> struct storage_dtype { static constexpr gg_dtype value = dtype_of<T>::value; };
template <typename T> struct storage_dtype<T, array_encoding<customfp<6, 10>>> { static constexpr gg_dtype value = GG_CFP_6_10; };
template <typename T> struct storage_dtype<T, array_encoding_wide<customfp<6, 10>>> { static constexpr gg_dtype value = GG_CFP_6_10; };
template <typename T> struct storage_dtype<T, array_encoding_wide<scustomfp<true, 8, 7, false, 0>>> { static constexpr gg_dtype value = GG_BF16_TRUNC; };
template <typename T, typename S> struct storage_dtype<T, array_encoding<S>> { static constexpr gg_dtype value = dtype_of<S>::value; };

// Host-side element proxy: reads/writes one element through the C ABI.
template <typename T>
class elem_proxy {
public:
    elem_proxy(gg_prop *p, VID v) : p_(p), v_(v) {}
    elem_proxy &operator=(T x) {
        check(gg_prop_set(p_, v_, &x), "gg_prop_set");
        ++device_epoch();
        return *this;
    }
    operator T() const {
        T x{};
        check(gg_prop_get(p_, v_, &x), "gg_prop_get");
        return x;
    }

private:
    gg_prop *p_;
    VID v_;
};

template <typename T>
class ptr_proxy {
public:
    explicit ptr_proxy(gg_prop *p) : p_(p) {}
    elem_proxy<T> operator[](VID v) const { return elem_proxy<T>(p_, v); }

private:
    gg_prop *p_;
};
}  // namespace graptor_b200

// mmap_ptr<T> (mm.h:680-945): an array of one element per vertex that the
// analytics index from host code as well as hand to the edgemap.  Element
// types the device knows live in managed memory (gg_prop_create_managed) and
// are registered as vertex properties; other types (size_t counters of the
// host-side helpers) are plain host arrays.  Host indexing first waits for
// the device work queued so far.
struct numa_allocation_partitioned {
    explicit numa_allocation_partitioned(const partitioner &p) : part(p) {}
    partitioner part;
};

template <typename T>
class mmap_ptr {
public:
    using type = T;
    void allocate(const numa_allocation_partitioned &a) {
        if constexpr (graptor_b200::has_dtype<T>::value) {
            // device arrays hold one element per vertex
            if (a.part.get_scale() != 1)
                throw graptor_b200::error(GG_ERR_UNSUPPORTED, "mmap_ptr of more than one element per vertex");
            graptor_b200::check(gg_prop_create_managed(a.part.graph(), graptor_b200::dtype_of<T>::value, &p_),
                                "gg_prop_create_managed");
            void *d = nullptr;
            gg_prop_device_ptr(p_, &d);
            graptor_b200::registry()[d] = p_;
            d_ = (T *)d;
            st_ = std::make_shared<graptor_b200::managed_state>();
            st_->p = p_;
        } else {
            d_ = (T *)std::calloc((size_t)a.part.get_num_elements() + 1, sizeof(T));
            if (!d_) throw graptor_b200::error(GG_ERR_OOM, "mmap_ptr host allocation");
        }
    }
    // the array, for host reads and writes: waits for the device work queued
    // so far and brings the pages to the host
    T *get() const {
        access();
        return d_;
    }
    operator T *() {
        access();
        return d_;
    }
    operator const T *() const { return d_; }
    explicit operator bool() const { return d_ != nullptr; }
    // host writes need no flush: the next kernel, queued after them, sees them
    T &operator[](size_t v) {
        access();
        return d_[v];
    }
    const T &operator[](size_t v) const {
        access();
        return d_[v];
    }
    void del() {
        if (p_) {
            graptor_b200::registry().erase(d_);
            graptor_b200::host_touched().erase(st_.get());
            st_.reset();
            gg_prop_destroy(p_);
        } else {
            std::free(d_);
        }
        p_ = nullptr;
        d_ = nullptr;
    }
    gg_prop *handle() const { return p_; }

private:
    void access() const {
        if (st_ && (st_->on_device || !st_->touched)) graptor_b200::host_access(st_.get());
        else graptor_b200::host_sync();
    }
    gg_prop *p_ = nullptr;
    T *d_ = nullptr;
    std::shared_ptr<graptor_b200::managed_state> st_;  // shared by copies
};

template <unsigned short B> mmap_ptr<uint8_t> array_encoding_bit<B>::allocate(const numa_allocation_partitioned &a) {
    mmap_ptr<uint8_t> p;
    p.allocate(a);
    return p;
}
template <unsigned short B> bitfield<B> array_encoding_bit<B>::get(const uint8_t *base, VID v) {
    graptor_b200::host_sync();
    return bitfield<B>{base[v]};
}

namespace expr {
// make_unop_cvt_to_vector<logical<W>>(c): c as a W-byte logical, all bits
// set where c holds (APRv.C:411-415)
template <typename T> inline E make_unop_cvt_to_vector(const E &c) {
    auto n = mk(NK::CvtVec, {c.node()});
    n->dt = graptor_b200::dtype_of<T>::value;
    return E(n);
}
template <typename Tr, typename K> inline E value() {
    static_assert(std::is_same<K, vk_zero>::value, "only the zero value kind");
    return cst(0, graptor_b200::dtype_of<typename Tr::member_type>::value);
}
}  // namespace expr

namespace api {

// ---------------------------------------------------------------------------
// vertexprop (api/vertexprop.h:30-140)
// ---------------------------------------------------------------------------
template <typename T, typename U = VID, short AID = 0, typename Enc = array_encoding<T>>
class vertexprop {
public:
    vertexprop(const partitioner &part, const char *name = nullptr) {
        (void)name;
        graptor_b200::check(gg_prop_create(part.graph(), graptor_b200::storage_dtype<T, Enc>::value, &p_),
                            "gg_prop_create");
        void *d = nullptr;
        gg_prop_device_ptr(p_, &d);
        graptor_b200::registry()[d] = p_;
        n_ = part.get_num_vertices();
    }
    static vertexprop create(const partitioner &part, const char *name = nullptr) { return vertexprop(part, name); }
    void del() {
        if (p_) {
            void *d = nullptr;
            gg_prop_device_ptr(p_, &d);
            graptor_b200::registry().erase(d);
            gg_prop_destroy(p_);
        }
        p_ = nullptr;
    }
    expr::E operator[](const expr::E &i) const {
        return expr::ref(p_, nullptr, graptor_b200::storage_dtype<T, Enc>::value, i);
    }
    // host read (vertexprop::operator[](VID)): served from a host mirror
    // refreshed when the device has written since the last read
    T operator[](VID v) const {
        if (mirror_epoch_.load() != graptor_b200::device_epoch().load() || mirror_n_.load() != n_) {
            std::lock_guard<std::mutex> lock(graptor_b200::host_mutex());
            const uint64_t e = graptor_b200::device_epoch().load();
            if (mirror_epoch_.load() != e || mirror_n_.load() != n_) {
                mirror_.resize(n_);
                graptor_b200::check(gg_prop_download(p_, mirror_.data()), "gg_prop_download");
                mirror_n_.store(n_);
                mirror_epoch_.store(e);
            }
        }
        return mirror_[v];
    }
    void set(VID v, T t) {
        graptor_b200::check(gg_prop_set(p_, v, &t), "gg_prop_set");
        ++graptor_b200::device_epoch();
    }
    graptor_b200::ptr_proxy<T> get_ptr() const { return graptor_b200::ptr_proxy<T>(p_); }
    void fill(const partitioner &, T val) {
        graptor_b200::check(gg_prop_fill(p_, &val), "gg_prop_fill");
        ++graptor_b200::device_epoch();
    }
    gg_prop *handle() const { return p_; }

private:
    gg_prop *p_ = nullptr;
    VID n_ = 0;
    mutable std::vector<T> mirror_;
    mutable graptor_b200::catomic<uint64_t> mirror_epoch_{0};
    mutable graptor_b200::catomic<VID> mirror_n_{0};
};

// ---------------------------------------------------------------------------
// Argument tags and argument objects (api.h:130-1985)
// ---------------------------------------------------------------------------
enum class filter_strength { weak, strong };
enum class filter_entity { src, dst };
enum class frontier_record { frontier_reduction, frontier_method, frontier_reduction_or_method };
template <filter_strength S> struct filter_strength_argument {};
template <filter_entity E_> struct filter_entity_argument {};
template <frontier_record R> struct frontier_record_argument {};
static constexpr filter_strength_argument<filter_strength::weak> weak{};
static constexpr filter_strength_argument<filter_strength::strong> strong{};
static constexpr filter_entity_argument<filter_entity::src> src{};
static constexpr filter_entity_argument<filter_entity::dst> dst{};
static constexpr frontier_record_argument<frontier_record::frontier_reduction> reduction{};
static constexpr frontier_record_argument<frontier_record::frontier_method> method{};
static constexpr frontier_record_argument<frontier_record::frontier_reduction_or_method> reduction_or_method{};

struct default_threshold {
    bool is_sparse(VID nactv, EID nacte, EID m) const { return (EID(nactv) + nacte) <= (m / 20); }
    bool is_sparse(const frontier &F, EID m) const { return is_sparse(F.nActiveVertices(), F.nActiveEdges(), m); }
};
class frac_threshold {
public:
    explicit frac_threshold(int k) : k_(k) {}
    bool is_sparse(VID nactv, EID nacte, EID m) const {
        return float(EID(nactv) + nacte) <= float(m) / (100.0f / (float)k_);
    }
    int k() const { return k_; }

private:
    int k_;
};
struct always_sparse_t {};
struct always_dense_t {};
struct learned_threshold_t {};
static constexpr always_sparse_t always_sparse{};
static constexpr always_dense_t always_dense{};
static constexpr learned_threshold_t learned_threshold{};
struct fusion_select { explicit fusion_select(bool e = true) : enable(e) {} bool enable; };

struct arg_config {
    int threshold = GG_THRESH_DEFAULT;
    int k = 0;
    bool fusion = true;
};
inline void config_one(arg_config &, const default_threshold &) {}
inline void config_one(arg_config &c, const frac_threshold &t) { c.threshold = GG_THRESH_FRAC; c.k = t.k(); }
inline void config_one(arg_config &c, const always_sparse_t &) { c.threshold = GG_THRESH_ALWAYS_SPARSE; }
inline void config_one(arg_config &c, const always_dense_t &) { c.threshold = GG_THRESH_ALWAYS_DENSE; }
inline void config_one(arg_config &c, const learned_threshold_t &) { c.threshold = GG_THRESH_LEARNED; }
inline void config_one(arg_config &c, const fusion_select &f) { c.fusion = f.enable; }
template <typename... A> arg_config config(const A &... a) {
    arg_config c;
    (config_one(c, a), ...);
    return c;
}

template <typename Fn> struct arg_relax { Fn fn; };
template <typename Fn> arg_relax<Fn> relax(Fn fn) { return arg_relax<Fn>{fn}; }
template <typename Fn> struct arg_fusion { Fn fn; };
template <typename Fn> arg_fusion<Fn> fusion(Fn fn) { return arg_fusion<Fn>{fn}; }

// A frontier filter: on sources (the input frontier), or on destinations
// (api::filter(F, dst, strong), MISv.C:254: every source active).  The
// reference takes the three arguments in any order.
struct arg_filter_src { frontier *F; bool strong; bool dst; };
template <typename Fn> struct arg_filter_dst { Fn fn; bool strong; };
template <filter_strength S, filter_entity E_>
arg_filter_src filter(filter_strength_argument<S>, filter_entity_argument<E_>, frontier &F) {
    return arg_filter_src{&F, S == filter_strength::strong, E_ == filter_entity::dst};
}
template <filter_strength S, filter_entity E_>
arg_filter_src filter(frontier &F, filter_strength_argument<S>, filter_entity_argument<E_>) {
    return arg_filter_src{&F, S == filter_strength::strong, E_ == filter_entity::dst};
}
template <filter_strength S, filter_entity E_>
arg_filter_src filter(frontier &F, filter_entity_argument<E_>, filter_strength_argument<S>) {
    return arg_filter_src{&F, S == filter_strength::strong, E_ == filter_entity::dst};
}
template <filter_strength S, filter_entity E_>
arg_filter_src filter(filter_entity_argument<E_>, filter_strength_argument<S>, frontier &F) {
    return arg_filter_src{&F, S == filter_strength::strong, E_ == filter_entity::dst};
}
template <filter_strength S, typename Fn>
arg_filter_dst<Fn> filter(filter_strength_argument<S>, filter_entity_argument<filter_entity::dst>, Fn fn) {
    return arg_filter_dst<Fn>{fn, S == filter_strength::strong};
}

struct no_method {};
template <typename Fn> struct arg_record { frontier *out; frontier_record kind; Fn fn; bool has_fn; };
template <filter_strength S = filter_strength::strong>
arg_record<no_method> record(frontier &f, filter_strength_argument<S> = strong) {
    return arg_record<no_method>{&f, frontier_record::frontier_reduction, no_method{}, false};
}
template <frontier_record R, filter_strength S = filter_strength::strong>
arg_record<no_method> record(frontier &f, frontier_record_argument<R>, filter_strength_argument<S> = strong) {
    return arg_record<no_method>{&f, R, no_method{}, false};
}
template <typename Fn, filter_strength S = filter_strength::strong,
          typename = std::enable_if_t<std::is_invocable<Fn, expr::E>::value>>
arg_record<Fn> record(frontier &f, Fn fn, filter_strength_argument<S> = strong) {
    return arg_record<Fn>{&f, frontier_record::frontier_method, fn, true};
}
template <frontier_record R, typename Fn, filter_strength S = filter_strength::strong,
          typename = std::enable_if_t<std::is_invocable<Fn, expr::E>::value>>
arg_record<Fn> record(frontier &f, frontier_record_argument<R>, Fn fn, filter_strength_argument<S> = strong) {
    return arg_record<Fn>{&f, R, fn, true};
}

}  // namespace api

// ---------------------------------------------------------------------------
// Lowering: expression trees -> gg_emap_desc / gg_vmap_desc
// ---------------------------------------------------------------------------
namespace graptor_b200 {
using expr::NK;
using expr::NP;

[[noreturn]] inline void unsupported(const char *what, const NP &n) {
    throw error(GG_ERR_UNSUPPORTED, std::string(what) + " not on the hot path: " + expr::show(n));
}

inline bool is_ref_at(const NP &n, NK var) { return n->k == NK::Ref && n->prop && n->c[0]->k == var; }
inline bool is_const(const NP &n, double v) { return n->k == NK::Const && n->cval == v; }
inline NP strip_cast(const NP &n) { return n->k == NK::Cast ? n->c[0] : n; }

// relax(s,d,e) -> descriptor fields: a[d].min(a[s] + 1) -> MIN_PLUS1_I32,
// a[d].min(a[s]) -> MIN_U32, a[d].setif(s) -> SETIF_U32,
// y[d] += cast(contrib[s]) -> ADD_GATHER
inline void lower_relax(const NP &r, gg_emap_desc &d) {
    if (r->k == NK::Min && is_ref_at(r->c[0], NK::VarDst)) {
        const NP &a = r->c[0], &x = r->c[1];
        if (x->k == NK::Add && is_ref_at(x->c[0], NK::VarSrc) && x->c[0]->prop == a->prop && is_const(x->c[1], 1) &&
            a->dt == GG_I32) {
            d.relax = GG_RELAX_MIN_PLUS1_I32;  // a[d].min(a[s] + _1)
            d.a = a->prop;
            return;
        }
        if (is_ref_at(x, NK::VarSrc) && x->prop == a->prop && a->dt == GG_U32) {
            d.relax = GG_RELAX_MIN_U32;  // a[d].min(a[s])
            d.a = a->prop;
            return;
        }
    }
    if (r->k == NK::Ne && is_ref_at(r->c[0], NK::VarDst) && is_ref_at(r->c[1], NK::VarSrc) &&
        r->c[0]->prop == r->c[1]->prop && r->c[0]->dt == GG_U32) {
        d.relax = GG_RELAX_NE_CHECK;  // a[d] != a[s]: record d, write nothing (CCv.C:612-617)
        d.a = r->c[0]->prop;
        return;
    }
    // a[s] > a[d] + 1 || a[s] < a[d] - 1 and a[s] < a[d] - 1 on int32 levels (BFSLVLv.C:288-305)
    auto ahead = [](const NP &x, gg_prop *&p) {  // a[s] < a[d] - 1
        if (x->k == NK::Lt && is_ref_at(x->c[0], NK::VarSrc) && x->c[1]->k == NK::Sub &&
            is_ref_at(x->c[1]->c[0], NK::VarDst) && is_const(x->c[1]->c[1], 1) && x->c[0]->prop == x->c[1]->c[0]->prop &&
            x->c[0]->dt == GG_I32) {
            p = x->c[0]->prop;
            return true;
        }
        return false;
    };
    auto behind = [](const NP &x, gg_prop *&p) {  // a[s] > a[d] + 1
        if (x->k == NK::Gt && is_ref_at(x->c[0], NK::VarSrc) && x->c[1]->k == NK::Add &&
            is_ref_at(x->c[1]->c[0], NK::VarDst) && is_const(x->c[1]->c[1], 1) && x->c[0]->prop == x->c[1]->c[0]->prop &&
            x->c[0]->dt == GG_I32) {
            p = x->c[0]->prop;
            return true;
        }
        return false;
    };
    {
        gg_prop *p1 = nullptr, *p2 = nullptr;
        if (r->k == NK::LOr && behind(r->c[0], p1) && ahead(r->c[1], p2) && p1 == p2) {
            d.relax = GG_RELAX_GAP_CHECK;
            d.a = p1;
            return;
        }
        if (ahead(r, p1)) {
            d.relax = GG_RELAX_AHEAD_CHECK;
            d.a = p1;
            return;
        }
    }
    // set_mask(s != d, make_dfsaop_MIS(a[d], a[s], s < d)) on uint8 states (MISv.C:235-245)
    if (r->k == NK::SetMask && r->c[0]->k == NK::Ne && r->c[0]->c[0]->k == NK::VarSrc &&
        r->c[0]->c[1]->k == NK::VarDst && r->c[1]->k == NK::MisOp) {
        const NP &op = r->c[1];
        if (is_ref_at(op->c[0], NK::VarDst) && is_ref_at(op->c[1], NK::VarSrc) && op->c[0]->prop == op->c[1]->prop &&
            op->c[0]->dt == GG_U8 && op->c[2]->k == NK::Lt && op->c[2]->c[0]->k == NK::VarSrc &&
            op->c[2]->c[1]->k == NK::VarDst) {
            d.relax = GG_RELAX_MIS_U8;
            d.a = op->c[0]->prop;
            return;
        }
    }
    if (r->k == NK::OrAssign && is_ref_at(r->c[0], NK::VarDst) && is_ref_at(r->c[1], NK::VarSrc) &&
        r->c[0]->dt == GG_U32 && r->c[1]->dt == GG_U32) {
        d.relax = GG_RELAX_OR_U32;  // a[d] |= b[s] (FMv.C:356-358)
        d.a = r->c[0]->prop;
        d.src = r->c[1]->prop;
        return;
    }
    if (r->k == NK::SetIf && is_ref_at(r->c[0], NK::VarDst) && r->c[1]->k == NK::VarSrc && r->c[0]->dt == GG_U32) {
        d.relax = GG_RELAX_SETIF_U32;  // a[d].setif(s)
        d.a = r->c[0]->prop;
        return;
    }
    if (r->k == NK::AddAssign && is_ref_at(r->c[0], NK::VarDst)) {
        const NP x = strip_cast(r->c[1]);
        if (is_ref_at(x, NK::VarSrc)) {
            d.relax = GG_RELAX_ADD_GATHER;  // y[d] += cast(contrib[s])
            d.a = r->c[0]->prop;
            d.src = x->prop;
            d.accum_f64 = r->c[1]->k == NK::Cast ? (r->c[1]->dt == GG_F64) : (r->c[0]->dt == GG_F64);
            return;
        }
    }
    unsupported("relax", r);
}

inline void lower_dst_filter(const NP &f, gg_emap_desc &d) {
    if (f->k == NK::Gt && is_ref_at(f->c[0], NK::VarDst) && f->c[1]->k == NK::Const) {
        d.dst_filter = GG_FILTER_GT_CONST;
        d.dst_filter_prop = f->c[0]->prop;
        d.dst_filter_k = (int64_t)f->c[1]->cval;
        return;
    }
    if (f->k == NK::Ne && is_ref_at(f->c[0], NK::VarDst) && is_const(f->c[1], 0)) {
        d.dst_filter = GG_FILTER_NE_ZERO;
        d.dst_filter_prop = f->c[0]->prop;
        return;
    }
    if (f->k == NK::Ne && is_ref_at(f->c[0], NK::VarDst) && f->c[1]->k == NK::Const) {
        d.dst_filter = GG_FILTER_NE_CONST;  // a[d] != k, e.g. k = _1s (FMv.C:353-354)
        d.dst_filter_prop = f->c[0]->prop;
        d.dst_filter_k = (int64_t)f->c[1]->cval;
        return;
    }
    if (f->k == NK::MsbSet && is_ref_at(f->c[0], NK::VarDst)) {
        d.dst_filter = GG_FILTER_MSB_SET;
        d.dst_filter_prop = f->c[0]->prop;
        return;
    }
    unsupported("dst filter", f);
}

inline void lower_record_method(const NP &m, gg_emap_desc &d) {
    if (m->k == NK::Eq && is_ref_at(m->c[0], NK::VarDst) && is_const(m->c[1], 0)) {
        d.record = GG_RECORD_EQ_ZERO;  // a[d] == 0 (MISv.C:246-253)
        return;
    }
    if (m->k == NK::Ne && is_ref_at(m->c[0], NK::VarDst) && is_ref_at(m->c[1], NK::VarDst)) {
        d.record = GG_RECORD_NE_PREV;  // a[d] != prev[d]
        d.prev = m->c[1]->prop;
        return;
    }
    unsupported("record method", m);
}

// Vertex statements -> stack program
struct VmBuilder {
    gg_vmap_desc d;
    std::vector<double *> red_targets;
    VmBuilder() { std::memset(&d, 0, sizeof(d)); }
    int prop_slot(gg_prop *p) {
        for (int i = 0; i < GG_VM_MAX_PROPS; ++i) {
            if (d.props[i] == p) return i;
            if (!d.props[i]) { d.props[i] = p; return i; }
        }
        return -1;
    }
    int const_slot(double v) {
        for (int i = 0; i < GG_VM_MAX_CONSTS; ++i) {
            if (i < nconst && d.consts[i] == v) return i;
        }
        if (nconst >= GG_VM_MAX_CONSTS) return -1;
        d.consts[nconst] = v;
        return nconst++;
    }
    int red_slot(double *h) {
        for (size_t i = 0; i < red_targets.size(); ++i) if (red_targets[i] == h) return (int)i;
        if (red_targets.size() >= GG_VM_MAX_REDUCE) return -1;
        red_targets.push_back(h);
        d.nreduce = (int)red_targets.size();
        return d.nreduce - 1;
    }
    bool emit(int op, int arg = 0) {
        if (d.ncode >= GG_VM_MAX_CODE) return false;
        d.code[d.ncode] = (uint8_t)op;
        d.arg[d.ncode] = (uint8_t)arg;
        ++d.ncode;
        return true;
    }
    int nconst = 0;
    int saved_code = 0, saved_const = 0;
    gg_vmap_desc saved;
    std::vector<double *> saved_red;
    std::map<const expr::Node *, int> tmps, saved_tmps;  // let temporaries -> slot
    void mark() { saved = d; saved_code = d.ncode; saved_const = nconst; saved_red = red_targets; saved_tmps = tmps; }
    void undo() { d = saved; nconst = saved_const; red_targets = saved_red; tmps = saved_tmps; }
    // let: evaluate init into a fresh temporary slot
    bool bind(const NP &let) {
        if (tmps.size() >= GG_VM_MAX_TMP) unsupported("let (too many temporaries)", let);
        const int slot = (int)tmps.size();
        if (!value(let->c[0]) || !emit(GG_VM_TSET, slot)) return false;
        tmps[let->c[2].get()] = slot;
        return true;
    }

    bool value(const NP &n) {
        switch (n->k) {
        case NK::Const: { int c = const_slot(n->cval); return c >= 0 && emit(GG_VM_CONST, c); }
        case NK::VarV: return emit(GG_VM_VID);
        case NK::Ref: {
            if (n->c[0]->k != NK::VarV || !n->prop) unsupported("vertex operand", n);
            int s = prop_slot(n->prop);
            return s >= 0 && emit(GG_VM_LOAD, s) && (n->dt == GG_F32 ? emit(GG_VM_TOF32) : true);
        }
        case NK::Add: case NK::Sub: case NK::Mul: case NK::Div: case NK::Eq: case NK::Ne:
        case NK::Lt: case NK::Gt: case NK::Le: case NK::Ge: case NK::BAnd: case NK::BOr: case NK::BXor: {
            static const std::map<NK, int> ops = {{NK::Add, GG_VM_ADD}, {NK::Sub, GG_VM_SUB}, {NK::Mul, GG_VM_MUL},
                                                  {NK::Div, GG_VM_DIV}, {NK::Eq, GG_VM_EQ}, {NK::Ne, GG_VM_NE},
                                                  {NK::Lt, GG_VM_LT}, {NK::Gt, GG_VM_GT}, {NK::Le, GG_VM_LE},
                                                  {NK::Ge, GG_VM_GE}, {NK::BAnd, GG_VM_AND}, {NK::BOr, GG_VM_OR},
                                                  {NK::BXor, GG_VM_XOR}};
            if (!value(n->c[0]) || !value(n->c[1]) || !emit(ops.at(n->k))) return false;
            const bool arith = n->k == NK::Add || n->k == NK::Sub || n->k == NK::Mul || n->k == NK::Div;
            // float arithmetic (float operands, no double one) rounds like the reference
            if (n->dt == GG_F32 && arith) return emit(GG_VM_TOF32);
            // uint32 arithmetic wraps modulo 2^32
            if (n->dt == GG_U32 && arith && n->k != NK::Div) return emit(GG_VM_TOU32);
            return true;
        }
        case NK::BNot: return value(n->c[0]) && emit(GG_VM_NOT);
        case NK::Tmp: {
            auto it = tmps.find(n.get());
            if (it == tmps.end()) unsupported("temporary outside its let", n);
            return emit(GG_VM_TGET, it->second);
        }
        case NK::Let: return bind(n) && value(n->c[1]);
        case NK::Pred: {  // c ? x : 0
            int z = const_slot(0.0);
            return z >= 0 && value(n->c[1]) && value(n->c[0]) && emit(GG_VM_CONST, z) && emit(GG_VM_SELECT);
        }
        case NK::CvtVec: {  // (c != 0) * all-ones
            int z = const_slot(0.0), o = const_slot(n->dt == GG_U8 ? 255.0 : 4294967295.0);
            return z >= 0 && o >= 0 && value(n->c[0]) && emit(GG_VM_CONST, z) && emit(GG_VM_NE) &&
                   emit(GG_VM_CONST, o) && emit(GG_VM_MUL);
        }
        case NK::Cast: {
            if (!value(n->c[0])) return false;
            return n->dt == GG_F32 ? emit(GG_VM_TOF32) : true;
        }
        case NK::Abs: return value(n->c[0]) && emit(GG_VM_ABS);
        case NK::Iif: return value(n->c[0]) && value(n->c[1]) && value(n->c[2]) && emit(GG_VM_SELECT);
        default: unsupported("vertex expression", n);
        }
    }
    // one statement; returns false when the program is full
    bool statement(const NP &s) {
        mark();
        const bool ok = stmt(s);
        if (!ok) undo();
        return ok;
    }
    bool stmt(const NP &s) {
        bool ok = true;
        if (s->k == NK::Noop) return true;
        if (s->k == NK::Seq) {
            for (const NP &c : s->c)
                if (!stmt(c)) return false;
            return true;
        }
        if (s->k == NK::Let) return bind(s) && stmt(s->c[1]);
        const NP &lhs = s->c.empty() ? s : s->c[0];
        if (lhs->k != NK::Ref) unsupported("vertex statement", s);
        if (lhs->host) {  // scalar accumulator: accum[_0(v)] += x
            if (s->k != NK::AddAssign) unsupported("scalar statement", s);
            int r = red_slot(lhs->host);
            ok = r >= 0 && value(s->c[1]) && emit(GG_VM_REDUCE_ADD, r);
        } else {
            if (lhs->c[0]->k != NK::VarV) unsupported("vertex statement", s);
            int p = prop_slot(lhs->prop);
            ok = p >= 0;
            if (ok) {
                if (s->k == NK::Assign) ok = value(s->c[1]) && emit(GG_VM_STORE, p);
                else if (s->k == NK::AddAssign && s->c[1]->k == NK::Pred)  // c ? a + x : a
                    ok = value(s->c[1]->c[1]) && emit(GG_VM_LOAD, p) && value(s->c[1]->c[0]) && emit(GG_VM_ADD) &&
                         (lhs->dt == GG_F32 ? emit(GG_VM_TOF32) : true) && emit(GG_VM_LOAD, p) &&
                         emit(GG_VM_SELECT) && emit(GG_VM_STORE, p);
                else if (s->k == NK::AddAssign) ok = emit(GG_VM_LOAD, p) && value(s->c[1]) && emit(GG_VM_ADD) && emit(GG_VM_STORE, p);
                else if (s->k == NK::MulAssign) ok = emit(GG_VM_LOAD, p) && value(s->c[1]) && emit(GG_VM_MUL) && emit(GG_VM_STORE, p);
                else unsupported("vertex statement", s);
            }
        }
        return ok;
    }
};

inline void run_vmap(gg_graph *g, VmBuilder &b, gg_frontier *filter, gg_frontier *out) {
    before_device();
    double red[GG_VM_MAX_REDUCE] = {0, 0, 0, 0};
    check(gg_vertexmap(g, &b.d, filter, out, red), "gg_vertexmap");
    ++device_epoch();
    for (size_t i = 0; i < b.red_targets.size(); ++i) *b.red_targets[i] += red[i];
}

}  // namespace graptor_b200

// ---------------------------------------------------------------------------
// Lazy executor (dsl/vertexmap.h:2120-2446): queued steps, merged passes
// ---------------------------------------------------------------------------
class lazy_executor {
public:
    explicit lazy_executor(const partitioner &part) : part_(part) {}

    template <typename Fn> lazy_executor &vertex_map(Fn fn) {
        stmts_.push_back(fn(expr::var(expr::NK::VarV)).node());
        return *this;
    }
    // vertex_map(F, fn): the statement on the vertices of frontier F only
    // (dsl/vertexmap.h:2190-2230), as its own pass
    template <typename Fn> lazy_executor &vertex_map(frontier &F, Fn fn) {
        flush();
        if (F.isEmpty()) return *this;
        graptor_b200::VmBuilder b;
        expr::NP st = fn(expr::var(expr::NK::VarV)).node();
        if (!b.statement(st)) graptor_b200::unsupported("vertex statement (too long)", st);
        graptor_b200::run_vmap(part_.graph(), b, F.all() ? nullptr : F.bind(part_.graph()), nullptr);
        return *this;
    }
    template <typename Fn> lazy_executor &vertex_scan(Fn fn) { return vertex_map(fn); }
    // vertex_scan(F, fn) (dsl/vertexmap.h:2217-2227): fn on the vertices of F,
    // its scalar reductions summed into their host variables
    template <typename Fn> lazy_executor &vertex_scan(frontier &F, Fn fn) { return vertex_map(F, fn); }
    template <typename G, typename Fn>
    lazy_executor &vertex_filter(const G &GA, frontier &F, frontier &out, Fn fn) {
        flush();
        graptor_b200::VmBuilder b;
        expr::NP c = fn(expr::var(expr::NK::VarV)).node();
        if (!b.value(c) || !b.emit(GG_VM_FILTER)) graptor_b200::unsupported("vertex filter", c);
        gg_frontier *fin = F.all() ? nullptr : F.bind(GA.handle());
        graptor_b200::run_vmap(GA.handle(), b, fin, out.output(GA.handle()));
        return *this;
    }
    // an edgemap step queued by api::edgemap
    lazy_executor &edge_step(std::function<void()> step) {
        flush();
        step();
        return *this;
    }
    void materialize() { flush(); }

private:
    void flush() {
        if (stmts_.empty()) return;
        graptor_b200::VmBuilder b;
        for (size_t i = 0; i < stmts_.size();) {
            if (b.statement(stmts_[i])) {
                ++i;
                continue;
            }
            if (b.d.ncode == 0) graptor_b200::unsupported("vertex statement (too long)", stmts_[i]);
            graptor_b200::run_vmap(part_.graph(), b, nullptr, nullptr);
            b = graptor_b200::VmBuilder();
        }
        if (b.d.ncode) graptor_b200::run_vmap(part_.graph(), b, nullptr, nullptr);
        stmts_.clear();
    }
    partitioner part_;
    std::vector<expr::NP> stmts_;
};

inline lazy_executor make_lazy_executor(const partitioner &part) { return lazy_executor(part); }

// maintain_copies(part, output, prev, cur): prev[v] = cur[v] on the output
// frontier (dsl/vertexmap.h:2515-2535)
template <typename P1, typename P2>
void maintain_copies(const partitioner &part, frontier &output, P1 &prev, P2 &cur) {
    graptor_b200::VmBuilder b;
    int s = b.prop_slot(cur.handle()), t = b.prop_slot(prev.handle());
    b.emit(GG_VM_LOAD, s);
    b.emit(GG_VM_STORE, t);
    if (output.isEmpty()) return;
    graptor_b200::run_vmap(part.graph(), b, output.all() ? nullptr : output.bind(part.graph()), nullptr);
}

namespace api {

// ---------------------------------------------------------------------------
// edgemap (api.h:2143-2415)
// ---------------------------------------------------------------------------
struct emap_state {
    gg_emap_desc d;
    frontier *in = nullptr;
    frontier *out = nullptr;
    std::vector<expr::NP> vertexops;
    emap_state() {
        std::memset(&d, 0, sizeof(d));
        d.variant = GG_VAR_AUTO;
    }
};

inline void emap_arg(emap_state &s, const arg_config &c) {
    s.d.threshold = c.threshold;
    s.d.threshold_k = c.k;
    s.d.fusion = c.fusion;
}
inline void emap_arg(emap_state &s, const arg_filter_src &f) {
    s.in = f.F;
    if (f.dst) s.d.dst_filter = GG_FILTER_IN_FRONTIER;
    else s.d.src_strong = f.strong;
}
template <typename Fn> void emap_arg(emap_state &s, const arg_filter_dst<Fn> &f) {
    graptor_b200::lower_dst_filter(f.fn(expr::var(expr::NK::VarDst)).node(), s.d);
}
template <typename Fn> void emap_arg(emap_state &s, const arg_record<Fn> &r) {
    s.out = r.out;
    if constexpr (std::is_same<Fn, no_method>::value) {
        s.d.record = GG_RECORD_REDUCTION;
    } else {
        graptor_b200::lower_record_method(r.fn(expr::var(expr::NK::VarDst)).node(), s.d);
    }
}
template <typename Fn> void emap_arg(emap_state &s, const arg_relax<Fn> &r) {
    graptor_b200::lower_relax(r.fn(expr::var(expr::NK::VarSrc), expr::var(expr::NK::VarDst),
                                    expr::var(expr::NK::VarEdge)).node(),
                               s.d);
}
template <typename Fn> void emap_arg(emap_state &s, const arg_fusion<Fn> &) {
    s.d.fusion = 1;  // the library's async push is always min-label/level safe
}
inline void emap_arg(emap_state &, int) {}  // unsupported config() forms return 0 in the reference

template <typename GraphType, typename... Args>
lazy_executor edgemap(const GraphType &GA, Args &&... args) {
    emap_state s;
    (emap_arg(s, args), ...);
    lazy_executor lz(GA.get_partitioner());
    gg_graph *g = GA.handle();
    lz.edge_step([=]() mutable {
        gg_frontier *fin = (s.in && !s.in->all()) ? s.in->bind(g) : nullptr;
        gg_frontier *fout = s.out ? s.out->output(g) : nullptr;
        if (!fout) s.d.record = GG_RECORD_NONE;
        if (s.d.relax == GG_RELAX_ADD_GATHER) s.d.record = GG_RECORD_NONE;
        if (s.d.record == GG_RECORD_NONE && fout) {
            // a recorded frontier with a gather relax: nothing is activated
            graptor_b200::check(gg_frontier_clear(fout), "gg_frontier_clear");
            fout = nullptr;
        }
        graptor_b200::before_device();
        graptor_b200::check(gg_edgemap(g, &s.d, fin, fout, nullptr), "gg_edgemap");
        ++graptor_b200::device_epoch();
    });
    return lz;
}

}  // namespace api

#endif  // GRAPTOR_B200_API_H
