/*
 * gg.h -- C ABI of the B200 edgemap/vertexmap library (libgg.so).
 *
 * This is the drop-in boundary under Graptor's operator surface.  Graptor is
 * a header-only C++ library whose analytics call
 *     api::edgemap(GA, api::record(...), api::filter(...), api::relax(...))
 *     make_lazy_executor(part).vertex_map(...).vertex_scan(...).materialize()
 * (include/graptor/api.h:2143-2415, include/graptor/dsl/vertexmap.h:2120-2446).
 * The C++ header include/graptor_b200/api.h keeps that surface and lowers each
 * recognised relax/filter/record expression to the descriptors below; the
 * entry points here are what it (or any ctypes/FFI caller) binds.
 *
 * Conventions
 *   - Every function returns gg_status and never aborts; gg_last_error()
 *     gives a message for the calling context.
 *   - Handles are opaque and owned by the caller (explicit *_destroy).
 *     Device memory belongs to the library.
 *   - One CUDA stream per context; calls on one context come from one host
 *     thread at a time (Graptor's own contract: one host thread calls the
 *     library, all parallelism is inside).
 *   - Vertex ids are uint32, edge offsets uint64 (include/graptor/itraits.h:80-85,
 *     VID = unsigned int, EID = size_t).
 */
#ifndef GG_H
#define GG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GG_API __attribute__((visibility("default")))

/* Status codes.  Graptor itself reports failures with assert/abort/exit
 * (include/graptor/dsl/edgemap.h:66-88, graph/GraphCSx.h:2152-2246); the
 * library returns these instead. */
typedef enum gg_status {
    GG_OK = 0,
    GG_ERR_ARG = 1,         /* invalid argument / descriptor */
    GG_ERR_OOM = 2,         /* device or host allocation failed */
    GG_ERR_CUDA = 3,        /* CUDA runtime error (message in gg_last_error) */
    GG_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    GG_ERR_UNSUPPORTED = 5, /* operator combination not lowered */
    GG_ERR_IO = 6,          /* file I/O or format error */
    GG_ERR_STATE = 7,       /* handle in the wrong state / device error flag */
    GG_ERR_NOT_FOUND = 8    /* CUDA device / symbol not available */
} gg_status;

typedef struct gg_ctx gg_ctx;
typedef struct gg_graph gg_graph;
typedef struct gg_prop gg_prop;
typedef struct gg_frontier gg_frontier;

/* Element types of vertex properties (api::vertexprop<T,...>,
 * include/graptor/api/vertexprop.h:30-140, plus the reduced-precision
 * storage formats of PR_vary, bench/PR_vary.C:247-648). */
typedef enum gg_dtype {
    GG_I32 = 0, GG_U32 = 1, GG_F32 = 2, GG_F64 = 3,
    GG_BF16 = 4,       /* bfloat16, round to nearest even */
    GG_F16 = 5,        /* IEEE half, round to nearest even */
    GG_FP8E4M3 = 6,    /* OCP e4m3, with a per-iteration power-of-two scale */
    GG_CFP_6_10 = 7,   /* Graptor customfp<6,10>: truncating, unsigned (customfp.h:21-186) */
    GG_BF16_TRUNC = 8, /* Graptor scustomfp<true,8,7>: bfloat16 by truncation */
    GG_U8 = 9
} gg_dtype;

GG_API const char *gg_status_string(gg_status s);
GG_API size_t gg_dtype_size(gg_dtype t);

/* ------------------------------------------------------------------ */
/* Context                                                            */
/* ------------------------------------------------------------------ */
GG_API gg_status gg_ctx_create(int device, gg_ctx **out);
GG_API gg_status gg_ctx_destroy(gg_ctx *ctx);
/* Use the caller's cudaStream_t for all work of this context (NULL =
 * the library's own stream). */
GG_API gg_status gg_ctx_set_stream(gg_ctx *ctx, void *cuda_stream);
GG_API gg_status gg_ctx_get_stream(gg_ctx *ctx, void **cuda_stream);
GG_API gg_status gg_ctx_sync(gg_ctx *ctx);
GG_API const char *gg_last_error(gg_ctx *ctx);
/* Number of kernels this context has launched so far. */
GG_API uint64_t gg_ctx_launch_count(gg_ctx *ctx);

/* ------------------------------------------------------------------ */
/* Graphs: device CSR (out-edges, push) + CSC (in-edges, pull).       */
/* Replaces GraphCSx / GraphVEBOGraptor (graph/GraphCSx.h:293-2262,   */
/* graph/CGraphVEBOGraptor.h:60-496): no VEBO reordering, no SIMD     */
/* slabs; the CSC aliases the CSR for symmetric graphs.               */
/* ------------------------------------------------------------------ */

/* Upload a host CSR: off has n+1 entries (off[n] == m), adj has m. */
GG_API gg_status gg_graph_upload(gg_ctx *ctx, uint32_t n, uint64_t m, const uint64_t *off,
                                 const uint32_t *adj, int symmetric, gg_graph **out);

/* Graptor version-2/3 binary file (GraphCSx::readFromBinaryFile,
 * graph/GraphCSx.h:2137-2262; writer GraphCSx.h:2009-2026). */
GG_API gg_status gg_graph_read_bin(gg_ctx *ctx, const char *path, int symmetric, gg_graph **out);

/* Ingest with cleaning on the device (the preprocessing the reference does
 * with its tools before loading: tools/CvtToUndir.C, RmDupEdges.C,
 * RmSelfEdges.C): duplicate edges and self-loops are dropped; with
 * GG_INGEST_SYMMETRISE every edge's reverse is added first and the graph is
 * symmetric.  gg_graph_from_edges takes an edge list (host arrays, or device
 * pointers with GG_INGEST_DEVICE); gg_graph_read_bin_clean a Graptor v2/v3
 * .bin file that may hold duplicates, self-loops or one direction only. */
#define GG_INGEST_SYMMETRISE 1
#define GG_INGEST_DEVICE 2
GG_API gg_status gg_graph_from_edges(gg_ctx *ctx, uint32_t n, uint64_t nedges, const uint32_t *src,
                                     const uint32_t *dst, int flags, gg_graph **out);
GG_API gg_status gg_graph_read_bin_clean(gg_ctx *ctx, const char *path, int flags, gg_graph **out);
GG_API gg_status gg_graph_write_bin(gg_graph *g, const char *path);

/* Seeded synthetic graphs built on the device (the workloads' inputs). */
typedef enum gg_gen_kind { GG_GEN_RMAT = 0, GG_GEN_ER = 1, GG_GEN_GRID = 2 } gg_gen_kind;
typedef struct gg_gen_params {
    int kind;            /* gg_gen_kind */
    int scale;           /* RMAT: n = 2^scale */
    uint64_t nedges;     /* RMAT: generated edges before symmetrising */
    double a, b, c;      /* RMAT quadrant probabilities (d = 1-a-b-c) */
    uint32_t n;          /* ER: vertices */
    double avgdeg;       /* ER: average out-degree */
    uint32_t rows, cols; /* GRID */
    uint32_t bp;         /* ER: dangling vertices, GRID: deleted edges (basis points) */
    uint64_t seed;
    int symmetric;       /* RMAT / ER: add reverse edges */
} gg_gen_params;
GG_API gg_status gg_graph_generate(gg_ctx *ctx, const gg_gen_params *p, gg_graph **out);

GG_API gg_status gg_graph_info(gg_graph *g, uint32_t *n, uint64_t *m, int *symmetric);
/* Host copies of the CSR (off: n+1 entries, adj: m entries). */
GG_API gg_status gg_graph_download(gg_graph *g, uint64_t *off, uint32_t *adj);
/* Device pointers of the CSR/CSC (valid until gg_graph_destroy). */
GG_API gg_status gg_graph_device_ptrs(gg_graph *g, const uint64_t **off, const uint32_t **adj,
                                      const uint64_t **in_off, const uint32_t **in_adj);
GG_API gg_status gg_graph_max_degree_vertex(gg_graph *g, uint32_t *v, uint32_t *deg);
GG_API gg_status gg_graph_destroy(gg_graph *g);

/* ------------------------------------------------------------------ */
/* Vertex properties (api::vertexprop, api/vertexprop.h:30-140).      */
/* ------------------------------------------------------------------ */
GG_API gg_status gg_prop_create(gg_graph *g, gg_dtype t, gg_prop **out);
GG_API gg_status gg_prop_fill(gg_prop *p, const void *value);             /* vertexprop::fill */
GG_API gg_status gg_prop_set(gg_prop *p, uint32_t v, const void *value);  /* vertexprop::set */
GG_API gg_status gg_prop_get(gg_prop *p, uint32_t v, void *value);        /* operator[](VID) */
GG_API gg_status gg_prop_download(gg_prop *p, void *host);
GG_API gg_status gg_prop_upload(gg_prop *p, const void *host);
GG_API gg_status gg_prop_device_ptr(gg_prop *p, void **dptr);
GG_API gg_status gg_prop_destroy(gg_prop *p);                             /* vertexprop::del */
/* A property whose storage is CUDA managed memory: gg_prop_device_ptr returns
 * an address that host code may also read and write (between library calls,
 * after gg_ctx_sync).  Replaces mmap_ptr<T>::allocate(numa_allocation_partitioned)
 * (mm.h:741-745), whose arrays the reference's analytics index from host code. */
GG_API gg_status gg_prop_create_managed(gg_graph *g, gg_dtype t, gg_prop **out);
/* Moves a managed property's pages to the device (to_device = 1) or to the
 * host (0) ahead of use, in order on the context's stream (one bulk
 * migration instead of page faults); 2 marks a property that is no longer
 * written read-mostly (host and device each keep a copy of the pages they
 * read) and prefetches it to the device.  A no-op for other properties. */
GG_API gg_status gg_prop_prefetch(gg_prop *p, int to_device);

/* ------------------------------------------------------------------ */
/* Frontiers (frontier/frontier.h:58-716).  A frontier holds a        */
/* vertex list (degree-binned), a bitmap, or "all vertices", plus the */
/* device-resident counts nactv (vertices) and nacte (sum of their    */
/* out-degrees) that drive the sparse/dense switch.                   */
/* ------------------------------------------------------------------ */
GG_API gg_status gg_frontier_create(gg_graph *g, gg_frontier **out);
GG_API gg_status gg_frontier_clear(gg_frontier *f);                    /* empty */
GG_API gg_status gg_frontier_set_single(gg_frontier *f, uint32_t v);   /* frontier::create(n,v,deg) */
GG_API gg_status gg_frontier_set_all(gg_frontier *f);                  /* frontier::all_true(n,m) */
GG_API gg_status gg_frontier_set_list(gg_frontier *f, const uint32_t *host_list, uint64_t k);
GG_API gg_status gg_frontier_counts(gg_frontier *f, uint64_t *nactv, uint64_t *nacte);
/* Active vertices, ascending, into host memory (cap entries). */
GG_API gg_status gg_frontier_download(gg_frontier *f, uint32_t *host_list, uint64_t cap,
                                      uint64_t *k);
GG_API gg_status gg_frontier_destroy(gg_frontier *f);

/* ------------------------------------------------------------------ */
/* edgemap (api::edgemap, api.h:2143-2415)                            */
/* ------------------------------------------------------------------ */

/* relax(s,d,e) expressions on the path (the AST -> descriptor lowering). */
typedef enum gg_relax_kind {
    GG_RELAX_MIN_PLUS1_I32 = 0, /* a[d].min(a[s] + _1) on int32      (BFSLVLv.C:209-215) */
    GG_RELAX_MIN_U32 = 1,       /* a[d].min(a[s]) on uint32          (CCv.C:575-581)     */
    GG_RELAX_SETIF_U32 = 2,     /* a[d].setif(s): a[d] = s once      (BFSv.C:144-146)    */
    GG_RELAX_ADD_GATHER = 3,    /* y[d] += cast(contrib[s])          (PRv.C:202-212)     */
    /* checks: record d when the condition holds for an active in-neighbour
     * s; nothing is written (the analytics' validation edgemaps) */
    GG_RELAX_NE_CHECK = 4,      /* a[d] != a[s] on uint32            (CCv.C:612-617)     */
    GG_RELAX_GAP_CHECK = 5,     /* a[s] > a[d] + 1 || a[s] < a[d] - 1 on int32
                                                                      (BFSLVLv.C:288-294) */
    GG_RELAX_AHEAD_CHECK = 6,   /* a[s] < a[d] - 1 on int32          (BFSLVLv.C:299-305) */
    GG_RELAX_OR_U32 = 7,        /* a[d] |= src[s] on uint32 (another property as source;
                                   FMv.C:356-358, its neighbourhood bit masks)          */
    GG_RELAX_MIS_U8 = 8,        /* maximal independent set states on uint8, 0 undecided,
                                   1 conditionally in, 2 out, 3 in: over the in-edges
                                   (s, d), s != d, d becomes out when some s is in, else
                                   undecided when it is conditionally in and some s < d
                                   is undecided or conditionally in (MISv.C:235-255,
                                   dsl/ast/dfsaop.h:49-230).  Takes dst filter NONE or
                                   IN_FRONTIER and record NONE or EQ_ZERO. */
    GG_RELAX_COUNT_DOWN_U32 = 9 /* a[d].count_down_value(_c(k)) on uint32: every active
                                   in-neighbour s takes one off a[d] while a[d] > k, never
                                   below the floor k (KC_bucket.C:343-380, the k-core
                                   peel).  Takes dst filter GT_CONST with k (the floor)
                                   and record NONE, REDUCTION (every vertex counted down)
                                   or AT_FLOOR.  Counts must stay below 2^31. */
} gg_relax_kind;

/* dst filters (api::filter(weak, dst, lambda), api.h:687-706). */
typedef enum gg_filter_kind {
    GG_FILTER_NONE = 0,
    GG_FILTER_GT_CONST = 1, /* a[d] > _c(k)       (BFSLVLv.C:190-194) */
    GG_FILTER_NE_ZERO = 2,  /* a[d] != zero_val   (CCv.C:566-570)     */
    GG_FILTER_MSB_SET = 3,  /* msbset(a[d])       (BFSv.C:139-142)    */
    GG_FILTER_NE_CONST = 4, /* a[d] != _c(k)      (FMv.C:353-354, k = _1s: all ones) */
    GG_FILTER_IN_FRONTIER = 5 /* d in the input frontier, every source active
                                 (api::filter(F, dst, strong), MISv.C:254)      */
} gg_filter_kind;

/* record (api::record, api.h:1450-1516). */
typedef enum gg_record_kind {
    GG_RECORD_NONE = 0,      /* no output frontier (PRv) */
    GG_RECORD_REDUCTION = 1, /* vertices whose relax returned true */
    GG_RECORD_NE_PREV = 2,   /* method a[d] != prev[d]; prev[d] = a[d] afterwards
                                (record(..., λd: a[d]!=prev[d]) + maintain_copies) */
    GG_RECORD_EQ_ZERO = 3,   /* method a[d] == 0 after the step (MISv.C:246-253) */
    GG_RECORD_AT_FLOOR = 4   /* COUNT_DOWN: the vertices whose count reached the floor k
                                in this step, each once (the fused k-core step's
                                old == k + 1 test, KC_bucket.C:353-369) */
} gg_record_kind;

/* sparse/dense threshold (api.h:130-222) and the learned selector. */
typedef enum gg_threshold_kind {
    GG_THRESH_DEFAULT = 0, /* sparse iff nactv+nacte <= m/20           */
    GG_THRESH_FRAC = 1,    /* sparse iff nactv+nacte <= m*k/100          */
    GG_THRESH_ALWAYS_SPARSE = 2,
    GG_THRESH_ALWAYS_DENSE = 3,
    GG_THRESH_LEARNED = 4  /* on-device MLP picks the variant; threshold is its fallback */
} gg_threshold_kind;

/* Traversal variants. */
typedef enum gg_variant {
    GG_VAR_AUTO = -1,
    GG_VAR_PUSH_SPARSE = 0, /* degree-binned thread/warp/CTA push over the frontier list */
    GG_VAR_PUSH_MERGE = 1,  /* edge-balanced (merge-path) push over the frontier list   */
    GG_VAR_PULL_DENSE = 2,  /* bitmap-frontier pull over the CSC with early exit         */
    GG_VAR_PUSH_DENSE = 3,  /* push from a bitmap frontier, dense bitmap output          */
    GG_VAR_HOOK = 4         /* CC only, reported in run stats: the rest of the run
                               finished by min-id hooking (road-like graphs, see gg_cc) */
} gg_variant;

typedef struct gg_emap_desc {
    int relax;              /* gg_relax_kind */
    gg_prop *a;             /* relaxed property a[d] (level / label / parent / y) */
    gg_prop *src;           /* ADD_GATHER: contrib[s] (may be reduced precision); OR_U32: src[s] */
    float src_scale;        /* ADD_GATHER: multiply gathered values by this (FP8 scale) */
    int accum_f64;          /* ADD_GATHER: accumulate in double (PRv) instead of float */
    int dst_filter;         /* gg_filter_kind */
    gg_prop *dst_filter_prop;
    int64_t dst_filter_k;   /* GT_CONST / NE_CONST constant */
    int src_strong;         /* api::strong src filter (0 = weak) */
    int record;             /* gg_record_kind */
    gg_prop *prev;          /* NE_PREV: previous copy of a */
    int threshold;          /* gg_threshold_kind */
    int threshold_k;        /* FRAC percentage */
    int variant;            /* gg_variant override (GG_VAR_AUTO = threshold decides) */
    int fusion;             /* api::fusion present: multi-hop push allowed */
    int src_level_sync;     /* MIN_PLUS1 with GT_CONST filter k: every active source
                               holds a[s] == k-1 (level-synchronous BFS), so the
                               relax offers k without loading a[s]; every vertex
                               passing the filter is unvisited and holds the same
                               value in a and prev (BFSLVLv.C:117-129 sets both
                               to n+1), so a step records the first writer of
                               each such vertex and prev is neither read nor
                               written */
} gg_emap_desc;

typedef struct gg_emap_stats {
    int variant;        /* variant that ran */
    uint64_t nactv_in;  /* F_i */
    uint64_t nacte_in;  /* E_i */
    uint64_t scanned;   /* S_i (edges examined) when counted, else 0 */
    uint64_t nactv_out; /* N_i */
    uint64_t nacte_out;
    double kernel_ms;   /* device time of the traversal kernel (CUDA events) */
} gg_emap_stats;

/* One edgemap step.  in may be NULL (all vertices active: no src filter).
 * out may be NULL when record == GG_RECORD_NONE.  stats may be NULL; when
 * non-NULL the call synchronises to fill it. */
GG_API gg_status gg_edgemap(gg_graph *g, const gg_emap_desc *d, gg_frontier *in,
                            gg_frontier *out, gg_emap_stats *stats);

/* ------------------------------------------------------------------ */
/* vertexmap / vertex_scan / vertex_filter (dsl/vertexmap.h:2120-2446) */
/* A fused pass over all vertices (or a frontier) executing a short    */
/* program of per-vertex statements; the lazy executor's merging of   */
/* consecutive maps and scans into one pass becomes one kernel.        */
/* ------------------------------------------------------------------ */
#define GG_VM_MAX_CODE 64
#define GG_VM_MAX_PROPS 8
#define GG_VM_MAX_CONSTS 8
#define GG_VM_MAX_REDUCE 4
#define GG_VM_MAX_TMP 4

/* Stack-machine opcodes.  Operands are double on the stack; property
 * loads/stores convert from/to the property's dtype. */
typedef enum gg_vm_op {
    GG_VM_END = 0,
    GG_VM_LOAD = 1,     /* push props[arg][v] */
    GG_VM_STORE = 2,    /* props[arg][v] = pop */
    GG_VM_CONST = 3,    /* push consts[arg] */
    GG_VM_VID = 4,      /* push v */
    GG_VM_DEGREE = 5,   /* push out-degree(v) */
    GG_VM_ADD = 6, GG_VM_SUB = 7, GG_VM_MUL = 8, GG_VM_DIV = 9,
    GG_VM_ABS = 10, GG_VM_MIN = 11, GG_VM_MAX = 12,
    GG_VM_EQ = 13, GG_VM_NE = 14, GG_VM_LT = 15, GG_VM_GT = 16,
    GG_VM_REDUCE_ADD = 17, /* reduce[arg] += pop (double accumulation) */
    GG_VM_TOF32 = 18,      /* round top of stack to float */
    GG_VM_SELECT = 19,     /* c ? x : y  (pops y, x, c) */
    GG_VM_FILTER = 20,     /* pop; if non-zero add v to the output frontier */
    GG_VM_DUP = 21,
    /* uint32 bit operations on the operands taken modulo 2^32 (FMv.C:370-392) */
    GG_VM_AND = 22, GG_VM_OR = 23, GG_VM_XOR = 24, GG_VM_NOT = 25,
    GG_VM_TOU32 = 26,      /* top of stack modulo 2^32 (unsigned arithmetic) */
    GG_VM_TSET = 27,       /* tmp[arg] = pop (expr::let bindings, GG_VM_MAX_TMP of them) */
    GG_VM_TGET = 28,       /* push tmp[arg] */
    GG_VM_LE = 29, GG_VM_GE = 30
} gg_vm_op;

typedef struct gg_vmap_desc {
    int ncode;
    uint8_t code[GG_VM_MAX_CODE];
    uint8_t arg[GG_VM_MAX_CODE];
    gg_prop *props[GG_VM_MAX_PROPS];
    double consts[GG_VM_MAX_CONSTS];
    int nreduce;
} gg_vmap_desc;

/* Runs the program for every vertex (filter == NULL) or every vertex of
 * filter.  reduce_out (nreduce doubles) receives the scan results;
 * out (may be NULL) receives the vertices a FILTER statement selected. */
GG_API gg_status gg_vertexmap(gg_graph *g, const gg_vmap_desc *d, gg_frontier *filter,
                              gg_frontier *out, double *reduce_out);

/* ------------------------------------------------------------------ */
/* Whole analytics on the device (the loops of bench/BFSLVLv.C,        */
/* BFSv.C, CCv.C, PRv.C, PR_vary.C), for FFI callers.  Results go to    */
/* device properties; host arrays may be NULL.                          */
/* ------------------------------------------------------------------ */
#define GG_MAX_ITERS 256
typedef struct gg_run_stats {
    int iterations;
    double total_ms;                  /* device time of the run (CUDA events) */
    uint64_t kernels;                 /* kernels launched */
    uint64_t scanned_edges;           /* sum of S_i */
    uint64_t vertices_reached;        /* sum of |F_i| over the input frontiers */
    uint64_t edges_reached;           /* sum of out-degrees over them (BFS: m_c) */
    int variant[GG_MAX_ITERS];        /* per iteration (-itimes) */
    uint64_t nactv[GG_MAX_ITERS];
    uint64_t nacte[GG_MAX_ITERS];
    uint64_t scanned[GG_MAX_ITERS];
    double delta[GG_MAX_ITERS];       /* PageRank L1 residual per iteration */
    double iter_ms[GG_MAX_ITERS];     /* the iteration's device time (collect_stats; graph- and device-driven
                                         runs: from its start to the next one's, launch gaps included) */
    double kernel_ms[GG_MAX_ITERS];   /* its traversal kernel's own span (first CTA start to last CTA end;
                                         = iter_ms where the step is not a separate kernel) */
} gg_run_stats;

typedef struct gg_run_opts {
    int threshold;      /* gg_threshold_kind */
    int threshold_k;
    int variant;        /* fixed variant (GG_VAR_AUTO: threshold / selector) */
    int collect_stats;  /* record per-iteration counts (forces a sync per iteration) */
} gg_run_opts;

/* BFS levels (BFSLVLv): level[root] = 0, unreached = n+1. */
GG_API gg_status gg_bfs_level(gg_graph *g, uint32_t root, const gg_run_opts *o, gg_prop *level,
                              int32_t *host_level, gg_run_stats *st);

/* BFS levels of one root delivered to host memory with the copy running
 * behind the caller's next call (the reference's BFSLVLv leaves its level
 * array in host memory, BFSLVLv.C:110-254; a GPU run pays a device-to-host
 * copy for it).  The call runs the BFS into one of two library-owned level
 * buffers, starts the copy of the levels into host_level (n entries) on the
 * graph's copy stream, and returns when the BFS is done and the copy started
 * by the PREVIOUS call on this graph has landed in its host_level.
 * gg_bfs_level_host_wait(g) waits for the last copy.  The caller may read
 * the host_level of call i once call i+1 (or the wait) has returned, and must
 * not reuse it before then.  host_level should be page-locked memory
 * (cudaHostAlloc / cudaHostRegister): a pageable destination makes each copy
 * synchronous.  Calls on one graph come from one host thread. */
GG_API gg_status gg_bfs_level_host_async(gg_graph *g, uint32_t root, const gg_run_opts *o,
                                         int32_t *host_level, gg_run_stats *st);
GG_API gg_status gg_bfs_level_host_wait(gg_graph *g);
/* BFS parents (BFSv): parent[root] = root, unreached = ~0u; any valid BFS tree. */
GG_API gg_status gg_bfs_parent(gg_graph *g, uint32_t root, const gg_run_opts *o, gg_prop *parent,
                               uint32_t *host_parent, gg_run_stats *st);
/* Connected components (CCv): label = minimum vertex id of the component.
 * Device-driven runs of a symmetric graph take CCv's road-network test after
 * the first step (PUSH_ZERO, bench/CCv.C:365-388: fewer than n/10 vertices
 * labelled 0) and, where it holds, finish the run by hooking every edge's
 * endpoints' roots, the larger under the smaller (labels unchanged: the
 * minimum id of each component); otherwise label propagation continues. */
GG_API gg_status gg_cc(gg_graph *g, const gg_run_opts *o, gg_prop *label, uint32_t *host_label,
                       gg_run_stats *st);
/* k-core decomposition (KC_bucket, bench/KC_bucket.C:107-420): coreness[v] =
 * the largest k such that v lies in a subgraph whose every vertex has at
 * least k neighbours in it (0 for isolated vertices).  The peel: the count
 * of every vertex starts at its degree; for floors k = 0, 1, 2, ... the
 * vertices whose count is k are removed and count down their neighbours
 * (edgemap with GG_RELAX_COUNT_DOWN_U32, floor k, record AT_FLOOR) until no
 * count reaches k; empty floors are skipped.  o NULL: every step a sparse
 * push (a count-down pull has no early exit).  Symmetric graphs only
 * (GG_ERR_UNSUPPORTED otherwise).  coreness: a U32 property of g, or NULL;
 * host_coreness: n entries of host memory, or NULL; largest_core: the
 * largest coreness, or NULL.  st: floors, peel steps and device time. */
GG_API gg_status gg_kcore(gg_graph *g, const gg_run_opts *o, gg_prop *coreness, uint32_t *host_coreness,
                          uint32_t *largest_core, gg_run_stats *st);

typedef struct gg_pr_params {
    int maxiter;        /* PRv -pr:maxiter (default 100) */
    double tol;         /* stop when L1 residual <= tol (PRv: 1e-7) */
    float damping;      /* 0.85 */
    int contrib_dtype;  /* gg_dtype of the stored contribution: F32, BF16, F16, FP8E4M3, CFP_6_10, BF16_TRUNC,
                           or F64 (PR_vary's FP64 variant: ranks, sums and contributions all double, x an
                           F64 property, damping taken as the shortest decimal of the float) */
    int accum_f64;      /* accumulate gathers in double (PRv) rather than float */
    int renorm_f32;     /* PRv renormalises by float(1)/float(s); PR_vary by double */
    /* Staged precision (PR_vary.C:652-757): nstages 2..4 runs stage k with
     * stage_dtype[k] contributions (not F64) and stage_accum_f64[k] sums
     * until the L1 residual <= stage_tol[k], the last stage until tol; the
     * switch is taken on the device and the next stage's contributions are
     * re-encoded from the ranks.  VARIANT 4620 = {CFP_6_10, float sums, 1e-3},
     * {F32, double sums}.  nstages 0 or 1: contrib_dtype / accum_f64 only. */
    int nstages;
    int stage_dtype[4];
    int stage_accum_f64[4];
    double stage_tol[4];
    /* BF16 contributions only (no reference counterpart): stochastic = 1
     * rounds each stored contribution up or down at random, with probability
     * by its distance to the two neighbouring bfloat16 values (16 random bits
     * per vertex and iteration from a counter hash, MurmurHash3's fmix32, so
     * runs repeat exactly); average_last = K > 0 returns the mean of the
     * ranks of iterations maxiter-K .. maxiter-1 (of those run).  Rounding
     * to nearest leaves a bias that the iteration amplifies; unbiased
     * rounding leaves noise that the average removes. */
    int stochastic;
    int average_last;
} gg_pr_params;
/* PageRank power iteration (PRv / PR_vary run_prec); x receives the ranks. */
GG_API gg_status gg_pagerank(gg_graph *g, const gg_pr_params *p, gg_prop *x, float *host_x,
                             gg_run_stats *st);

/* ------------------------------------------------------------------ */
/* BFS levels without allocation.  This entry point has no counterpart */
/* in the reference.  It is for callers that cannot let a library call */
/* cudaMalloc (a fixed device-memory budget owned by the caller's own  */
/* pool, pipelines that must avoid the implicit device synchronisation */
/* of cudaMalloc/cudaFree, hosts that forbid allocation by plug-ins).  */
/* No context is needed and nothing is allocated: the caller passes    */
/* the device CSR (d_off: n+1 entries, d_adj: d_off[n] entries) and    */
/* the device output d_level (n entries: level of every vertex, root 0,*/
/* unreached n+1, as gg_bfs_level).  Work runs on cuda_stream (NULL =  */
/* the legacy default stream) of the current device.                   */
/*   - n must not exceed GG_NOALLOC_MAX_VERTICES; larger graphs return */
/*     GG_ERR_ARG with a message in err (may be NULL) and launch       */
/*     nothing.                                                        */
/*   - The frontier queues live in one fixed __device__ array of about */
/*     8 MiB that every GPU loading the library keeps until exit.      */
/*     Every call on a device shares it and each call clears what must */
/*     start at zero; calls that overlap on the GPU (other streams or  */
/*     host threads) race on it, so the caller must serialise them.    */
/*   - Every call looks up the array's device address in the current   */
/*     context (cudaGetSymbolAddress), so the address stays right after*/
/*     cudaDeviceReset or under a second context on the same device.  */
/*     The first call on a device also loads the module there; make    */
/*     that first call before any stream capture begins.               */
/*   - An adjacency entry >= n is skipped and reported: GG_ERR_ARG.    */
/*   - The call synchronises cuda_stream once per BFS level.           */
/* ------------------------------------------------------------------ */
#define GG_NOALLOC_MAX_VERTICES (1u << 20)
GG_API gg_status gg_bfs_level_noalloc(const uint64_t *d_off, const uint32_t *d_adj, uint32_t n,
                                      uint32_t root, int32_t *d_level, void *cuda_stream,
                                      int *iterations, char *err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* GG_H */
