/*
 * oracle.c -- CPU restatement of the reference's edgemap/vertexmap analytics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library (graptor_b200/csrc).  Only the test suite, the smoke check and the
 * CPU-baseline leg of the benchmark load it; the GPU library never links it,
 * and no product code path falls back to it.
 *
 * Parity pinning: the restatement is cross-checked in the test suite against
 * the reference's own build (oracle/Makefile compiles the reference analytics
 * from their sources into oracle/_ref/), run on the same seeded graphs, and
 * against committed golden fixtures (tests/golden/) made by that build.
 *
 * Contents
 *   - seeded graph generators (R-MAT, Erdos-Renyi, 2-D grid) and the CSR
 *     normalisation the workloads prescribe (symmetrise, drop self-loops,
 *     deduplicate); the same generator is implemented on the GPU by the
 *     library and both must agree bit for bit;
 *   - Graptor version-2 binary graph file I/O
 *     (reference: include/graptor/graph/GraphCSx.h:2009-2026 writer,
 *      GraphCSx.h:2137-2262 reader);
 *   - BFS levels       (reference: bench/BFSLVLv.C:110-254, unreached = n+1);
 *   - BFS parent check (reference: bench/BFSv.C:88-232);
 *   - connected-component labels by min-label propagation
 *     (reference: bench/CCv.C:521-588; canonical output = minimum vertex id of
 *      the component, CCv.C:122-169 / 591-601);
 *   - PageRank power iteration, FP32 storage / FP64 sums
 *     (reference: bench/PRv.C:115-290), and a float64 version;
 *   - Graptor's truncating customfp<E,M> conversions
 *     (reference: include/graptor/customfp.h:97-166).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Counter-based hashing: SplitMix64 finaliser (Steele, Lea, Flood,   */
/* "Fast splittable pseudorandom number generators", OOPSLA 2014).    */
/* ------------------------------------------------------------------ */
static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Stream key for (seed, stream id): the generators draw from independent
 * streams so that edge i at level l always gets the same number. */
static inline uint64_t stream_base(uint64_t seed, uint64_t stream) {
    return mix64(seed ^ mix64(stream + 0x51ED270B27A8C3F1ull));
}

/* Probability -> 32-bit threshold, rounded to nearest. */
static inline uint64_t prob_u32(double p) {
    double t = p * 4294967296.0;
    if (t < 0) t = 0;
    if (t > 4294967296.0) t = 4294967296.0;
    return (uint64_t)(t + 0.5);
}

/* ------------------------------------------------------------------ */
/* Edge list -> CSR normalisation                                      */
/* ------------------------------------------------------------------ */

/* Build CSR from packed (src<<32|dst) keys: drop self-loops and
 * duplicates, rows sorted ascending.  Counting sort on src, then an
 * in-row sort.  Consumes keys (freed). */
static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

static void sort_u32(uint32_t *a, uint64_t k) {
    if (k < 2) return;
    if (k <= 32) { /* insertion sort for short rows */
        for (uint64_t i = 1; i < k; ++i) {
            uint32_t v = a[i];
            uint64_t j = i;
            while (j > 0 && a[j - 1] > v) { a[j] = a[j - 1]; --j; }
            a[j] = v;
        }
        return;
    }
    qsort(a, k, sizeof(uint32_t), cmp_u32);
}

static int keys_to_csr(uint32_t n, uint64_t nkeys, uint64_t *keys,
                       uint64_t **off_out, uint32_t **adj_out, uint64_t *m_out) {
    uint64_t *cnt = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    if (!cnt) return -1;
    for (uint64_t i = 0; i < nkeys; ++i) {
        uint32_t s = (uint32_t)(keys[i] >> 32), d = (uint32_t)keys[i];
        if (s != d) cnt[s + 1]++;
    }
    for (uint32_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
    uint64_t tot = cnt[n];
    uint32_t *tmp = (uint32_t *)malloc((tot ? tot : 1) * sizeof(uint32_t));
    uint64_t *pos = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    if (!tmp || !pos) { free(cnt); free(tmp); free(pos); return -1; }
    memcpy(pos, cnt, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < nkeys; ++i) {
        uint32_t s = (uint32_t)(keys[i] >> 32), d = (uint32_t)keys[i];
        if (s != d) tmp[pos[s]++] = d;
    }
    free(keys);
    free(pos);
    /* sort + dedup each row, compacting in place */
    uint64_t *off = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    if (!off) { free(cnt); free(tmp); return -1; }
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
        uint32_t *row = tmp + cnt[v];
        uint64_t k = cnt[v + 1] - cnt[v];
        sort_u32(row, k);
        uint64_t u = 0;
        for (uint64_t i = 0; i < k; ++i)
            if (u == 0 || row[u - 1] != row[i]) row[u++] = row[i];
        off[v + 1] = u; /* unique count, temporarily */
    }
    off[0] = 0;
    for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
    uint64_t m = off[n];
    uint32_t *adj = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!adj) { free(cnt); free(tmp); free(off); return -1; }
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)n; ++v)
        memcpy(adj + off[v], tmp + cnt[v], (off[v + 1] - off[v]) * sizeof(uint32_t));
    free(tmp);
    free(cnt);
    *off_out = off;
    *adj_out = adj;
    *m_out = m;
    return 0;
}

ORC_API void orc_free(void *p) { free(p); }

/* R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004).  Edge i, level l uses the
 * 32-bit draw u = mix64(base + i*64 + l) >> 32 and picks quadrant
 * a (u < Ta), b (u < Tb), c (u < Tc) else d, with T* the rounded cumulative
 * probabilities.  Quadrant b sets the destination bit, c the source bit,
 * d both; level 0 decides the most significant bit.  symmetric != 0 adds
 * the reverse of every edge.  Self-loops and duplicates are removed. */
ORC_API int orc_gen_rmat(int scale, uint64_t nedges, double a, double b, double c,
                         uint64_t seed, int symmetric, uint32_t *n_out,
                         uint64_t *m_out, uint64_t **off_out, uint32_t **adj_out) {
    if (scale < 1 || scale > 31) return -1;
    uint32_t n = 1u << scale;
    uint64_t ta = prob_u32(a), tb = prob_u32(a + b), tc = prob_u32(a + b + c);
    uint64_t base = stream_base(seed, 1);
    uint64_t nk = symmetric ? 2 * nedges : nedges;
    uint64_t *keys = (uint64_t *)malloc((nk ? nk : 1) * sizeof(uint64_t));
    if (!keys) return -1;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)nedges; ++i) {
        uint32_t s = 0, d = 0;
        for (int l = 0; l < scale; ++l) {
            uint64_t u = mix64(base + (uint64_t)i * 64 + (uint64_t)l) >> 32;
            uint32_t sb = (u >= tb) ? 1u : 0u;
            uint32_t db = ((u >= ta && u < tb) || u >= tc) ? 1u : 0u;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        keys[i] = ((uint64_t)s << 32) | d;
        if (symmetric) keys[nedges + i] = ((uint64_t)d << 32) | s;
    }
    *n_out = n;
    return keys_to_csr(n, nk, keys, off_out, adj_out, m_out);
}

/* Erdos-Renyi style G(n, M): M = n*avgdeg/2 (symmetric) or n*avgdeg
 * (directed) uniform pairs, src = hi32(h1)*n>>32, dst likewise from h2.
 * Vertices with mix64(dbase + v) % 10000 < dangling_bp (basis points) lose
 * their out-edges (directed graphs only: they become dangling). */
ORC_API int orc_gen_er(uint32_t n, double avgdeg, uint32_t dangling_bp, uint64_t seed,
                       int symmetric, uint32_t *n_out, uint64_t *m_out,
                       uint64_t **off_out, uint32_t **adj_out) {
    uint64_t M = (uint64_t)((double)n * avgdeg / (symmetric ? 2.0 : 1.0) + 0.5);
    uint64_t base = stream_base(seed, 2), dbase = stream_base(seed, 3);
    uint64_t nk = symmetric ? 2 * M : M;
    uint64_t *keys = (uint64_t *)malloc((nk ? nk : 1) * sizeof(uint64_t));
    if (!keys) return -1;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)M; ++i) {
        uint64_t h1 = mix64(base + 2 * (uint64_t)i), h2 = mix64(base + 2 * (uint64_t)i + 1);
        uint32_t s = (uint32_t)(((h1 >> 32) * (uint64_t)n) >> 32);
        uint32_t d = (uint32_t)(((h2 >> 32) * (uint64_t)n) >> 32);
        if (!symmetric && dangling_bp && (mix64(dbase + s) % 10000) < dangling_bp)
            d = s; /* becomes a self-loop, dropped below */
        keys[i] = ((uint64_t)s << 32) | d;
        if (symmetric) keys[M + i] = ((uint64_t)d << 32) | s;
    }
    *n_out = n;
    return keys_to_csr(n, nk, keys, off_out, adj_out, m_out);
}

/* 2-D grid, rows x cols, 4-neighbour, symmetric.  The undirected edge
 * {u, u+1} (horizontal) or {u, u+cols} (vertical) is deleted when
 * mix64(base + 2u + dir) % 10000 < del_bp. */
ORC_API int orc_gen_grid(uint32_t rows, uint32_t cols, uint32_t del_bp, uint64_t seed,
                         uint32_t *n_out, uint64_t *m_out, uint64_t **off_out,
                         uint32_t **adj_out) {
    uint64_t n64 = (uint64_t)rows * cols;
    if (n64 == 0 || n64 > 0xFFFFFFFFull) return -1;
    uint32_t n = (uint32_t)n64;
    uint64_t base = stream_base(seed, 4);
    uint64_t *keys = (uint64_t *)malloc(4 * n64 * sizeof(uint64_t));
    if (!keys) return -1;
    uint64_t nk = 0;
    for (uint64_t u = 0; u < n64; ++u) {
        uint32_t r = (uint32_t)(u / cols), c = (uint32_t)(u % cols);
        if (c + 1 < cols && (mix64(base + 2 * u) % 10000) >= del_bp) {
            keys[nk++] = (u << 32) | (u + 1);
            keys[nk++] = ((u + 1) << 32) | u;
        }
        if (r + 1 < rows && (mix64(base + 2 * u + 1) % 10000) >= del_bp) {
            keys[nk++] = (u << 32) | (u + cols);
            keys[nk++] = ((u + cols) << 32) | u;
        }
    }
    *n_out = n;
    return keys_to_csr(n, nk, keys, off_out, adj_out, m_out);
}

/* Transpose (CSR -> CSC), rows sorted. */
ORC_API int orc_transpose(uint32_t n, const uint64_t *off, const uint32_t *adj,
                          uint64_t **toff_out, uint32_t **tadj_out) {
    uint64_t m = off[n];
    uint64_t *toff = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *tadj = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    uint64_t *pos = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    if (!toff || !tadj || !pos) { free(toff); free(tadj); free(pos); return -1; }
    for (uint64_t e = 0; e < m; ++e) toff[adj[e] + 1]++;
    for (uint32_t v = 0; v < n; ++v) toff[v + 1] += toff[v];
    memcpy(pos, toff, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint32_t s = 0; s < n; ++s) /* ascending s gives sorted rows */
        for (uint64_t e = off[s]; e < off[s + 1]; ++e) tadj[pos[adj[e]]++] = s;
    free(pos);
    *toff_out = toff;
    *tadj_out = tadj;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Graptor version-2 binary file (GraphCSx.h:2009-2026, 2137-2262):   */
/* u64 header[8] = {2, 1, n, m, sizeof(VID)=4, sizeof(EID)=8, 0, 0},   */
/* then index u64[n] (offset of each row; index[n]=m implied), then   */
/* edges u32[m].  Version 3 additionally stores index[n].             */
/* ------------------------------------------------------------------ */
ORC_API int orc_write_bin(const char *path, uint32_t n, uint64_t m, const uint64_t *off,
                          const uint32_t *adj) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    uint64_t hdr[8] = {2, 1, n, m, 4, 8, 0, 0};
    int ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
             (n == 0 || fwrite(off, sizeof(uint64_t), n, f) == n) &&
             (m == 0 || fwrite(adj, sizeof(uint32_t), m, f) == m);
    ok = (fclose(f) == 0) && ok;
    return ok ? 0 : -1;
}

ORC_API int orc_read_bin(const char *path, uint32_t *n_out, uint64_t *m_out,
                         uint64_t **off_out, uint32_t **adj_out) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    uint64_t hdr[8];
    if (fread(hdr, sizeof(hdr), 1, f) != 1) { fclose(f); return -2; }
    if ((hdr[0] != 2 && hdr[0] != 3) || hdr[4] != 4 || hdr[5] != 8 ||
        hdr[2] > 0xFFFFFFFFull) { fclose(f); return -3; }
    uint32_t n = (uint32_t)hdr[2];
    uint64_t m = hdr[3];
    uint64_t *off = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *adj = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!off || !adj) { free(off); free(adj); fclose(f); return -1; }
    int ok = (n == 0 || fread(off, sizeof(uint64_t), n, f) == n);
    if (ok && hdr[0] == 3) { uint64_t last; ok = fread(&last, 8, 1, f) == 1 && last == m; }
    ok = ok && (m == 0 || fread(adj, sizeof(uint32_t), m, f) == m);
    fclose(f);
    off[n] = m;
    for (uint32_t v = 0; ok && v < n; ++v)
        if (off[v] > off[v + 1]) ok = 0;
    for (uint64_t e = 0; ok && e < m; ++e)
        if (adj[e] >= n) ok = 0;
    if (!ok) { free(off); free(adj); return -4; }
    *n_out = n; *m_out = m; *off_out = off; *adj_out = adj;
    return 0;
}

/* ------------------------------------------------------------------ */
/* BFS levels (BFSLVLv.C:110-254): level[root]=0, level of vertex at   */
/* hop distance k is k, unreached vertices keep n+1 (BFSLVLv.C:117).  */
/* The levels of a fixed root are unique, so a plain queue BFS gives  */
/* the same answer as the reference's asynchronous min-relaxation.    */
/* Returns the number of iterations (BFS depth + 1 frontier rounds).  */
/* ------------------------------------------------------------------ */
ORC_API int orc_bfs_level(uint32_t n, const uint64_t *off, const uint32_t *adj,
                          uint32_t root, int32_t *level) {
    for (uint32_t v = 0; v < n; ++v) level[v] = (int32_t)(n + 1);
    if (root >= n) return -1;
    uint32_t *q = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    if (!q) return -1;
    uint64_t head = 0, tail = 0;
    q[tail++] = root;
    level[root] = 0;
    int depth = 0;
    while (head < tail) {
        uint32_t u = q[head++];
        if (level[u] + 1 > depth) depth = level[u] + 1;
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
            uint32_t v = adj[e];
            if (level[v] == (int32_t)(n + 1)) {
                level[v] = level[u] + 1;
                q[tail++] = v;
            }
        }
    }
    free(q);
    return depth;
}

/* BFS levels with several start vertices at level 0 (a multi-root run of
 * BFSLVLv's level relaxation, BFSLVLv.C:165-216, as on a disjoint union of
 * graphs with one root per part): unreached = n + 1.  Returns the depth. */
ORC_API int orc_bfs_level_multi(uint32_t n, const uint64_t *off, const uint32_t *adj,
                                const uint32_t *roots, uint64_t k, int32_t *level) {
    for (uint32_t v = 0; v < n; ++v) level[v] = (int32_t)(n + 1);
    uint32_t *q = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!q) return -1;
    uint64_t head = 0, tail = 0;
    for (uint64_t i = 0; i < k; ++i) {
        if (roots[i] >= n) { free(q); return -1; }
        if (level[roots[i]] != 0) {
            level[roots[i]] = 0;
            q[tail++] = roots[i];
        }
    }
    int depth = 0;
    while (head < tail) {
        uint32_t u = q[head++];
        if (level[u] + 1 > depth) depth = level[u] + 1;
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
            uint32_t v = adj[e];
            if (level[v] == (int32_t)(n + 1)) {
                level[v] = level[u] + 1;
                q[tail++] = v;
            }
        }
    }
    free(q);
    return depth;
}

/* Sum of out-degrees of reached vertices (= directed edges incident to
 * the reached component of a symmetric graph): the GTEPS numerator. */
ORC_API uint64_t orc_reached_edges(uint32_t n, const uint64_t *off, const int32_t *level) {
    uint64_t s = 0;
    for (uint32_t v = 0; v < n; ++v)
        if (level[v] <= (int32_t)n) s += off[v + 1] - off[v];
    return s;
}

/* Validity of a BFS parent array (BFSv.C:128-148 semantics: unset =
 * ~0u, parent[root]=root).  With exact levels from orc_bfs_level a valid
 * BFS tree has: parent set iff reached; for v != root, the edge
 * parent[v] -> v exists and level[parent[v]] == level[v]-1.
 * Returns the number of violating vertices. */
ORC_API uint64_t orc_check_parents(uint32_t n, const uint64_t *off, const uint32_t *adj,
                                   uint32_t root, const uint32_t *parent,
                                   const int32_t *level) {
    uint64_t bad = 0;
    for (uint32_t v = 0; v < n; ++v) {
        int reached = level[v] <= (int32_t)n;
        uint32_t p = parent[v];
        if (!reached) { bad += (p != 0xFFFFFFFFu); continue; }
        if (v == root) { bad += (p != root); continue; }
        if (p >= n || level[p] != level[v] - 1) { ++bad; continue; }
        /* edge p -> v must exist (rows are sorted: binary search) */
        uint64_t lo = off[p], hi = off[p + 1];
        int found = 0;
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo) / 2;
            if (adj[mid] == v) { found = 1; break; }
            if (adj[mid] < v) lo = mid + 1; else hi = mid;
        }
        bad += !found;
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* Connected components by min-label propagation (CCv.C:521-588):     */
/* label[v] starts at v and relax label[d] = min(label[d], label[s])  */
/* runs along every edge s->d until nothing changes.  On a symmetric  */
/* graph the fixed point is the minimum vertex id of v's component,   */
/* which is exactly the reference's canonical output (CCv.C:122-169). */
/* Worklist version; returns the number of rounds.                    */
/* ------------------------------------------------------------------ */
ORC_API int orc_cc(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t *label) {
    uint8_t *inq = (uint8_t *)calloc(n ? n : 1, 1);
    uint32_t *cur = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t *nxt = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!inq || !cur || !nxt) { free(inq); free(cur); free(nxt); return -1; }
    uint64_t nc = 0;
    for (uint32_t v = 0; v < n; ++v) { label[v] = v; cur[nc++] = v; }
    int rounds = 0;
    while (nc) {
        ++rounds;
        uint64_t nn = 0;
        for (uint64_t i = 0; i < nc; ++i) {
            uint32_t s = cur[i];
            for (uint64_t e = off[s]; e < off[s + 1]; ++e) {
                uint32_t d = adj[e];
                if (label[s] < label[d]) {
                    label[d] = label[s];
                    if (!inq[d]) { inq[d] = 1; nxt[nn++] = d; }
                }
            }
        }
        for (uint64_t i = 0; i < nn; ++i) inq[nxt[i]] = 0;
        uint32_t *t = cur; cur = nxt; nxt = t;
        nc = nn;
    }
    free(inq); free(cur); free(nxt);
    return rounds;
}

/* ------------------------------------------------------------------ */
/* PageRank power iteration (PRv.C:115-290).  in_off/in_adj is the    */
/* CSC (in-edges), outdeg the out-degree.  Per iteration:             */
/*   y[d]   = sum_{s->d} contrib[s]          (sum in double, stored f32)
 *   s      = sum y                          (double)
 *   y     += (1-s)/n                        (double w, stored f32)
 *   s      = sum y                          (double)
 *   w      = 1.0f / (float)s                (FP32, PRv.C:246)
 *   y     *= w
 *   delta  = sum |x - y|                    (double)
 *   x = y; y = 0; contrib = 0.85f * x / (float)outdeg
 * starting from x = 1/n, contrib = 0.85f*x/deg; stop when
 * iter == maxiter or delta <= tol.  Returns the iteration count; the
 * per-iteration delta goes to deltas[] when non-null.                */
/* ------------------------------------------------------------------ */
ORC_API int orc_pr_f32(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj,
                       const uint32_t *outdeg, int maxiter, double tol, float *x,
                       double *deltas) {
    const float damp = 0.85f;
    float *y = (float *)calloc(n ? n : 1, sizeof(float));
    float *contrib = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    if (!y || !contrib) { free(y); free(contrib); return -1; }
    for (uint32_t v = 0; v < n; ++v) {
        x[v] = 1.0f / (float)n;
        contrib[v] = damp * x[v] / (float)outdeg[v];
    }
    int iter = 0;
    double sdelta = 2;
    while (iter < maxiter && sdelta > tol) {
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t d = 0; d < (int64_t)n; ++d) {
            double acc = (double)y[d];
            for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e)
                acc += (double)contrib[in_adj[e]];
            y[d] = (float)acc;
        }
        double s = 0;
        for (uint32_t v = 0; v < n; ++v) s += (double)y[v];
        double w = (1.0 - s) / (double)n;
        s = 0;
        for (uint32_t v = 0; v < n; ++v) {
            y[v] = (float)((double)y[v] + w);
            s += (double)y[v];
        }
        float wf = 1.0f / (float)s;
        sdelta = 0;
        for (uint32_t v = 0; v < n; ++v) {
            y[v] = y[v] * wf;
            sdelta += (double)fabsf(x[v] - y[v]);
            x[v] = y[v];
            y[v] = 0.0f;
            contrib[v] = damp * x[v] / (float)outdeg[v];
        }
        if (deltas) deltas[iter] = sdelta;
        ++iter;
    }
    free(y);
    free(contrib);
    return iter;
}

/* Same iteration carried out entirely in float64: the FP64 oracle that
 * the reduced-precision PageRank runs are measured against (the reference
 * has the same in PR_vary.C:635-648, variant 11). */
ORC_API int orc_pr_f64(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj,
                       const uint32_t *outdeg, int maxiter, double tol, double *x,
                       double *deltas) {
    const double damp = 0.85;
    double *y = (double *)calloc(n ? n : 1, sizeof(double));
    double *contrib = (double *)malloc((size_t)(n ? n : 1) * sizeof(double));
    if (!y || !contrib) { free(y); free(contrib); return -1; }
    for (uint32_t v = 0; v < n; ++v) {
        x[v] = 1.0 / (double)n;
        contrib[v] = damp * x[v] / (double)outdeg[v];
    }
    int iter = 0;
    double sdelta = 2;
    while (iter < maxiter && sdelta > tol) {
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t d = 0; d < (int64_t)n; ++d) {
            double acc = 0;
            for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e) acc += contrib[in_adj[e]];
            y[d] = acc;
        }
        double s = 0;
        for (uint32_t v = 0; v < n; ++v) s += y[v];
        double w = (1.0 - s) / (double)n;
        s = 0;
        for (uint32_t v = 0; v < n; ++v) { y[v] += w; s += y[v]; }
        double wf = 1.0 / s;
        sdelta = 0;
        for (uint32_t v = 0; v < n; ++v) {
            y[v] *= wf;
            sdelta += fabs(x[v] - y[v]);
            x[v] = y[v];
            y[v] = 0;
            contrib[v] = damp * x[v] / (double)outdeg[v];
        }
        if (deltas) deltas[iter] = sdelta;
        ++iter;
    }
    free(y);
    free(contrib);
    return iter;
}

/* ------------------------------------------------------------------ */
/* customfp formats (customfp.h:21-186, class customfp_em<S,E,M,Z,B>) */
/* for the bias-free, no-zero-special-case forms that PR_vary uses:    */
/* customfp<E,M> = customfp_em<false,E,M,false,0> and                  */
/* scustomfp<S,E,M,false,0>.  Encoding keeps the low E bits of the     */
/* float exponent field and the top M mantissa bits by truncation,     */
/* plus the sign when S; decoding sets the missing upper exponent bits */
/* to 0b0111.. (so customfp<6,10> covers exponents 64..127, i.e.       */
/* magnitudes in [2^-63, 2)).  scustomfp<true,8,7> is bfloat16 by      */
/* truncation.                                                         */
/* ------------------------------------------------------------------ */
ORC_API uint32_t orc_cfp_from_float(float f, int S, int E, int M) {
    uint32_t tt;
    memcpy(&tt, &f, 4);
    uint32_t mask = (E + M >= 32) ? 0xFFFFFFFFu : ((1u << (E + M)) - 1u);
    uint32_t t = (tt >> (23 - M)) & mask;
    if (S) t |= (tt >> (31 - M - E)) & (1u << (M + E));
    return t;
}

ORC_API float orc_cfp_to_float(uint32_t c, int S, int E, int M) {
    uint32_t t = c;
    if (E < 8) t |= ((1u << (8 - E - 1)) - 1u) << (E + M);
    t <<= (23 - M);
    if (S) t |= (c & (1u << (M + E))) << (31 - (M + E));
    float f;
    memcpy(&f, &t, 4);
    return f;
}

/* Array form on raw float bit patterns (no float->double round trip, so
 * signalling NaNs keep their bits): codes[i] = encode(in[i]) and
 * dec_bits[i] = bits of decode(codes[i]). */
ORC_API void orc_cfp_convert_bits(const uint32_t *in, uint64_t k, int S, int E, int M,
                                  uint32_t *codes, uint32_t *dec_bits) {
    for (uint64_t i = 0; i < k; ++i) {
        float f;
        memcpy(&f, in + i, 4);
        uint32_t c = orc_cfp_from_float(f, S, E, M);
        float d = orc_cfp_to_float(c, S, E, M);
        codes[i] = c;
        memcpy(dec_bits + i, &d, 4);
    }
}

/* Storage formats of the PageRank contribution vector in the
 * reduced-precision runs.  The cfp ones restate the reference
 * (PR_vary.C:511-570); the others are the GPU library's own formats:
 * round-to-nearest-even bf16 / fp16 and fp8 e4m3 with a per-iteration
 * power-of-two scale (max |contrib| maps below 448). */
enum { ORC_F32 = 0, ORC_F64 = 1, ORC_BF16 = 2, ORC_F16 = 3, ORC_FP8 = 4,
       ORC_CFP_6_10 = 5, ORC_BF16_TRUNC = 6 };

static float q_bf16_rne(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return f;
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return f;
}

/* round-to-nearest-even onto a binary float grid with 'mb' stored mantissa
 * bits, minimum normal exponent emin and largest finite value maxv
 * (saturating); subnormals are kept on the fixed 2^(emin-mb) grid. */
static float q_grid(float f, int mb, int emin, float maxv) {
    if (f == 0.0f || !isfinite(f)) return f;
    float a = fabsf(f);
    int e;
    frexpf(a, &e); /* a = fr * 2^e, fr in [0.5,1) -> exponent e-1 */
    int ex = e - 1;
    if (ex < emin) ex = emin;
    float ulp = ldexpf(1.0f, ex - mb);
    float q = nearbyintf(a / ulp) * ulp; /* default mode: nearest-even */
    if (q > maxv) q = maxv;
    return copysignf(q, f);
}

static float q_f16(float f) { return q_grid(f, 10, -14, 65504.0f); }
static float q_e4m3(float f) { return q_grid(f, 3, -6, 448.0f); }

/* PR_vary's run_prec (PR_vary.C:247-447) with the contribution stored in
 * format fmt and the gather accumulated in double (accum_f64) or float.
 * Unlike PRv, run_prec renormalises by the double 1/s.  For ORC_FP8 the
 * contribution is stored as q(contrib * scale) with scale = 2^k chosen
 * each iteration so that max|contrib|*scale <= 448, and the gather
 * multiplies by 1/scale; ORC_F16 is scaled the same way (to 65504).
 * x_out gets the FP32 rank vector. */
/* One run_prec stage from the current x: iterations continue the shared
 * count *iter while *iter < maxiter and the residual exceeds tol
 * (PR_vary.C:247-447; a staged VARIANT such as 4620 calls run_prec once per
 * stage with the previous stage's ranks, PR_vary.C:652-757). */
ORC_API int orc_pr_vary_staged(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj,
                               const uint32_t *outdeg, int nstages, const int *fmts, const int *accs,
                               const double *tols, int maxiter, double tol, float *x_out, double *deltas);

static int pr_vary_stage(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj, const uint32_t *outdeg,
                         int fmt, int accum_f64, int *iter, int maxiter, double tol, float *x, double *y,
                         float *cq, double *deltas) {
    const float damp = 0.85f;
    double sdelta = 2;
    while (*iter < maxiter && sdelta > tol) {
        /* contribution encode */
        float cmax = 0.0f;
        for (uint32_t v = 0; v < n; ++v) {
            float c = outdeg[v] ? damp * x[v] / (float)outdeg[v] : 0.0f;
            cq[v] = c;
            if (c > cmax) cmax = c;
        }
        float scale = 1.0f;
        if ((fmt == ORC_FP8 || fmt == ORC_F16) && cmax > 0.0f) {
            int e;
            frexpf((fmt == ORC_FP8 ? 448.0f : 65504.0f) / cmax, &e);
            scale = ldexpf(1.0f, e - 1);
        }
        for (uint32_t v = 0; v < n; ++v) {
            float c = cq[v];
            switch (fmt) {
            case ORC_BF16: c = q_bf16_rne(c); break;
            case ORC_F16: c = q_f16(c * scale) / scale; break;
            case ORC_FP8: c = q_e4m3(c * scale) / scale; break;
            case ORC_CFP_6_10: c = orc_cfp_to_float(orc_cfp_from_float(c, 0, 6, 10), 0, 6, 10); break;
            case ORC_BF16_TRUNC: c = orc_cfp_to_float(orc_cfp_from_float(c, 1, 8, 7), 1, 8, 7); break;
            default: break;
            }
            cq[v] = c;
        }
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t d = 0; d < (int64_t)n; ++d) {
            if (accum_f64) {
                double acc = 0;
                for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e) acc += (double)cq[in_adj[e]];
                y[d] = (double)(float)acc;
            } else {
                float acc = 0;
                for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e) acc += cq[in_adj[e]];
                y[d] = (double)acc;
            }
        }
        double s = 0;
        for (uint32_t v = 0; v < n; ++v) s += y[v];
        double w = (1.0 - s) / (double)n;
        s = 0;
        for (uint32_t v = 0; v < n; ++v) { y[v] = (double)(float)(y[v] + w); s += y[v]; }
        double wr = 1.0 / s;
        sdelta = 0;
        for (uint32_t v = 0; v < n; ++v) {
            float yv = (float)(y[v] * wr);
            sdelta += (double)fabsf(x[v] - yv);
            x[v] = yv;
        }
        if (deltas) deltas[*iter] = sdelta;
        ++*iter;
    }
    return 0;
}

/* BF16 PageRank with stochastic rounding and tail averaging (the GPU
 * library's own extension, no reference counterpart): the GPU's update
 * formula (y + (1 - s)/n, renormalised by the double 1/s), float sums,
 * contributions rounded to bfloat16 up or down at random with 16 bits from
 * MurmurHash3's fmix32 of (vertex, iteration) -- the same bits the device
 * uses -- and, with average_last = K, the ranks returned as the mean of
 * iterations maxiter-K .. maxiter-1.  The initial contributions are rounded
 * to nearest. */
static uint32_t sr_bits(uint32_t v, uint32_t it) {
    uint32_t h = v * 0x9E3779B1u + it * 0x85EBCA77u + 0x165667B1u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h & 0xFFFFu;
}

static float bf16_sr(float f, uint32_t v, uint32_t it) {
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u += sr_bits(v, it);
    u &= 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return f;
}

ORC_API int orc_pr_bf16_sr(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj, const uint32_t *outdeg,
                           int stochastic, int maxiter, double tol, int average_last, float *x,
                           double *deltas) {
    const float damp = 0.85f;
    float *c = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    float *y = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    float *acc = (float *)calloc(n ? n : 1, sizeof(float));
    if (!c || !y || !acc) { free(c); free(y); free(acc); return -1; }
    const float x0 = 1.0f / (float)n;
    for (uint32_t v = 0; v < n; ++v) {
        x[v] = x0;
        c[v] = q_bf16_rne(damp * x0 / (float)outdeg[v]);
    }
    const int avg_from = average_last > 0 ? (maxiter - average_last > 0 ? maxiter - average_last : 0) : -1;
    int it = 0, navg = 0;
    double sdelta = 2;
    while (it < maxiter && sdelta > tol) {
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t d = 0; d < (int64_t)n; ++d) {
            float a = 0;
            for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e) a += c[in_adj[e]];
            y[d] = a;
        }
        double s1 = 0;
        for (uint32_t v = 0; v < n; ++v) s1 += (double)y[v];
        const double w = (1.0 - s1) / (double)n;
        const double wf64 = 1.0 / (s1 + (double)n * w);
        sdelta = 0;
        for (uint32_t v = 0; v < n; ++v) {
            float yv = (float)((double)y[v] + w);
            yv = (float)((double)yv * wf64);
            sdelta += (double)fabsf(x[v] - yv);
            x[v] = yv;
            const float cv = damp * yv / (float)outdeg[v];
            c[v] = stochastic ? bf16_sr(cv, v, (uint32_t)it) : q_bf16_rne(cv);
            if (avg_from >= 0 && it >= avg_from) acc[v] += yv;
        }
        if (avg_from >= 0 && it >= avg_from) ++navg;
        if (deltas) deltas[it] = sdelta;
        ++it;
    }
    if (navg > 0) {
        const float inv = 1.0f / (float)navg;
        for (uint32_t v = 0; v < n; ++v) x[v] = acc[v] * inv;
    }
    free(c);
    free(y);
    free(acc);
    return it;
}

ORC_API int orc_pr_vary(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj,
                        const uint32_t *outdeg, int fmt, int accum_f64, int maxiter,
                        double tol, float *x_out, double *deltas) {
    int f[1] = {fmt}, a[1] = {accum_f64};
    double t[1] = {tol};
    return orc_pr_vary_staged(n, in_off, in_adj, outdeg, 1, f, a, t, maxiter, tol, x_out, deltas);
}

/* Staged PR_vary run: stage k with format fmts[k] and accumulation accs[k]
 * until the residual <= tols[k]; the last stage until tol. */
ORC_API int orc_pr_vary_staged(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj,
                               const uint32_t *outdeg, int nstages, const int *fmts, const int *accs,
                               const double *tols, int maxiter, double tol, float *x_out, double *deltas) {
    float *x = x_out;
    double *y = (double *)calloc(n ? n : 1, sizeof(double));
    float *cq = (float *)malloc((size_t)(n ? n : 1) * sizeof(float));
    if (!y || !cq) { free(y); free(cq); return -1; }
    for (uint32_t v = 0; v < n; ++v) x[v] = (float)(1.0 / (double)n);
    int iter = 0;
    for (int k = 0; k < nstages; ++k)
        pr_vary_stage(n, in_off, in_adj, outdeg, fmts[k], accs[k], &iter, maxiter,
                      k + 1 < nstages ? tols[k] : tol, x, y, cq, deltas);
    free(y);
    free(cq);
    return iter;
}

/* ---------------------------------------------------------------------------
 * Flajolet-Martin neighbourhood sizes (reference: bench/FMv.C:262-452, K = 1
 * bit string of 32 bits per vertex, DEFERRED_UPDATE / CONVERGENCE on).
 *
 * mask/prev start at init.  Each iteration over the frontier F (all vertices
 * first): mask[d] |= prev[s] for every edge s->d with s in F (FMv.C:356-358);
 * the output frontier is {d : mask[d] != prev[d]} (FMv.C:347-350).  Over the
 * output, in vertex order: the estimate 2^(lowest zero bit of mask[v]) / 0.77351
 * (2^32-1 for mask 0, 0 for all ones) replaces est[v] (a float), prev[v] =
 * mask[v], and the iteration's sum accumulates estimate - old estimate
 * (FMv.C:386-412); nhm[i] is the running sum as a float, nactv[i] = |F|.
 * Returns the iteration count (the first empty output ends the loop), or -1
 * on an allocation failure or when more than max_iters would be needed.
 * ------------------------------------------------------------------------ */
ORC_API int orc_fm(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *init,
                   uint32_t *mask, float *nhm, uint64_t *nactv, int max_iters) {
    uint32_t *prev = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    float *est = (float *)calloc(n ? n : 1, sizeof(float));
    uint32_t *F = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t *out = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!prev || !est || !F || !out) { free(prev); free(est); free(F); free(out); return -1; }
    for (uint32_t v = 0; v < n; ++v) { mask[v] = prev[v] = init[v]; F[v] = v; }
    uint64_t nf = n;
    double accum = 0;
    int it = 0;
    while (nf) {
        if (it >= max_iters) { it = -1; break; }
        nactv[it] = nf;
        for (uint64_t i = 0; i < nf; ++i) {
            const uint32_t s = F[i];
            for (uint64_t e = off[s]; e < off[s + 1]; ++e) mask[adj[e]] |= prev[s];
        }
        uint64_t no = 0;
        for (uint32_t v = 0; v < n; ++v)
            if (mask[v] != prev[v]) out[no++] = v;
        double sum = 0;
        for (uint64_t i = 0; i < no; ++i) {
            const uint32_t v = out[i], z = ~mask[v];
            const double low = mask[v] == 0 ? 4294967295.0 : (double)(z & (0u - z));
            const double e_new = (1.0 / 0.77351) * low, e_old = (double)est[v];
            prev[v] = mask[v];
            est[v] = (float)e_new;
            sum += e_new - e_old;
        }
        accum += sum;
        nhm[it] = (float)accum;
        uint32_t *t = F; F = out; out = t;
        nf = no;
        ++it;
    }
    free(prev); free(est); free(F); free(out);
    return it;
}

/* The effective diameter FMv derives from the running sums (FMv.C:452-478):
 * interpolated hop count at which the sum reaches 0.9 of its final value,
 * in float arithmetic. */
ORC_API float orc_fm_deffg(const float *nhm, int iters) {
    if (iters <= 1) return 1.0f;
    const float nmax = nhm[iters - 1];
    float nh = nmax, nhm1 = nmax;
    int i;
    for (i = iters - 2; i >= 0; --i) {
        nhm1 = nhm[i];
        if (nhm1 < 0.9 * nmax) break;
        nh = nhm1;
    }
    if (nh == nhm1) return 1.0f;
    return (float)(i + (0.9 * nmax - nhm1) / (nh - nhm1));
}

/* ---------------------------------------------------------------------------
 * Maximal independent set (reference: bench/MISv.C:165-300 with the
 * dfsaop_MIS relation, dsl/ast/dfsaop.h:49-230).  MISv's rounds settle on the
 * greedy set in priority order: a vertex is in (3) when no neighbour of
 * lower priority is in, else out (2); self loops are ignored.  prio[v] is the
 * vertex's rank (MISv compares vertex ids: the file's ids on the device, the
 * layout's ids in the reference build).  Returns the number of vertices in,
 * or -1 on an allocation failure.
 * ------------------------------------------------------------------------ */
ORC_API int64_t orc_mis(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *prio,
                        uint8_t *state) {
    uint32_t *order = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!order) return -1;
    for (uint32_t v = 0; v < n; ++v) { order[v] = 0xFFFFFFFFu; state[v] = 0; }
    for (uint32_t v = 0; v < n; ++v) {
        if (prio[v] >= n || order[prio[v]] != 0xFFFFFFFFu) { free(order); return -1; }  /* not a permutation */
        order[prio[v]] = v;
    }
    int64_t in = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t v = order[i];
        int blocked = 0;
        for (uint64_t e = off[v]; e < off[v + 1] && !blocked; ++e)
            blocked = adj[e] != v && state[adj[e]] == 3;
        state[v] = blocked ? 2 : 3;
        in += !blocked;
    }
    free(order);
    return in;
}

/* ---------------------------------------------------------------------------
 * Accelerated (delta) PageRank (reference: bench/APRv.C:289-505; FloatTy
 * float, DEFERRED_UPDATE, MEMO and UNCOND_EXEC on, UNCOND_EXEC_THRESHOLD 0.6).
 *
 * x = 0, delta = 1/n.  Iteration 0: contrib = delta / outdeg, z[d] = sum of
 * contrib over all in-edges, delta = 0.85 z + 0.15/n, x += delta, delta -=
 * 1/n.  Later iterations sum either over all in-edges with every vertex's
 * contrib (frontier density (|F| + outdeg(F)) / m above 0.6) or over the
 * in-edges from the frontier F only; then delta = 0.85 z and x += delta
 * where the vertex is active.  Active: |delta| > 0.01 x; the active set is
 * the next F.  The loop ends after maxiter iterations or once sum |delta|
 * (a compensated double sum, as a float) is below 1e-7; x is then scaled by
 * 1 / sum |x|.  All vertex arithmetic in float, z summed in float in CSC
 * order.  l1[i] receives each iteration's sum |delta|.  Returns the iteration
 * count, or -1 on an allocation failure.
 * ------------------------------------------------------------------------ */
static double apr_abs_sum(const float *a, uint32_t n) {
    double d = 0.0, err = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        const double t = d, y = fabs((double)a[i]) + err;
        d = t + y;
        err = t - d;
        err += y;
    }
    return d;
}

ORC_API int orc_apr(uint32_t n, const uint64_t *in_off, const uint32_t *in_adj, const uint32_t *outdeg,
                    int maxiter, float *x, double *l1) {
    const size_t nb = (size_t)(n ? n : 1);
    float *delta = (float *)malloc(nb * sizeof(float)), *z = (float *)malloc(nb * sizeof(float));
    float *contrib = (float *)malloc(nb * sizeof(float)), *od = (float *)malloc(nb * sizeof(float));
    uint8_t *F = (uint8_t *)malloc(nb), *act = (uint8_t *)malloc(nb);
    if (!delta || !z || !contrib || !od || !F || !act) {
        free(delta); free(z); free(contrib); free(od); free(F); free(act);
        return -1;
    }
    const float dampen = 0.85f, eps = 1e-7f, eps2 = 1e-2f;
    const float ninv = 1.0f / (float)n;
    const uint64_t m = in_off[n];
    for (uint32_t v = 0; v < n; ++v) {
        x[v] = 0.0f;
        delta[v] = ninv;
        od[v] = (float)outdeg[v];
        F[v] = 1;
    }
    double nactv = n, nacte = (double)m;
    int iter = 0;
    while (iter < maxiter) {
        const float cst = (1.0f - dampen) * ninv;
        const int all_src = iter == 0 || (nactv + nacte) / (double)m > 0.6;
        for (uint32_t v = 0; v < n; ++v) {
            z[v] = 0.0f;
            if (all_src || F[v]) contrib[v] = delta[v] / od[v];
        }
        for (uint32_t d = 0; d < n; ++d) {
            float acc = z[d];
            for (uint64_t e = in_off[d]; e < in_off[d + 1]; ++e)
                if (all_src || F[in_adj[e]]) acc += contrib[in_adj[e]];
            z[d] = acc;
        }
        nactv = 0;
        nacte = 0;
        for (uint32_t v = 0; v < n; ++v) {
            if (iter == 0) {
                delta[v] = dampen * z[v] + cst;
                x[v] += delta[v];
                delta[v] = delta[v] - ninv;
                act[v] = fabsf(delta[v]) > eps2 * x[v];
            } else {
                delta[v] = z[v] * dampen;
                act[v] = fabsf(delta[v]) > eps2 * x[v];
                if (act[v]) x[v] += delta[v];
            }
            if (act[v]) {
                nactv += 1;
                nacte += outdeg[v];
            }
        }
        const float L1 = (float)apr_abs_sum(delta, n);
        if (l1) l1[iter] = L1;
        ++iter;
        memcpy(F, act, nb);
        if (L1 < eps) break;
    }
    const float s = 1.0f / (float)apr_abs_sum(x, n);
    for (uint32_t v = 0; v < n; ++v) x[v] *= s;
    free(delta); free(z); free(contrib); free(od); free(F); free(act);
    return iter;
}

/* ------------------------------------------------------------------------
 * k-core decomposition (reference: bench/KC_bucket.C:107-420, whose peel
 * counts each vertex down from its degree, removes the vertices whose count
 * equals the current bucket K and counts their neighbours down, never below
 * K, KC_bucket.C:343-380).  Restated as the sequential bucket peel of
 * Batagelj and Zaversnik (2003): vertices sorted by count in bins, always
 * removing one of smallest count and moving each neighbour with a larger
 * count one bin down.  Both give every vertex the largest k of a k-core
 * that holds it (the decomposition is unique), except for isolated vertices
 * in the case noted at the end.  core[v]: coreness; returns the largest
 * coreness, or -1 on an allocation failure.
 * ------------------------------------------------------------------------ */
ORC_API int64_t orc_kcore(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t *core) {
    if (n == 0) return 0;
    uint64_t md = 0;
    for (uint32_t v = 0; v < n; ++v) {
        const uint64_t d = off[v + 1] - off[v];
        core[v] = (uint32_t)d;
        if (d > md) md = d;
    }
    uint64_t *bin = (uint64_t *)calloc(md + 2, sizeof(uint64_t));
    uint64_t *pos = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    uint32_t *vert = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    if (!bin || !pos || !vert) { free(bin); free(pos); free(vert); return -1; }
    for (uint32_t v = 0; v < n; ++v) bin[core[v]]++;
    uint64_t start = 0;
    for (uint64_t d = 0; d <= md; ++d) { const uint64_t c = bin[d]; bin[d] = start; start += c; }
    for (uint32_t v = 0; v < n; ++v) { pos[v] = bin[core[v]]++; vert[pos[v]] = v; }
    for (uint64_t d = md; d > 0; --d) bin[d] = bin[d - 1];
    bin[0] = 0;
    int64_t largest = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t v = vert[i];
        if ((int64_t)core[v] > largest) largest = core[v];
        for (uint64_t e = off[v]; e < off[v + 1]; ++e) {
            const uint32_t u = adj[e];
            if (core[u] > core[v]) {   /* u one bin down: swap it with its bin's first */
                const uint32_t du = core[u];
                const uint64_t pu = pos[u], pw = bin[du];
                const uint32_t w = vert[pw];
                if (u != w) { pos[u] = pw; vert[pu] = w; pos[w] = pu; vert[pw] = u; }
                bin[du]++;
                core[u]--;
            }
        }
    }
    free(bin); free(pos); free(vert);
    /* The reference's degree-one preprocessing (KC_bucket.C:131-160): when
     * fewer than n/2 vertices have a degree above one, it counts every
     * vertex's degree-one neighbours off and raises every count to at least
     * 1, isolated vertices included, which keep that 1 (they are in no
     * bucket).  Its output has coreness 1 for them in that case. */
    uint64_t ngt1 = 0;
    for (uint32_t v = 0; v < n; ++v) ngt1 += off[v + 1] - off[v] > 1;
    if (ngt1 < (uint64_t)(n / 2))
        for (uint32_t v = 0; v < n; ++v)
            if (off[v + 1] == off[v]) core[v] = 1;
    if (largest == 0 && ngt1 < (uint64_t)(n / 2)) largest = 1;
    return largest;
}
