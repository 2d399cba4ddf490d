// gg_noalloc.cu -- BFS levels without any allocation by the library.
//
// Some callers cannot let a library call cudaMalloc: code that runs inside a
// memory budget fixed up front (a serving process that owns all device memory
// through its own pool), callers that must not trigger the implicit device
// synchronisation of cudaMalloc/cudaFree in the middle of a pipeline, and
// plug-in hosts that forbid allocation from foreign code.  For them this file
// provides gg_bfs_level_noalloc: the caller passes the graph (device CSR) and
// the output level array (device memory); the frontier queues the traversal
// needs live in one file-scope __device__ array of fixed size, which every GPU
// that loads the library holds until the process exits.
//
// The traversal is the level-synchronous sparse push of the BFS-level
// analytic (relax level[d] = level[s] + 1 for unvisited d, frontier kept as a
// vertex queue), with one warp per frontier vertex; its levels are identical
// to gg_bfs_level's (unreached = n+1).
//
// Limits and rules (also in include/gg.h):
//   * n <= GG_NOALLOC_MAX_VERTICES (2^20); larger graphs are rejected with
//     GG_ERR_ARG and a message, nothing is launched.
//   * The scratch array is shared by every call on a device and keeps the
//     last call's contents; each call clears what must start at zero.  Calls
//     whose work overlaps on the GPU (different streams or host threads)
//     race on it and must be serialised by the caller.
//   * Every call looks up the array's device address with
//     cudaGetSymbolAddress, with the caller's device current.  The address
//     belongs to the current context: after cudaDeviceReset, or under a second
//     context that a driver-API caller created on the same device, the module
//     is loaded again at another address, so no address is kept between calls.
//     The first call on a device also loads the module there; make that first
//     call before any stream capture begins.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "gg.h"

namespace {

constexpr uint32_t kMaxV = GG_NOALLOC_MAX_VERTICES;
// [0, kMaxV)        frontier queue A
// [kMaxV, 2 kMaxV)  frontier queue B
// [2 kMaxV + 0]     length of the queue being written
// [2 kMaxV + 1]     error flag (adjacency entry out of range)
constexpr size_t kWords = 2 * (size_t)kMaxV + 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

void put_err(char *buf, size_t len, const char *msg) {
    if (buf && len) {
        std::strncpy(buf, msg, len - 1);
        buf[len - 1] = '\0';
    }
}

__global__ void k_na_init(int32_t *level, uint32_t n, uint32_t root, uint32_t *qa, uint32_t *ctl) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        level[v] = v == root ? 0 : (int32_t)(n + 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        qa[0] = root;
        ctl[0] = 0;
        ctl[1] = 0;
    }
}

// One warp per queued vertex; unvisited neighbours get level it+1 and are
// appended (warp-aggregated) to the next queue.
__global__ void k_na_push(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                          uint32_t n, int32_t *level, const uint32_t *cur, uint32_t ncur,
                          uint32_t *next, uint32_t *ctl, int32_t it) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const int32_t inf = (int32_t)(n + 1);
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < ncur; i += nw) {
        const uint32_t s = cur[i];
        const uint64_t beg = off[s], end = off[s + 1];
        for (uint64_t base = beg; base < end; base += 32) {
            const uint64_t e = base + lane;
            bool add = false;
            uint32_t d = 0;
            if (e < end) {
                d = adj[e];
                if (d >= n) {
                    ctl[1] = 1;  // malformed graph: skip the edge, report it
                } else if (level[d] == inf) {
                    add = atomicCAS(level + d, inf, it + 1) == inf;
                }
            }
            const unsigned mk = __ballot_sync(0xffffffffu, add);
            if (mk) {
                uint32_t basepos = 0;
                if (lane == (uint32_t)(__ffs(mk) - 1)) basepos = atomicAdd(ctl, (uint32_t)__popc(mk));
                basepos = __shfl_sync(0xffffffffu, basepos, __ffs(mk) - 1);
                if (add) next[basepos + __popc(mk & ((1u << lane) - 1u))] = d;
            }
        }
    }
}

}  // namespace

extern "C" gg_status gg_bfs_level_noalloc(const uint64_t *d_off, const uint32_t *d_adj, uint32_t n,
                                          uint32_t root, int32_t *d_level, void *cuda_stream,
                                          int *iterations, char *err, size_t err_len) {
    put_err(err, err_len, "");
    if (!d_off || !d_adj || !d_level || n == 0) {
        put_err(err, err_len, "gg_bfs_level_noalloc: null pointer or empty graph");
        return GG_ERR_ARG;
    }
    if (n > kMaxV) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "gg_bfs_level_noalloc: n = %u exceeds the fixed scratch limit of %u vertices",
                      n, kMaxV);
        put_err(err, err_len, msg);
        return GG_ERR_ARG;
    }
    if (root >= n) {
        put_err(err, err_len, "gg_bfs_level_noalloc: root out of range");
        return GG_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        put_err(err, err_len, "gg_bfs_level_noalloc: no current CUDA device");
        return GG_ERR_NOT_FOUND;
    }
    // The host-side name of a __device__ array is not its device address:
    // look the address up in the current context.
    void *sp = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress(&sp, g_noalloc_scratch);
        if (e != cudaSuccess || !sp) {
            cudaGetLastError();
            put_err(err, err_len, "gg_bfs_level_noalloc: cudaGetSymbolAddress failed");
            return GG_ERR_CUDA;
        }
    }
    uint32_t *scratch = (uint32_t *)sp;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    uint32_t *qa = scratch, *qb = scratch + kMaxV, *ctl = scratch + 2 * (size_t)kMaxV;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_na_init<<<sms * 4, 256, 0, st>>>(d_level, n, root, qa, ctl);
    {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { put_err(err, err_len, cudaGetErrorString(e)); return GG_ERR_CUDA; }
    }
    uint32_t ncur = 1;
    int it = 0;
    uint32_t *cur = qa, *next = qb;
    while (ncur) {
        cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(uint32_t), st);  // next-queue length
        if (e != cudaSuccess) { put_err(err, err_len, cudaGetErrorString(e)); return GG_ERR_CUDA; }
        uint32_t warps = ncur, blocks = (warps + 7) / 8;
        if (blocks > (uint32_t)sms * 8) blocks = (uint32_t)sms * 8;
        k_na_push<<<blocks, 256, 0, st>>>(d_off, d_adj, n, d_level, cur, ncur, next, ctl, it);
        if ((e = cudaGetLastError()) != cudaSuccess) { put_err(err, err_len, cudaGetErrorString(e)); return GG_ERR_CUDA; }
        uint32_t hctl[2] = {0, 0};
        e = cudaMemcpyAsync(hctl, ctl, sizeof(hctl), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { put_err(err, err_len, cudaGetErrorString(e)); return GG_ERR_CUDA; }
        if (hctl[1]) {
            put_err(err, err_len, "gg_bfs_level_noalloc: adjacency entry >= n");
            return GG_ERR_ARG;
        }
        ncur = hctl[0];
        ++it;
        uint32_t *t = cur; cur = next; next = t;
        if (it > (int)n + 1) { put_err(err, err_len, "gg_bfs_level_noalloc: no convergence"); return GG_ERR_STATE; }
    }
    if (iterations) *iterations = it;
    return GG_OK;
}
