// gg_vmap.cu -- vertex_map / vertex_scan / vertex_filter.
//
// Graptor's lazy executor (include/graptor/dsl/vertexmap.h:2120-2446) merges
// consecutive vertex maps and scans into one pass over the vertices.  Here a
// merged chain is a short stack-machine program (gg_vmap_desc) that one
// kernel executes per vertex: loads and stores of vertex properties in their
// storage dtype, double arithmetic on the stack, scan reductions accumulated
// in double (one atomic per CTA per reduction) and an optional filter
// statement that records vertices into an output frontier (vertex_filter).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <cstring>

#include "gg_internal.cuh"

namespace gg {

struct VmArgs {
    uint8_t code[GG_VM_MAX_CODE];
    uint8_t arg[GG_VM_MAX_CODE];
    void *props[GG_VM_MAX_PROPS];
    int dt[GG_VM_MAX_PROPS];
    double consts[GG_VM_MAX_CONSTS];
    int ncode;
    int nreduce;
    double *red_out;
    const uint64_t *off;
    uint32_t n;
    const uint32_t *filter_bits;  // nullptr: all vertices
    uint32_t *out_bits;
    uint32_t *out_b0, *out_b1, *out_b2;
    unsigned long long *out_cnt;
    uint32_t smax, mmax;
};

__device__ __forceinline__ double vm_load(const VmArgs &A, int p, uint32_t v) {
    const void *b = A.props[p];
    switch (A.dt[p]) {
    case GG_I32: return (double)((const int32_t *)b)[v];
    case GG_U32: return (double)((const uint32_t *)b)[v];
    case GG_F32: return (double)((const float *)b)[v];
    case GG_F64: return ((const double *)b)[v];
    case GG_BF16: return (double)__bfloat162float(((const __nv_bfloat16 *)b)[v]);
    case GG_F16: return (double)__half2float(((const __half *)b)[v]);
    case GG_FP8E4M3: {
        __half_raw h = __nv_cvt_fp8_to_halfraw(((const __nv_fp8_storage_t *)b)[v], __NV_E4M3);
        return (double)__half2float(__half(h));
    }
    case GG_CFP_6_10: return (double)__uint_as_float(((uint32_t)((const uint16_t *)b)[v] | (1u << 16)) << 13);
    case GG_BF16_TRUNC: return (double)__uint_as_float((uint32_t)((const uint16_t *)b)[v] << 16);
    case GG_U8: return (double)((const uint8_t *)b)[v];
    }
    return 0.0;
}

__device__ __forceinline__ void vm_store(const VmArgs &A, int p, uint32_t v, double x) {
    void *b = A.props[p];
    switch (A.dt[p]) {
    case GG_I32: ((int32_t *)b)[v] = (int32_t)x; break;
    case GG_U32: ((uint32_t *)b)[v] = (uint32_t)x; break;
    case GG_F32: ((float *)b)[v] = (float)x; break;
    case GG_F64: ((double *)b)[v] = x; break;
    case GG_BF16: ((__nv_bfloat16 *)b)[v] = __float2bfloat16_rn((float)x); break;
    case GG_F16: ((__half *)b)[v] = __float2half_rn((float)x); break;
    case GG_FP8E4M3: ((__nv_fp8_storage_t *)b)[v] = __nv_cvt_float_to_fp8((float)x, __NV_SATFINITE, __NV_E4M3); break;
    case GG_CFP_6_10: ((uint16_t *)b)[v] = (uint16_t)((__float_as_uint((float)x) >> 13) & 0xFFFFu); break;
    case GG_BF16_TRUNC: ((uint16_t *)b)[v] = (uint16_t)(__float_as_uint((float)x) >> 16); break;
    case GG_U8: ((uint8_t *)b)[v] = (uint8_t)x; break;
    }
}

constexpr int kVmStack = 16;
constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_vmap(VmArgs A) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwords = (A.n + 31u) >> 5;
    const uint32_t nw = (gridDim.x * kBlock) >> 5;
    double red[GG_VM_MAX_REDUCE] = {0, 0, 0, 0};
    unsigned long long nv = 0, ne = 0;
    auto u32 = [](double x) { return (uint32_t)(int64_t)x; };
    for (uint32_t w = (blockIdx.x * kBlock + threadIdx.x) >> 5; w < nwords; w += nw) {
        const uint32_t v = (w << 5) + lane;
        bool act = v < A.n;
        if (act && A.filter_bits) act = (A.filter_bits[w] >> lane) & 1u;
        bool sel = false;
        if (act) {
            double st[kVmStack];
            double tmp[GG_VM_MAX_TMP];
            int sp = 0;
            for (int pc = 0; pc < A.ncode; ++pc) {
                const int a = A.arg[pc];
                switch (A.code[pc]) {
                case GG_VM_LOAD: st[sp++] = vm_load(A, a, v); break;
                case GG_VM_STORE: vm_store(A, a, v, st[--sp]); break;
                case GG_VM_CONST: st[sp++] = A.consts[a]; break;
                case GG_VM_VID: st[sp++] = (double)v; break;
                case GG_VM_DEGREE: st[sp++] = (double)(A.off[v + 1] - A.off[v]); break;
                case GG_VM_ADD: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
                case GG_VM_SUB: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
                case GG_VM_MUL: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
                case GG_VM_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
                case GG_VM_ABS: st[sp - 1] = fabs(st[sp - 1]); break;
                case GG_VM_MIN: --sp; st[sp - 1] = fmin(st[sp - 1], st[sp]); break;
                case GG_VM_MAX: --sp; st[sp - 1] = fmax(st[sp - 1], st[sp]); break;
                case GG_VM_EQ: --sp; st[sp - 1] = st[sp - 1] == st[sp] ? 1.0 : 0.0; break;
                case GG_VM_NE: --sp; st[sp - 1] = st[sp - 1] != st[sp] ? 1.0 : 0.0; break;
                case GG_VM_LT: --sp; st[sp - 1] = st[sp - 1] < st[sp] ? 1.0 : 0.0; break;
                case GG_VM_GT: --sp; st[sp - 1] = st[sp - 1] > st[sp] ? 1.0 : 0.0; break;
                case GG_VM_REDUCE_ADD: red[a & 3] += st[--sp]; break;
                case GG_VM_TOF32: st[sp - 1] = (double)(float)st[sp - 1]; break;
                case GG_VM_SELECT: sp -= 2; st[sp - 1] = st[sp - 1] != 0.0 ? st[sp] : st[sp + 1]; break;
                case GG_VM_FILTER: sel = st[--sp] != 0.0; break;
                case GG_VM_DUP: st[sp] = st[sp - 1]; ++sp; break;
                case GG_VM_AND: --sp; st[sp - 1] = (double)(u32(st[sp - 1]) & u32(st[sp])); break;
                case GG_VM_OR: --sp; st[sp - 1] = (double)(u32(st[sp - 1]) | u32(st[sp])); break;
                case GG_VM_XOR: --sp; st[sp - 1] = (double)(u32(st[sp - 1]) ^ u32(st[sp])); break;
                case GG_VM_NOT: st[sp - 1] = (double)(~u32(st[sp - 1])); break;
                case GG_VM_TOU32: st[sp - 1] = (double)u32(st[sp - 1]); break;
                case GG_VM_TSET: tmp[a & (GG_VM_MAX_TMP - 1)] = st[--sp]; break;
                case GG_VM_TGET: st[sp++] = tmp[a & (GG_VM_MAX_TMP - 1)]; break;
                case GG_VM_LE: --sp; st[sp - 1] = st[sp - 1] <= st[sp] ? 1.0 : 0.0; break;
                case GG_VM_GE: --sp; st[sp - 1] = st[sp - 1] >= st[sp] ? 1.0 : 0.0; break;
                default: break;
                }
            }
        }
        if (A.out_cnt) {
            if (A.out_bits) {
                const unsigned bits = __ballot_sync(0xffffffffu, sel);
                if (lane == 0) A.out_bits[w] = bits;
            }
            uint64_t deg = sel ? A.off[v + 1] - A.off[v] : 0;
            if (sel) { nv++; ne += deg; }
            uint32_t bin = deg <= A.smax ? 0u : (deg <= A.mmax ? 1u : 2u);
            const unsigned am = __activemask();
#pragma unroll
            for (uint32_t b = 0; b < NBINS; ++b) {
                unsigned mk = __ballot_sync(am, sel && bin == b);
                if (mk == 0) continue;
                int leader = __ffs(mk) - 1;
                unsigned long long base = 0;
                if ((int)lane == leader) base = atomicAdd(A.out_cnt + FC_BIN0 + b, (unsigned long long)__popc(mk));
                base = __shfl_sync(am, base, leader);
                if (sel && bin == b) {
                    uint32_t *dst = b == 0 ? A.out_b0 : (b == 1 ? A.out_b1 : A.out_b2);
                    dst[base + __popc(mk & ((1u << lane) - 1u))] = v;
                }
            }
        }
    }
    for (int r = 0; r < A.nreduce; ++r) {
        double s = dev::block_sum<double, kBlock>(red[r]);
        if (threadIdx.x == 0) atomicAdd(A.red_out + r, s);
    }
    if (A.out_cnt) {
        nv = dev::block_sum<unsigned long long, kBlock>(nv);
        ne = dev::block_sum<unsigned long long, kBlock>(ne);
        if (threadIdx.x == 0) {
            if (nv) atomicAdd(A.out_cnt + FC_NACTV, nv);
            if (ne) atomicAdd(A.out_cnt + FC_NACTE, ne);
        }
    }
}

// Static check of a program: operand stack depth, indices, opcodes.
static bool vm_validate(const gg_vmap_desc *d, gg_graph *g, std::string &why) {
    if (d->ncode < 0 || d->ncode > GG_VM_MAX_CODE) { why = "ncode out of range"; return false; }
    if (d->nreduce < 0 || d->nreduce > GG_VM_MAX_REDUCE) { why = "nreduce out of range"; return false; }
    int sp = 0;
    for (int pc = 0; pc < d->ncode; ++pc) {
        const int op = d->code[pc], a = d->arg[pc];
        int pop = 0, push = 0;
        switch (op) {
        case GG_VM_END: pc = d->ncode; continue;
        case GG_VM_LOAD: case GG_VM_STORE:
            if (a >= GG_VM_MAX_PROPS || !d->props[a] || d->props[a]->g != g) { why = "bad property operand"; return false; }
            if (op == GG_VM_LOAD) push = 1; else pop = 1;
            break;
        case GG_VM_CONST: if (a >= GG_VM_MAX_CONSTS) { why = "bad constant"; return false; } push = 1; break;
        case GG_VM_VID: case GG_VM_DEGREE: push = 1; break;
        case GG_VM_ADD: case GG_VM_SUB: case GG_VM_MUL: case GG_VM_DIV: case GG_VM_MIN:
        case GG_VM_MAX: case GG_VM_EQ: case GG_VM_NE: case GG_VM_LT: case GG_VM_GT:
        case GG_VM_AND: case GG_VM_OR: case GG_VM_XOR: case GG_VM_LE: case GG_VM_GE:
            pop = 2; push = 1; break;
        case GG_VM_ABS: case GG_VM_TOF32: case GG_VM_NOT: case GG_VM_TOU32: pop = 1; push = 1; break;
        case GG_VM_TSET: if (a >= GG_VM_MAX_TMP) { why = "bad temporary"; return false; } pop = 1; break;
        case GG_VM_TGET: if (a >= GG_VM_MAX_TMP) { why = "bad temporary"; return false; } push = 1; break;
        case GG_VM_REDUCE_ADD: if (a >= d->nreduce) { why = "reduction index"; return false; } pop = 1; break;
        case GG_VM_SELECT: pop = 3; push = 1; break;
        case GG_VM_FILTER: pop = 1; break;
        case GG_VM_DUP: pop = 1; push = 2; break;
        default: why = "unknown opcode"; return false;
        }
        if (sp < pop) { why = "stack underflow"; return false; }
        sp += push - pop;
        if (sp > kVmStack) { why = "stack overflow"; return false; }
    }
    return true;
}

}  // namespace gg

using namespace gg;

extern "C" gg_status gg_vertexmap(gg_graph *g, const gg_vmap_desc *d, gg_frontier *filter,
                                  gg_frontier *out, double *reduce_out) {
    if (!g || !d) return GG_ERR_ARG;
    gg_ctx *ctx = g->ctx;
    std::string why;
    if (!vm_validate(d, g, why)) return set_error(ctx, GG_ERR_ARG, "gg_vertexmap: " + why);
    if (d->nreduce && !reduce_out) return set_error(ctx, GG_ERR_ARG, "gg_vertexmap: reduce_out missing");
    if ((filter && filter->g != g) || (out && out->g != g) || (out && out == filter))
        return set_error(ctx, GG_ERR_ARG, "gg_vertexmap: frontier mismatch");
    VmArgs A;
    memset(&A, 0, sizeof(A));
    memcpy(A.code, d->code, sizeof(A.code));
    memcpy(A.arg, d->arg, sizeof(A.arg));
    for (int i = 0; i < GG_VM_MAX_PROPS; ++i) {
        A.props[i] = d->props[i] ? d->props[i]->d : nullptr;
        A.dt[i] = d->props[i] ? (int)d->props[i]->t : 0;
    }
    memcpy(A.consts, d->consts, sizeof(A.consts));
    A.ncode = d->ncode;
    A.nreduce = d->nreduce;
    A.off = g->off;
    A.n = g->n;
    const Tuning &t = tuning();
    A.smax = t.bin_small_max;
    A.mmax = t.bin_medium_max;
    if (filter && !filter->all) {
        GG_CHECK(frontier_ensure_bitmap(filter));
        A.filter_bits = filter->bitmap;
    }
    if (out) {
        GG_CHECK(frontier_alloc_bins(out));
        GG_CHECK(frontier_alloc_bitmap(out));
        GG_CHECK(frontier_reset_counts(out));
        A.out_bits = out->bitmap;
        A.out_b0 = out->bins[0];
        A.out_b1 = out->bins[1];
        A.out_b2 = out->bins[2];
        A.out_cnt = (unsigned long long *)out->d_cnt;
    }
    double *dred = nullptr;
    if (d->nreduce) {
        void *p;
        GG_CHECK(graph_scratch(g, GG_VM_MAX_REDUCE * sizeof(double), &p));
        dred = (double *)p;
        GG_CUDA(ctx, cudaMemsetAsync(dred, 0, GG_VM_MAX_REDUCE * sizeof(double), ctx->stream));
        A.red_out = dred;
    }
    const uint32_t words = (g->n + 31) / 32;
    uint64_t blocks = ((uint64_t)words * 32 + kBlock - 1) / kBlock;
    uint64_t cap = (uint64_t)ctx->sm_count * t.blocks_per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_vmap<<<(unsigned)blocks, kBlock, 0, ctx->stream>>>(A);
    GG_LAUNCHED(ctx);
    if (out) {
        out->all = false;
        out->has_list = true;
        out->has_bitmap = true;
        out->host_valid = false;
    }
    if (d->nreduce) {
        GG_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, dred, d->nreduce * sizeof(double), cudaMemcpyDeviceToHost,
                                     ctx->stream));
        GG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        memcpy(reduce_out, ctx->h_pinned, d->nreduce * sizeof(double));
    }
    return GG_OK;
}
