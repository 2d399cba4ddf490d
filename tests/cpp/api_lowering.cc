// Lowering of the operator surface (include/graptor_b200/api.h) checked on
// the host: the analytics' relax / filter / record expressions become the
// descriptor kinds of gg.h, vertex statements the expected stack programs.
// Built and run by tests/test_api_lowering.py; prints "ok" and returns 0.
#include <cstdio>
#include <cstdlib>

#include "graptor_b200/api.h"

using namespace expr;

static int fails = 0;
#define CHECK(c)                                                   \
    do {                                                           \
        if (!(c)) {                                                \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                               \
        }                                                          \
    } while (0)

static gg_prop *P(int i) { return reinterpret_cast<gg_prop *>(0x1000 * i); }
static E at(int p, gg_dtype dt, NK who) { return ref(P(p), nullptr, dt, var(who)); }

static gg_emap_desc relax_of(const E &e) {
    gg_emap_desc d;
    std::memset(&d, 0, sizeof(d));
    graptor_b200::lower_relax(e.node(), d);
    return d;
}

int main() {
    const NK S = NK::VarSrc, D = NK::VarDst, V = NK::VarV;
    // BFSLVLv.C:209-215, CCv.C:575-581, BFSv.C:144-146, PRv.C:202-212
    CHECK(relax_of(at(1, GG_I32, D).min(at(1, GG_I32, S) + _1)).relax == GG_RELAX_MIN_PLUS1_I32);
    CHECK(relax_of(at(2, GG_U32, D).min(at(2, GG_U32, S))).relax == GG_RELAX_MIN_U32);
    CHECK(relax_of(at(3, GG_U32, D).setif(var(S))).relax == GG_RELAX_SETIF_U32);
    {
        gg_emap_desc d = relax_of(at(4, GG_F64, D) += cast<double>(at(5, GG_F32, S)));
        CHECK(d.relax == GG_RELAX_ADD_GATHER && d.a == P(4) && d.src == P(5) && d.accum_f64 == 1);
        d = relax_of(at(4, GG_F32, D) += cast<float>(at(5, GG_F32, S)));
        CHECK(d.relax == GG_RELAX_ADD_GATHER && d.accum_f64 == 0);
    }
    // validation edgemaps: CCv.C:612-617, BFSLVLv.C:288-305
    CHECK(relax_of(at(2, GG_U32, D) != at(2, GG_U32, S)).relax == GG_RELAX_NE_CHECK);
    CHECK(relax_of(at(1, GG_I32, S) > at(1, GG_I32, D) + _1 || at(1, GG_I32, S) < at(1, GG_I32, D) - _1).relax ==
          GG_RELAX_GAP_CHECK);
    CHECK(relax_of(at(1, GG_I32, S) < at(1, GG_I32, D) - _1).relax == GG_RELAX_AHEAD_CHECK);
    // a relax outside the table names itself
    bool threw = false;
    try {
        relax_of(at(1, GG_I32, D) += at(1, GG_I32, S) * at(1, GG_I32, S));
    } catch (const graptor_b200::error &e) {
        threw = e.status == GG_ERR_UNSUPPORTED;
    }
    CHECK(threw);
    // dst filters and the record method
    {
        gg_emap_desc d;
        std::memset(&d, 0, sizeof(d));
        graptor_b200::lower_dst_filter((at(1, GG_I32, D) > _c(7)).node(), d);
        CHECK(d.dst_filter == GG_FILTER_GT_CONST && d.dst_filter_k == 7);
        graptor_b200::lower_dst_filter((at(2, GG_U32, D) != zero_val(var(D))).node(), d);
        CHECK(d.dst_filter == GG_FILTER_NE_ZERO);
        graptor_b200::lower_record_method((at(2, GG_U32, D) != at(6, GG_U32, D)).node(), d);
        CHECK(d.record == GG_RECORD_NE_PREV && d.prev == P(6));
    }
    // iif(c, l, r) takes r where c holds (the reference's blend order): the
    // program pushes c, then r, then l, then selects
    {
        graptor_b200::VmBuilder b;
        E st = (at(7, GG_F64, V) = iif(at(8, GG_F64, V) > _c(0.5), _c(1.0), _c(2.0)));
        CHECK(b.statement(st.node()));
        // LOAD 8, CONST 0.5, GT, CONST 2.0, CONST 1.0, SELECT, STORE 7
        CHECK(b.d.ncode == 7 && b.d.code[5] == GG_VM_SELECT && b.d.code[6] == GG_VM_STORE);
        CHECK(b.d.consts[b.d.arg[3]] == 2.0 && b.d.consts[b.d.arg[4]] == 1.0);
    }
    // float arithmetic rounds to float; constant_val takes the operand's type
    {
        graptor_b200::VmBuilder b;
        E y = at(9, GG_F32, V);
        CHECK(b.statement((y = constant_val(y, 0.85) * y).node()));
        int tof32 = 0;
        for (int i = 0; i < b.d.ncode; ++i) tof32 += b.d.code[i] == GG_VM_TOF32;
        CHECK(tof32 >= 2);  // the load of y and the float product
        CHECK(b.d.consts[0] == (double)0.85f);
    }
    // FMv.C:347-358: a[d] |= b[s] relax, dst filter a[d] != _1s
    {
        gg_emap_desc d = relax_of(at(1, GG_U32, D) |= at(2, GG_U32, S));
        CHECK(d.relax == GG_RELAX_OR_U32 && d.a == P(1) && d.src == P(2));
        std::memset(&d, 0, sizeof(d));
        graptor_b200::lower_dst_filter((at(1, GG_U32, D) != _1s).node(), d);
        CHECK(d.dst_filter == GG_FILTER_NE_CONST && (uint32_t)d.dst_filter_k == 0xFFFFFFFFu);
    }
    // FMv.C:386-412: the neighbourhood estimate as one vertex program, run
    // here through the documented stack semantics of the opcodes
    {
        double accum = 0;
        E m = at(1, GG_U32, V), pm = at(2, GG_U32, V), est = at(3, GG_F32, V);
        E acc = ref(nullptr, &accum, GG_F64, zero_val(var(V)));
        E st = let<4>(cast<double>(est), [&](E old_est) {
            return let<3>(_c<double>(1.0 / 0.77351) * cast<double>(iif(m != _0, _1s, ~m ^ (~m & (~m - _1)))),
                          [&](E new_est) {
                              return make_seq(pm = m, est = cast<float>(new_est), acc += new_est - old_est);
                          });
        });
        graptor_b200::VmBuilder b;
        CHECK(b.statement(st.node()));
        CHECK(b.d.nreduce == 1);
        const uint32_t masks[] = {0u, 1u, 3u, 0x17u, 0x7FFFFFFFu, 0xFFFFFFFFu, 0x80000000u};
        for (uint32_t mv : masks) {
            double props[8] = {0};
            const int sm = b.prop_slot(P(1)), sp = b.prop_slot(P(2)), se = b.prop_slot(P(3));
            props[sm] = mv;
            props[se] = 5.0;  // the previous estimate
            double stk[16], tmp[GG_VM_MAX_TMP] = {0}, red = 0;
            int sp_ = 0;
            auto u = [](double x) { return (uint32_t)(int64_t)x; };
            for (int i = 0; i < b.d.ncode; ++i) {
                const int a = b.d.arg[i];
                switch (b.d.code[i]) {
                case GG_VM_CONST: stk[sp_++] = b.d.consts[a]; break;
                case GG_VM_LOAD: stk[sp_++] = props[a]; break;
                case GG_VM_STORE: props[a] = stk[--sp_]; break;
                case GG_VM_ADD: --sp_; stk[sp_ - 1] += stk[sp_]; break;
                case GG_VM_SUB: --sp_; stk[sp_ - 1] -= stk[sp_]; break;
                case GG_VM_MUL: --sp_; stk[sp_ - 1] *= stk[sp_]; break;
                case GG_VM_NE: --sp_; stk[sp_ - 1] = stk[sp_ - 1] != stk[sp_]; break;
                case GG_VM_AND: --sp_; stk[sp_ - 1] = u(stk[sp_ - 1]) & u(stk[sp_]); break;
                case GG_VM_XOR: --sp_; stk[sp_ - 1] = u(stk[sp_ - 1]) ^ u(stk[sp_]); break;
                case GG_VM_NOT: stk[sp_ - 1] = (uint32_t)~u(stk[sp_ - 1]); break;
                case GG_VM_TOU32: stk[sp_ - 1] = u(stk[sp_ - 1]); break;
                case GG_VM_TOF32: stk[sp_ - 1] = (float)stk[sp_ - 1]; break;
                case GG_VM_TSET: tmp[a] = stk[--sp_]; break;
                case GG_VM_TGET: stk[sp_++] = tmp[a]; break;
                case GG_VM_SELECT: sp_ -= 2; stk[sp_ - 1] = stk[sp_ - 1] != 0 ? stk[sp_] : stk[sp_ + 1]; break;
                case GG_VM_REDUCE_ADD: red += stk[--sp_]; break;
                default: CHECK(!"unexpected opcode"); i = b.d.ncode; break;
                }
            }
            // rho(~m) = lowest zero bit of m; m == 0 counts as 2^32 - 1 (FMv.C:83-103)
            double lowest = mv == 0 ? 4294967295.0 : (~mv == 0 ? 0.0 : (double)(~mv & (0u - ~mv)));
            const double want = (1.0 / 0.77351) * lowest;
            CHECK(sp_ == 0);
            CHECK(props[sp] == (double)mv);
            CHECK(props[se] == (double)(float)want);
            CHECK(red == want - 5.0);
        }
    }
    // MISv.C:235-256: the MIS relation, record a[d] == 0, frontier on destinations
    {
        E rel = set_mask(var(S) != var(D),
                         make_dfsaop_MIS(at(7, GG_U8, D), at(7, GG_U8, S), make_unop_cvt_to_mask<int>(var(S) < var(D))));
        gg_emap_desc d = relax_of(rel);
        CHECK(d.relax == GG_RELAX_MIS_U8 && d.a == P(7));
        graptor_b200::lower_record_method((at(7, GG_U8, D) == value<simd::ty<uint8_t, 1>, vk_zero>()).node(), d);
        CHECK(d.record == GG_RECORD_EQ_ZERO);
        frontier F;
        api::emap_state st;
        api::emap_arg(st, api::filter(F, api::dst, api::strong));
        CHECK(st.in == &F && st.d.dst_filter == GG_FILTER_IN_FRONTIER);
        api::emap_state st2;
        api::emap_arg(st2, api::filter(F, api::strong, api::src));
        CHECK(st2.in == &F && st2.d.dst_filter == GG_FILTER_NONE && st2.d.src_strong == 1);
    }
    // APRv.C:409-416,455-458: active = cvt_to_vector(|delta| > eps2 * x); x += add_predicate(delta, active != 0)
    {
        graptor_b200::VmBuilder b;
        E x = at(1, GG_F32, V), delta = at(2, GG_F32, V), active = at(3, GG_U32, V);
        CHECK(b.statement((active = make_unop_cvt_to_vector<logical<4>>(make_unop_abs(delta) >
                                                                       constant_val(x, 0.01f) * x)).node()));
        CHECK(b.d.code[b.d.ncode - 1] == GG_VM_STORE && b.d.code[b.d.ncode - 2] == GG_VM_MUL);
        CHECK(b.d.consts[b.d.arg[b.d.ncode - 3]] == 4294967295.0);
        graptor_b200::VmBuilder c;
        CHECK(c.statement((x += add_predicate(delta, active != _0)).node()));
        // the untaken side reloads x: masked vertices keep their value exactly
        CHECK(c.d.code[c.d.ncode - 1] == GG_VM_STORE && c.d.code[c.d.ncode - 2] == GG_VM_SELECT &&
              c.d.code[c.d.ncode - 3] == GG_VM_LOAD && c.d.code[c.d.ncode - 4] == GG_VM_TOF32);
    }
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
