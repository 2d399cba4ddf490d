// ref_cfp.C -- TEST HARNESS around the reference's customfp conversions.
//
// Compiled (by oracle/Makefile) against the UNMODIFIED reference header
// include/graptor/customfp.h.  It converts a list of float bit patterns with
// the reference's own class detail::customfp_em (customfp.h:21-186) in the
// two storage formats that PR_vary uses for the PageRank contribution:
//   customfp<6,10>              (variants 40-46, PR_vary.C:449-526)
//   scustomfp<true,8,7,false,0> (bfloat16 by truncation, variant 99,
//                                PR_vary.C:554-568)
// and writes, per input, four uint32 words: the customfp<6,10> code, the
// bit pattern of its float decode, the scustomfp<true,8,7> code and the bit
// pattern of its float decode.
//
// Usage: ref_cfp <in.u32> <out.u32>   (raw little-endian uint32 arrays)
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "graptor/customfp.h"

using Cfp610 = customfp<6, 10>;
using Bf16T = scustomfp<true, 8, 7, false, 0>;

static uint32_t bits_of(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <in.u32> <out.u32>\n", argv[0]);
        return 2;
    }
    FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return 1;
    std::vector<uint32_t> in;
    uint32_t w;
    while (std::fread(&w, 4, 1, fi) == 1) in.push_back(w);
    std::fclose(fi);
    std::vector<uint32_t> out;
    out.reserve(in.size() * 4);
    for (uint32_t u : in) {
        float f;
        std::memcpy(&f, &u, 4);
        Cfp610 a(f);
        Bf16T b(f);
        out.push_back((uint32_t)a.get());
        out.push_back(bits_of((float)a));
        out.push_back((uint32_t)b.get());
        out.push_back(bits_of((float)b));
    }
    FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return 1;
    std::fwrite(out.data(), 4, out.size(), fo);
    std::fclose(fo);
    return 0;
}
