// fm_draws.cc -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// The initial Flajolet-Martin bit masks FMv draws on the host
// (bench/FMv.C:138-165, 291-298): one draw per vertex in vertex order from a
// std::mt19937_64 at its default seed, each a uniform integer in
// [0, 2^32-1] taken through std::uniform_int_distribution, mapped to the mask
// with bit i set where i is the number of leading one bits of the draw
// (probability 2^-(i+1)); the all-ones draw gives the empty mask.  The C++
// standard library is called, not restated, so the draws equal those of any
// program built with the same library (the drop-in FMv and the reference's).
#include <cstdint>
#include <random>

extern "C" void orc_fm_draws(uint64_t n, uint32_t *out) {
    std::mt19937_64 gen;
    gen.seed(std::mt19937_64::default_seed);
    std::uniform_int_distribution<std::mt19937_64::result_type> dist(0, 0xFFFFFFFFu);
    for (uint64_t v = 0; v < n; ++v) {
        const uint32_t h = (uint32_t)dist(gen);
        out[v] = h == 0xFFFFFFFFu ? 0u : (1u << __builtin_clz(~h));
    }
}
