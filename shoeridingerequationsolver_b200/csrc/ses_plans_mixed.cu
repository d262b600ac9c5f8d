// Compiled plans with radix-3/5 factors: 48 = 12x4 (complex128: 4x4x3), 96 =
// 6x4x4 (complex64 strided passes: 12x8), 160 = 10x4x4 (complex64 strided
// passes: 20x8); radix 6, 10, 12 and 20 are prime-factor butterflies.
// Pipelined complex64 variants.
#include "ses_plans.cuh"

namespace sesk {
void register_plans_mixed(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    // complex64 48 = 12 x 4 (prime-factor radix 12): two stages instead of three
    f.push_back(make_plan_entry<float, 48, 12, 12, 4, 1, 32>());
    add_x_variant<float, 48, 12, 12, 4, 1, 4, 2, 3>(f.back());
    add_s_variant<float, 48, 12, 12, 4, 1, 48, 2, 3>(f.back());
    add_s_variant<float, 48, 12, 12, 4, 1, 16, 2, 8>(f.back());
    d.push_back(make_plan_entry<double, 48, 12, 4, 4, 3, 16>());
    // complex64 96: 6x4x4 on the contiguous passes, 12x8 (E = 24) on the strided ones
    f.push_back(make_plan_entry<float, 96, 12, 6, 4, 4, 32>());
    f.back().kinds = 1;
    add_x_variant<float, 96, 12, 6, 4, 4, 4, 2, 3>(f.back());
    add_x_variant<float, 96, 12, 6, 4, 4, 2, 2, 6>(f.back());
    f.push_back(make_plan_entry<float, 96, 24, 12, 8, 1, 32>());
    f.back().kinds = 2;
    add_s_variant<float, 96, 24, 12, 8, 1, 32, 2, 4>(f.back());
    add_s_variant<float, 96, 24, 12, 8, 1, 16, 2, 8>(f.back());
    d.push_back(make_plan_entry<double, 96, 12, 6, 4, 4, 16>());
    // complex64 160: the contiguous passes keep 10 x 4 x 4 (20 elements per
    // thread, 16 warps per SM); the strided passes run 20 x 8 with 40 elements
    // per thread -- one exchange and one twiddled stage per transform, where
    // the tile in shared memory, not the registers, limits the warps per SM.
    f.push_back(make_plan_entry<float, 160, 20, 10, 4, 4, 32>());
    f.back().kinds = 1;
    add_x_variant<float, 160, 20, 10, 4, 4, 4, 2, 2>(f.back());
    add_x_variant<float, 160, 20, 10, 4, 4, 2, 2, 4>(f.back());
    f.push_back(make_plan_entry<float, 160, 40, 20, 8, 1, 32>());
    f.back().kinds = 2;
    add_s_variant<float, 160, 40, 20, 8, 1, 32, 2, 2>(f.back());
    add_s_variant<float, 160, 40, 20, 8, 1, 16, 2, 4>(f.back());
    d.push_back(make_plan_entry<double, 160, 20, 10, 4, 4, 16>());
}
}  // namespace sesk
