// Compiled plans: 512 = 8 x 8 x 8 (complex64 strided passes: 16 x 32), 1024 = 16 x 8 x 8
// (complex64 strided passes: 32 x 32; complex64 only).
#include "ses_plans.cuh"

namespace sesk {
void register_plans_large(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    // complex64 512: 8x8x8 on the contiguous passes, 16x32 (E = 32: one exchange
    // and one twiddled stage per transform) on the strided ones
    f.push_back(make_plan_entry<float, 512, 16, 8, 8, 8, 16>());
    f.back().kinds = 1;
    add_x_variant<float, 512, 16, 8, 8, 8, 4, 2, 1>(f.back());
    add_x_variant<float, 512, 16, 8, 8, 8, 4, 2, 3>(f.back());
    f.push_back(make_plan_entry<float, 512, 32, 16, 32, 1, 8>());
    f.back().kinds = 2;
    add_s_variant<float, 512, 32, 16, 32, 1, 8, 2, 2>(f.back());
    add_s_variant<float, 512, 32, 16, 32, 1, 4, 2, 4>(f.back());
    d.push_back(make_plan_entry<double, 512, 16, 8, 8, 8, 8>());
    add_x_variant<double, 512, 16, 8, 8, 8, 2, 2, 1>(d.back());
    add_s_variant<double, 512, 16, 8, 8, 8, 8, 2, 1>(d.back());
    f.push_back(make_plan_entry<float, 1024, 32, 16, 8, 8, 8>());
    f.back().kinds = 1;
    // complex64 1024 strided passes (the y pass of 1024^2 planes): 32x32, two stages
    f.push_back(make_plan_entry<float, 1024, 32, 32, 32, 1, 4>());
    f.back().kinds = 2;
    add_s_variant<float, 1024, 32, 32, 32, 1, 4, 2, 2>(f.back());
}
}  // namespace sesk
