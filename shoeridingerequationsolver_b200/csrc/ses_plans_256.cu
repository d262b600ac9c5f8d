// Compiled plan 256 = 16 x 16 with its pipelined variants.
#include "ses_plans.cuh"

namespace sesk {
void register_plans_256(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    f.push_back(make_plan_entry<float, 256, 16, 16, 16, 1, 32>());
    add_x_variant<float, 256, 16, 16, 16, 1, 4, 2, 1>(f.back());
    add_x_variant<float, 256, 16, 16, 16, 1, 4, 2, 3>(f.back());
    add_x_variant<float, 256, 16, 16, 16, 1, 8, 2, 2>(f.back());
    add_x_variant<float, 256, 16, 16, 16, 1, 4, 2, 4>(f.back());
    add_x_variant<float, 256, 16, 16, 16, 1, 2, 2, 6>(f.back());
    add_s_variant<float, 256, 16, 16, 16, 1, 32, 2, 1>(f.back());
    add_s_variant<float, 256, 16, 16, 16, 1, 16, 2, 2>(f.back());
    add_s_variant<float, 256, 16, 16, 16, 1, 16, 3, 2>(f.back());
    add_s_variant<float, 256, 16, 16, 16, 1, 8, 2, 4>(f.back());
    d.push_back(make_plan_entry<double, 256, 16, 16, 16, 1, 16>());
    add_x_variant<double, 256, 16, 16, 16, 1, 2, 2, 1>(d.back());
    add_x_variant<double, 256, 16, 16, 16, 1, 4, 2, 2>(d.back());
    add_x_variant<double, 256, 16, 16, 16, 1, 1, 2, 8>(d.back());
    add_s_variant<double, 256, 16, 16, 16, 1, 16, 2, 1>(d.back());
    add_s_variant<double, 256, 16, 16, 16, 1, 8, 2, 2>(d.back());
    add_s_variant<double, 256, 16, 16, 16, 1, 4, 2, 4>(d.back());
}
}  // namespace sesk
