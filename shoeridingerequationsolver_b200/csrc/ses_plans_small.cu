// Compiled plans: 16, 32, 64, 128 (pipelined variants for 32, 64, 128).
#include "ses_plans.cuh"

namespace sesk {
void register_plans_small(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    f.push_back(make_plan_entry<float, 16, 16, 16, 1, 1, 32>());
    d.push_back(make_plan_entry<double, 16, 16, 16, 1, 1, 16>());
    f.push_back(make_plan_entry<float, 32, 8, 8, 4, 1, 32>());
    add_x_variant<float, 32, 8, 8, 4, 1, 4, 2, 4>(f.back());
    add_x_variant<float, 32, 8, 8, 4, 1, 8, 2, 2>(f.back());
    add_s_variant<float, 32, 8, 8, 4, 1, 32, 2, 4>(f.back());
    add_s_variant<float, 32, 8, 8, 4, 1, 32, 3, 3>(f.back());
    d.push_back(make_plan_entry<double, 32, 8, 8, 4, 1, 16>());
    f.push_back(make_plan_entry<float, 64, 8, 8, 8, 1, 32>());
    add_x_variant<float, 64, 8, 8, 8, 1, 4, 2, 2>(f.back());
    add_s_variant<float, 64, 8, 8, 8, 1, 32, 2, 2>(f.back());
    d.push_back(make_plan_entry<double, 64, 8, 8, 8, 1, 16>());
    add_x_variant<double, 64, 8, 8, 8, 1, 4, 2, 2>(d.back());
    add_s_variant<double, 64, 8, 8, 8, 1, 16, 2, 2>(d.back());
    f.push_back(make_plan_entry<float, 128, 16, 16, 8, 1, 32>());
    add_x_variant<float, 128, 16, 16, 8, 1, 4, 2, 3>(f.back());
    add_x_variant<float, 128, 16, 16, 8, 1, 2, 2, 6>(f.back());
    add_s_variant<float, 128, 16, 16, 8, 1, 32, 2, 1>(f.back());
    add_s_variant<float, 128, 16, 16, 8, 1, 16, 2, 2>(f.back());
    add_s_variant<float, 128, 16, 16, 8, 1, 8, 2, 4>(f.back());
    d.push_back(make_plan_entry<double, 128, 16, 16, 8, 1, 16>());
}
}  // namespace sesk
