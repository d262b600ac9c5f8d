// Compiled plans: 512 = 8 x 8 x 8, 1024 = 16 x 8 x 8 (complex64 only).
#include "ses_plans.cuh"

namespace sesk {
void register_plans_large(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    f.push_back(make_plan_entry<float, 512, 16, 8, 8, 8, 16>());
    add_x_variant<float, 512, 16, 8, 8, 8, 4, 2, 1>(f.back());
    add_x_variant<float, 512, 16, 8, 8, 8, 4, 2, 3>(f.back());
    add_s_variant<float, 512, 16, 8, 8, 8, 16, 2, 1>(f.back());
    add_s_variant<float, 512, 16, 8, 8, 8, 8, 2, 2>(f.back());
    d.push_back(make_plan_entry<double, 512, 16, 8, 8, 8, 8>());
    add_x_variant<double, 512, 16, 8, 8, 8, 2, 2, 1>(d.back());
    add_s_variant<double, 512, 16, 8, 8, 8, 8, 2, 1>(d.back());
    f.push_back(make_plan_entry<float, 1024, 32, 16, 8, 8, 8>());
}
}  // namespace sesk
