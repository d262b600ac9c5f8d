// Compiled plans with radix-3/5 stages: 48, 96, 160 (160: complex64 only).
#include "ses_plans.cuh"

namespace sesk {
void register_plans_mixed(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    f.push_back(make_plan_entry<float, 48, 12, 4, 4, 3, 32>());
    d.push_back(make_plan_entry<double, 48, 12, 4, 4, 3, 16>());
    f.push_back(make_plan_entry<float, 96, 24, 8, 4, 3, 32>());
    d.push_back(make_plan_entry<double, 96, 24, 8, 4, 3, 16>());
    f.push_back(make_plan_entry<float, 160, 40, 8, 4, 5, 32>());
}
}  // namespace sesk
