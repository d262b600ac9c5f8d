// Compiled plan: 256 = 16 x 16.
#include "ses_plans.cuh"

namespace sesk {
void register_plans_256(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d) {
    f.push_back(make_plan_entry<float, 256, 16, 16, 16, 1, 32>());
    d.push_back(make_plan_entry<double, 256, 16, 16, 16, 1, 16>());
}
}  // namespace sesk
