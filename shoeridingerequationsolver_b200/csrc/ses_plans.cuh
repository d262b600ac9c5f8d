// Registry of compiled line-FFT plans (axis length -> radices, elements per
// thread, strided-pass tile width) and their kernels.  Lengths without an
// entry run on the run-time-plan kernels of ses_pass.cuh.
#pragma once

#include <vector>

#include "ses_pass2.cuh"

namespace sesk {

template <typename T>
using PassKernel = void (*)(const PassArgs<T>);

template <typename T>
struct PlanEntry {
    int n = 0, e = 0, r0 = 1, r1 = 1, r2 = 1;
    int ls = 0;             // lines per strided-pass CTA
    int xw = 4;             // warps per contiguous-pass CTA
    PassKernel<T> xk[7];    // by XMode
    PassKernel<T> sk[4];    // by SModeK
};

template <typename K>
inline void allow_smem(K k, int bytes) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <typename T, int N, int E, int R0, int R1, int R2, int LS>
PlanEntry<T> make_plan_entry() {
    PlanEntry<T> p;
    p.n = N;
    p.e = E;
    p.r0 = R0;
    p.r1 = R1;
    p.r2 = R2;
    p.ls = LS;
    p.xw = XShape<T, N, E>::NW;
    p.xk[XM_FWD] = xpass2_kernel<T, XM_FWD, N, E, R0, R1, R2>;
    p.xk[XM_INV] = xpass2_kernel<T, XM_INV, N, E, R0, R1, R2>;
    p.xk[XM_START] = xpass2_kernel<T, XM_START, N, E, R0, R1, R2>;
    p.xk[XM_MID] = xpass2_kernel<T, XM_MID, N, E, R0, R1, R2>;
    p.xk[XM_END] = xpass2_kernel<T, XM_END, N, E, R0, R1, R2>;
    p.xk[XM_1D] = xpass2_kernel<T, XM_1D, N, E, R0, R1, R2>;
    p.xk[XM_REDUCE] = xpass2_kernel<T, XM_REDUCE, N, E, R0, R1, R2>;
    p.sk[SM_FWD] = spass2_kernel<T, SM_FWD, N, E, R0, R1, R2, LS>;
    p.sk[SM_INV] = spass2_kernel<T, SM_INV, N, E, R0, R1, R2, LS>;
    p.sk[SM_FUSED] = spass2_kernel<T, SM_FUSED, N, E, R0, R1, R2, LS>;
    p.sk[SM_REDUCE] = spass2_kernel<T, SM_REDUCE, N, E, R0, R1, R2, LS>;
    const int smem = N * LS * (int)sizeof(cx<T>);
    for (auto k : p.sk) allow_smem(k, smem);
    return p;
}

// defined in ses_plans_*.cu
void register_plans_small(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_mixed(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_256(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_large(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);

}  // namespace sesk
