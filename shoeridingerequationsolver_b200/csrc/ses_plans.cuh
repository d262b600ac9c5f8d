// Registry of compiled line-FFT plans (axis length -> radices, elements per
// thread, strided-pass tile width) and their kernels.  Lengths without an
// entry run on the run-time-plan kernels of ses_pass.cuh.
#pragma once

#include <vector>

#include "ses_pass2.cuh"
#include "ses_pass3.cuh"

namespace sesk {

template <typename T>
using PassKernel = void (*)(const PassArgs<T>);

template <typename T>
struct PlanEntry {
    int n = 0, e = 0, r0 = 1, r1 = 1, r2 = 1;
    int ls = 0;             // lines per strided-pass CTA
    int kinds = 3;          // passes this entry serves: 1 contiguous (x), 2 strided (y, z)
    int xw = 4;             // warps per contiguous-pass CTA
    size_t twb = 0;         // bytes of the shared-memory stage-twiddle copy (persistent kernels)
    size_t xbsm = 0;        // dynamic shared memory of the batched register-path x pass
    PassKernel<T> xk[7];    // by XMode
    PassKernel<T> sk[kSModes];  // by SModeK
    // pipelined variants; the solver picks one per axis (default 0, or autotuned)
    using XPipe = void (*)(const PassArgs<T>, const PipeArgs);
    using SPipe = void (*)(const PassArgs<T>, const CUtensorMap, const PipeArgs);
    // batched forms: per-instance arguments (and tensor maps) in global memory
    using XBPipe = void (*)(const PassArgs<T>*, const BatchWork, const PipeArgs);
    using SBPipe = void (*)(const PassArgs<T>*, const CUtensorMap*, const BatchWork, const PipeArgs);
    struct XVar {
        XPipe k[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        XBPipe kb[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        int warps = 0, lpc = 0, nbuf = 0;
        size_t smem[7] = {0, 0, 0, 0, 0, 0, 0};
        size_t smemb[7] = {0, 0, 0, 0, 0, 0, 0};  // batched forms
        int bps[7] = {0, 0, 0, 0, 0, 0, 0};  // resident CTAs per SM
        int bbps[7] = {0, 0, 0, 0, 0, 0, 0};
    };
    struct SVar {
        SPipe k[kSModes] = {};
        SBPipe kb[kSModes] = {};
        int ls = 0, nbuf = 0;
        size_t smem = 0;
        int bps[kSModes] = {};
        int bbps[kSModes] = {};
    };
    std::vector<XVar> xv;
    std::vector<SVar> sv;
    // batched kernels (many fields of this length per launch), by mode
    using XBatch = void (*)(const PassArgs<T>*, const BatchWork);
    XBatch xb[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    XBatch sb[kSModes] = {};
    int xb_bps[7] = {0, 0, 0, 0, 0, 0, 0};  // resident CTAs per SM
    int sb_bps[kSModes] = {};
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
    p.twb = TwStage<T, R0, R1, R2>::bytes;
    p.xbsm = xbatch_smem<T, N, E, R0, R1, R2>();
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
    p.sk[SM_TW_START] = spass2_kernel<T, SM_TW_START, N, E, R0, R1, R2, LS>;
    p.sk[SM_TW_MID] = spass2_kernel<T, SM_TW_MID, N, E, R0, R1, R2, LS>;
    p.sk[SM_TW_END] = spass2_kernel<T, SM_TW_END, N, E, R0, R1, R2, LS>;
    const int smem = N * LS * (int)sizeof(cx<T>);
    for (auto k : p.sk) allow_smem(k, smem);
    p.xb[XM_START] = xbatch_kernel<T, XM_START, N, E, R0, R1, R2>;
    p.xb[XM_MID] = xbatch_kernel<T, XM_MID, N, E, R0, R1, R2>;
    p.xb[XM_END] = xbatch_kernel<T, XM_END, N, E, R0, R1, R2>;
    p.xb[XM_1D] = xbatch_kernel<T, XM_1D, N, E, R0, R1, R2>;
    p.sb[SM_FWD] = sbatch_kernel<T, SM_FWD, N, E, R0, R1, R2, LS>;
    p.sb[SM_INV] = sbatch_kernel<T, SM_INV, N, E, R0, R1, R2, LS>;
    p.sb[SM_FUSED] = sbatch_kernel<T, SM_FUSED, N, E, R0, R1, R2, LS>;
    p.sb[SM_TW_START] = sbatch_kernel<T, SM_TW_START, N, E, R0, R1, R2, LS>;
    p.sb[SM_TW_MID] = sbatch_kernel<T, SM_TW_MID, N, E, R0, R1, R2, LS>;
    p.sb[SM_TW_END] = sbatch_kernel<T, SM_TW_END, N, E, R0, R1, R2, LS>;
    for (int m = 0; m < 7; ++m)
        if (p.xb[m]) {
            allow_smem(p.xb[m], (int)p.xbsm);
            cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&p.xb_bps[m], p.xb[m], p.xw * 32, p.xbsm,
                                                                  cudaOccupancyDefault);
        }
    for (int m = 0; m < kSModes; ++m)
        if (p.sb[m]) {
            allow_smem(p.sb[m], smem + (int)p.twb);
            cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&p.sb_bps[m], p.sb[m], LS * (N / E),
                                                                  smem + p.twb, cudaOccupancyDefault);
        }
    cudaGetLastError();
    return p;
}

// Pipelined variants: contiguous pass with NW warps per CTA, strided pass with
// LS lines per CTA; NBUF-deep tile rings; MINB = CTAs per SM the register
// allocation is sized for.
template <typename T, int N, int E, int R0, int R1, int R2, int NW, int NBUF, int MINB>
void add_x_variant(PlanEntry<T>& p) {
    constexpr int TL = N / E;
    constexpr int LPC = NW * (32 / TL);
    typename PlanEntry<T>::XVar v;
    v.warps = NW;
    v.lpc = LPC;
    v.nbuf = NBUF;
    v.k[XM_FWD] = xpass3_kernel<T, XM_FWD, N, E, R0, R1, R2, NW, NBUF, MINB>;
    v.k[XM_START] = xpass3_kernel<T, XM_START, N, E, R0, R1, R2, NW, NBUF, MINB>;
    v.k[XM_MID] = xpass3_kernel<T, XM_MID, N, E, R0, R1, R2, NW, NBUF, MINB>;
    v.k[XM_END] = xpass3_kernel<T, XM_END, N, E, R0, R1, R2, NW, NBUF, MINB>;
    const size_t psi = (size_t)LPC * N * sizeof(cx<T>);
    if constexpr (sizeof(T) == 4) {  // batched forms for the complex64 batch path
        v.kb[XM_START] = xbatch3_kernel<T, XM_START, N, E, R0, R1, R2, NW, NBUF, MINB>;
        v.kb[XM_MID] = xbatch3_kernel<T, XM_MID, N, E, R0, R1, R2, NW, NBUF, MINB>;
        v.kb[XM_END] = xbatch3_kernel<T, XM_END, N, E, R0, R1, R2, NW, NBUF, MINB>;
    }
    for (int m : {XM_FWD, XM_START, XM_MID, XM_END}) {
        v.smem[m] = pipe_tw_offset(NBUF * (m != XM_FWD ? 2 * psi : psi), NBUF) + TwStage<T, R0, R1, R2>::bytes;
        // batched: each tile buffer also carries its instance's absorber x profile
        v.smemb[m] = pipe_tw_offset(NBUF * (m != XM_FWD ? 2 * psi + N * sizeof(double) : psi), NBUF) +
                     TwStage<T, R0, R1, R2>::bytes;
        allow_smem(v.k[m], (int)v.smem[m]);
        cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&v.bps[m], v.k[m], NW * 32, v.smem[m],
                                                              cudaOccupancyDefault);
        if (v.kb[m]) {
            allow_smem(v.kb[m], (int)v.smemb[m]);
            cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&v.bbps[m], v.kb[m], NW * 32, v.smemb[m],
                                                                  cudaOccupancyDefault);
        }
    }
    cudaGetLastError();
    p.xv.push_back(v);
}

template <typename T, int N, int E, int R0, int R1, int R2, int LS, int NBUF, int MINB>
void add_s_variant(PlanEntry<T>& p) {
    constexpr int TL = N / E;
    typename PlanEntry<T>::SVar v;
    v.ls = LS;
    v.nbuf = NBUF;
    v.k[SM_FWD] = spass3_kernel<T, SM_FWD, N, E, R0, R1, R2, LS, NBUF, MINB>;
    v.k[SM_INV] = spass3_kernel<T, SM_INV, N, E, R0, R1, R2, LS, NBUF, MINB>;
    v.k[SM_FUSED] = spass3_kernel<T, SM_FUSED, N, E, R0, R1, R2, LS, NBUF, MINB>;
    if constexpr (sizeof(T) == 4) {
        v.kb[SM_FWD] = sbatch3_kernel<T, SM_FWD, N, E, R0, R1, R2, LS, NBUF, MINB>;
        v.kb[SM_INV] = sbatch3_kernel<T, SM_INV, N, E, R0, R1, R2, LS, NBUF, MINB>;
        v.kb[SM_FUSED] = sbatch3_kernel<T, SM_FUSED, N, E, R0, R1, R2, LS, NBUF, MINB>;
    }
    v.smem = pipe_tw_offset(NBUF * (size_t)N * LS * sizeof(cx<T>), NBUF) + TwStage<T, R0, R1, R2>::bytes;
    for (int m : {SM_FWD, SM_INV, SM_FUSED}) {
        allow_smem(v.k[m], (int)v.smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&v.bps[m], v.k[m], LS * TL, v.smem,
                                                              cudaOccupancyDefault);
        if (v.kb[m]) {
            allow_smem(v.kb[m], (int)v.smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessorWithFlags(&v.bbps[m], v.kb[m], LS * TL, v.smem,
                                                                  cudaOccupancyDefault);
        }
    }
    cudaGetLastError();
    p.sv.push_back(v);
}

// defined in ses_plans_*.cu
void register_plans_small(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_mixed(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_256(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);
void register_plans_large(std::vector<PlanEntry<float>>& f, std::vector<PlanEntry<double>>& d);

}  // namespace sesk
