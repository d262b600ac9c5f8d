// Element-wise kernels of the engine surface: the norm / peak readout and the
// drift rescale of the reference GPU engine, and the conjugation and transpose
// that give long 1D lines (stored N1 x N2 for the four-step transform) a
// natural-order FFT.  Included by ses_gpu.cu only.
#pragma once

#include "ses_pass.cuh"

namespace sesk {

constexpr int kNormPeakBlocks = 592;  // 4 x 148 SMs, fixed -> deterministic sums

// Engine::norm_and_peak (solver/src/vk_engine.ixx:1665-1692, shader
// solver/shaders/norm_peak.comp.slang): per CTA the FP64 sum and maximum of
// |psi|^2 over a grid-stride range, folded in a fixed order -- partials[2b] =
// sum, partials[2b + 1] = max.
template <typename T>
__global__ void __launch_bounds__(256) norm_peak_kernel(const cx<T>* __restrict__ psi, long long N,
                                                        double* __restrict__ partials) {
    __shared__ double ss[256], sm[256];
    double s = 0.0, m = 0.0;
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < N; i += (long long)gridDim.x * 256) {
        const cx<double> p = widen(psi[i]);
        const double d = p.x * p.x + p.y * p.y;
        s += d;
        m = fmax(m, d);
    }
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            ss[threadIdx.x] += ss[threadIdx.x + h];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = ss[0];
        partials[2 * blockIdx.x + 1] = sm[0];
    }
}

// out[0] = sum of the CTA sums in CTA order, out[1] = largest CTA maximum.
__global__ void norm_peak_finalize(const double* __restrict__ partials, int nblocks, double* out) {
    if (threadIdx.x == 0) {
        double s = 0.0, m = 0.0;
        for (int b = 0; b < nblocks; ++b) {
            s += partials[2 * b];
            m = fmax(m, partials[2 * b + 1]);
        }
        out[0] = s;
        out[1] = m;
    }
}

// psi <- s * conj(psi) when conj, else s * psi (Engine::scale,
// solver/shaders/scale.comp.slang:12-19; complex64 applies the FP64 factor as
// hi + lo, like the 1/N of the step).
template <typename T>
__global__ void __launch_bounds__(256) scale_kernel(cx<T>* __restrict__ psi, long long N, double s, int conj) {
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < N; i += (long long)gridDim.x * 256) {
        const cx<T> v = psi[i];
        psi[i] = scale_d(conj ? cconj(v) : v, s);
    }
}

// out[c * rows + r] = in[r * cols + c] for a rows x cols row-major matrix, in
// 32 x 32 tiles staged through shared memory (both sides coalesced).  Block
// (32, 8), grid (ceil(cols / 32), ceil(rows / 32)).
template <typename T>
__global__ void __launch_bounds__(256) transpose_kernel(const cx<T>* __restrict__ in, cx<T>* __restrict__ out,
                                                        int rows, int cols) {
    __shared__ cx<T> tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * rows + r] = tile[threadIdx.x][k];
    }
}

}  // namespace sesk
