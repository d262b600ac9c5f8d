// Allocation-free real-space observables (ses_observe_real_noalloc).
//
// For callers that cannot allocate device memory: a host framework whose
// caching allocator already owns the GPU's memory (a cudaMalloc from a library
// can fail with out-of-memory while the framework holds free blocks), or a
// latency-critical loop that must not pay cudaMalloc/cudaFree's device-wide
// synchronisation.  The caller passes psi, V and the output in its own device
// memory; the per-CTA partial sums live in a fixed file-scope device array.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "ses_gpu.h"
#include "ses_pass.cuh"

using namespace sesk;

namespace sesk {
void set_last_error(const std::string& msg);  // ses_gpu.cu: the message ses_last_error() returns
}

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 16;
constexpr long long kNoAllocChunk = (long long)kNoAllocThreads * kNoAllocPerThread;  // points per CTA
constexpr long long kNoAllocMaxRows = 32768;  // => at most 32768 * 4096 = 2^27 points (512^3)
constexpr size_t kNoAllocHeader = 256;        // completion counter
constexpr size_t kNoAllocBytes = kNoAllocHeader + (size_t)kNoAllocMaxRows * kRedR * sizeof(double);

// Shared by every call on a device and kept between calls (2.25 MiB per GPU
// that loads the library, held until the process exits).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

ses_status nfail(ses_status s, const std::string& msg) {
    sesk::set_last_error(msg);
    return s;
}

// One CTA reduces a fixed chunk of kNoAllocChunk points into one row of FP64
// partial sums; the last CTA to finish sums the rows in row order (the result
// does not depend on which CTA finishes last) and writes the 9 outputs.
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads)
    obs_real_noalloc_kernel(const cx<T>* __restrict__ psi, const double* __restrict__ V, ObsArgs o,
                            double dv, unsigned char* scratch, double* out) {
    unsigned* done = reinterpret_cast<unsigned*>(scratch);
    double* rows = reinterpret_cast<double*>(scratch + kNoAllocHeader);
    double acc[kRedR];
#pragma unroll
    for (int q = 0; q < kRedR; ++q) acc[q] = 0.0;
    const long long base = (long long)blockIdx.x * kNoAllocChunk;
#pragma unroll 4
    for (int it = 0; it < kNoAllocPerThread; ++it) {
        const long long idx = base + (long long)it * kNoAllocThreads + threadIdx.x;
        if (idx < o.N) {  // N <= 2^27: the 32-bit division by invariant integers applies
            const uint32_t line = fdiv((uint32_t)idx, o.fnx);
            const int i = (int)(idx - (long long)line * o.nx);
            const uint32_t k = fdiv(line, o.fny);
            const int j = (int)(line - k * (uint32_t)o.ny);
            const cx<double> p = widen(psi[idx]);
            const double w = p.x * p.x + p.y * p.y;
            const double x = o.x0 + i * o.hx, y = o.y0 + j * o.hy, z = o.z0 + (double)k * o.hz;
            acc[0] += w;
            if (V) acc[1] += V[idx] * w;
            if (x >= o.xlo && x < o.xhi) acc[2] += w;
            acc[3] += x * w;
            acc[4] += y * w;
            acc[5] += z * w;
            acc[6] += x * x * w;
            acc[7] += y * y * w;
            acc[8] += z * z * w;
        }
    }
    block_reduce_store<kRedR>(acc, rows);  // row blockIdx.x
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double tot[kRedR];
    if (threadIdx.x < kRedR) {
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(&rows[(size_t)b * kRedR + threadIdx.x]);
        tot[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        auto ratio = [](double a, double b) { return b > 0.0 ? a / b : 0.0; };
        out[0] = tot[0] * dv;                 // norm
        out[1] = ratio(tot[1], tot[0]);       // <V>
        out[2] = tot[2] * dv;                 // probability in [xlo, xhi)
        for (int a = 0; a < 3; ++a) {
            const double m = ratio(tot[3 + a], tot[0]);
            const double var = ratio(tot[6 + a], tot[0]) - m * m;
            out[3 + a] = m;                                    // mean position
            out[6 + a] = sqrt(var > 0.0 ? var : 0.0);          // sigma
        }
        *done = 0u;  // ready for the next call
    }
}

// Device address of the scratch array, resolved once per device and context with
// that device current (the host-side symbol is only a stand-in for it).  The
// cache is keyed by the current context as well as the ordinal: after a device
// reset the library's module is loaded again into a new context, at a new
// address, which is then resolved afresh.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (CtxGetCurrentFn) nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    CUcontext c = nullptr;
    if (fn) fn(&c);
    return c;
}

std::mutex g_mu;
void* g_addr[64] = {nullptr};
CUcontext g_ctx[64] = {nullptr};

ses_status scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= 64) return nfail(SES_EINVAL, "device ordinal out of range");
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev] || g_ctx[dev] != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return nfail(SES_EDEVICE, std::string("cudaGetSymbolAddress(scratch) failed: ") +
                                          cudaGetErrorString(e));
        }
        g_addr[dev] = p;
        g_ctx[dev] = ctx;
    }
    *out = static_cast<unsigned char*>(g_addr[dev]);
    return SES_OK;
}

}  // namespace

extern "C" ses_status ses_observe_real_noalloc(const ses_grid_desc* grid, ses_precision prec,
                                               const void* psi_dev, const double* V_dev, double xlo,
                                               double xhi, double* out_dev, void* cuda_stream) {
    if (!grid || !psi_dev || !out_dev) return nfail(SES_EINVAL, "null grid, psi or output pointer");
    if (prec != SES_C128 && prec != SES_C64) return nfail(SES_EINVAL, "unknown precision");
    const ses_axis ax[3] = {grid->x, grid->y, grid->z};
    for (const ses_axis& a : ax)
        if (a.n < 1 || !(a.xmax > a.xmin)) return nfail(SES_EINVAL, "axis needs n >= 1 and xmax > xmin");
    const long long N = (long long)ax[0].n * ax[1].n * ax[2].n;
    const long long rows = (N + kNoAllocChunk - 1) / kNoAllocChunk;
    if (rows > kNoAllocMaxRows)
        return nfail(SES_EINVAL,
                     "grid too large for the allocation-free reduction: at most 134217728 points "
                     "(2^27, e.g. 512^3); use ses_gpu_observe");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nfail(SES_EDEVICE, "no current CUDA device");
    }
    unsigned char* scratch = nullptr;
    ses_status st = scratch_address(dev, &scratch);
    if (st != SES_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(cuda_stream);
    // the completion counter must start at zero (a previous call leaves it at
    // zero; clearing it again keeps a call correct after an interrupted one)
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nfail(SES_EDEVICE, "clearing the scratch counter failed");
    }
    ObsArgs o{};
    o.N = N;
    o.nx = ax[0].n;
    o.ny = ax[1].n;
    o.fnx = make_fastdiv((uint32_t)o.nx);
    o.fny = make_fastdiv((uint32_t)o.ny);
    o.x0 = ax[0].xmin;
    o.hx = (ax[0].xmax - ax[0].xmin) / ax[0].n;
    o.y0 = ax[1].xmin;
    o.hy = (ax[1].xmax - ax[1].xmin) / ax[1].n;
    o.z0 = ax[2].xmin;
    o.hz = (ax[2].xmax - ax[2].xmin) / ax[2].n;
    o.xlo = xlo;
    o.xhi = xhi;
    const double dv = o.hx * o.hy * o.hz;
    if (prec == SES_C128)
        obs_real_noalloc_kernel<double><<<(unsigned)rows, kNoAllocThreads, 0, s>>>(
            static_cast<const cx<double>*>(psi_dev), V_dev, o, dv, scratch, out_dev);
    else
        obs_real_noalloc_kernel<float><<<(unsigned)rows, kNoAllocThreads, 0, s>>>(
            static_cast<const cx<float>*>(psi_dev), V_dev, o, dv, scratch, out_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return nfail(SES_EDEVICE, std::string("launch failed: ") + cudaGetErrorString(e));
    return SES_OK;
}
