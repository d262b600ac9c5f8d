// Host side of the C ABI declared in include/ses_gpu.h: axis plans, the
// solver handle (resident psi + FP64-built tables in HBM), the Strang step
// program, observables and the fft / tables surfaces.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sys/stat.h>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include <mutex>

#include "ses_gpu.h"
#include "ses_aux.cuh"
#include "ses_engine.cuh"
#include "ses_pass.cuh"
#include "ses_plans.cuh"
#include "ses_plane.cuh"

using namespace sesk;

namespace {

thread_local std::string g_err;

ses_status fail(ses_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define SES_CU(call)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(SES_EDEVICE, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

#define SES_TRY(expr)                  \
    do {                               \
        ses_status s_ = (expr);        \
        if (s_ != SES_OK) return s_;   \
    } while (0)

constexpr int kEPT = kEPTDev;      // elements a thread holds per in-place Stockham stage
constexpr int kMaxLog2Radix = kEPTDev >= 16 ? 4 : 3;
constexpr int kMaxAxis = 4096;    // longest supported axis
constexpr int kObsBlocks = 592;   // 4 x 148 SMs, fixed -> deterministic sums
constexpr int kBodyUnroll = 8;    // interior steps per captured graph launch

bool factor_radices(int n, std::vector<int>& rad) {
    rad.clear();
    if (n < 1) return false;
    int a = 0, b = 0, c = 0, m = n;
    while (m % 2 == 0) { m /= 2; ++a; }
    while (m % 3 == 0) { m /= 3; ++b; }
    while (m % 5 == 0) { m /= 5; ++c; }
    if (m != 1) return false;
    if (a) {  // power-of-two part: fewest radix <= kMaxRadix stages, exponents balanced
        const int p = (a + kMaxLog2Radix - 1) / kMaxLog2Radix, base = a / p, extra = a % p;
        for (int i = 0; i < p; ++i) rad.push_back(1 << (base + (i < extra ? 1 : 0)));
    }
    for (int i = 0; i < b; ++i) rad.push_back(3);
    for (int i = 0; i < c; ++i) rad.push_back(5);
    return true;
}

struct PassPlan {
    Geo g{};
    size_t smem = 0;
    unsigned grid = 0;
    long long nlines = 0;
    long long nu = 0, sw = 0, se = 0;
    // compiled plan (nullptr: run-time plan kernels)
    const void* cp = nullptr;
    unsigned cgrid = 0, cblock = 0;
    size_t csmem = 0;
};

struct Registry {
    std::vector<PlanEntry<float>> f;
    std::vector<PlanEntry<double>> d;
    std::vector<PlaneEntry<float>> pf;  // plane passes of the two-sweep step
    std::vector<PlaneEntry<double>> pd;
};

const Registry& registry() {
    static Registry r;
    static std::once_flag once;
    std::call_once(once, [] {
        register_plans_small(r.f, r.d);
        register_plans_mixed(r.f, r.d);
        register_plans_256(r.f, r.d);
        register_plans_large(r.f, r.d);
        register_planes(r.pf, r.pd);
    });
    return r;
}

// The compiled plan of length n for contiguous (kind 1) or strided (kind 2)
// passes; a length may have a different plan for each kind.
template <typename T>
const PlanEntry<T>* find_plan(int n, int kind) {
    const auto& v = [] () -> const std::vector<PlanEntry<T>>& {
        if constexpr (sizeof(T) == 4) return registry().f;
        else return registry().d;
    }();
    for (const auto& e : v)
        if (e.n == n && (e.kinds & kind)) return &e;
    return nullptr;
}

// The plane passes (one per CTAs-per-plane variant) for an nx x ny plane whose x
// and y passes run the compiled plans px and py: the plane pass runs exactly
// those passes' plans and radix orders.
template <typename T>
std::vector<const PlaneEntry<T>*> plane_candidates(int nx, int ny, const PlanEntry<T>* px, const PlanEntry<T>* py) {
    std::vector<const PlaneEntry<T>*> out;
    if (!px || !py) return out;
    const auto& v = [] () -> const std::vector<PlaneEntry<T>>& {
        if constexpr (sizeof(T) == 4) return registry().pf;
        else return registry().pd;
    }();
    for (const auto& e : v)
        if (e.nx == nx && e.ny == ny && e.xe == px->e && e.xr[0] == px->r0 && e.xr[1] == px->r1 &&
            e.xr[2] == px->r2 && e.ye == py->e && e.yr[0] == py->r0 && e.yr[1] == py->r1 && e.yr[2] == py->r2)
            out.push_back(&e);
    return out;
}

// Per-stage twiddles of a compiled plan, forward order then reversed order:
// stage (R, Ns) holds w^{r k N/(Ns R)} at [r*Ns + k], w = e^{-2 pi i/N}, in FP64.
std::vector<double> stage_twiddles(int n, int r0, int r1, int r2) {
    std::vector<double> out;
    auto add_plan = [&](const int* rad, int cnt) {
        int Ns = 1;
        for (int p = 0; p < cnt; ++p) {
            const int R = rad[p];
            for (int r = 0; r < R; ++r)
                for (int k = 0; k < Ns; ++k) {
                    const long long e = ((long long)r * k * (n / (Ns * R))) % n;
                    const double th = -2.0 * 3.14159265358979323846 * (double)e / (double)n;
                    out.push_back(std::cos(th));
                    out.push_back(std::sin(th));
                }
            Ns *= R;
        }
    };
    int fwd[3], cnt = 0;
    for (int r : {r0, r1, r2})
        if (r > 1) fwd[cnt++] = r;
    if (cnt == 0) fwd[cnt++] = 1;
    int rev[3];
    for (int i = 0; i < cnt; ++i) rev[i] = fwd[cnt - 1 - i];
    add_plan(fwd, cnt);
    add_plan(rev, cnt);
    return out;
}

int threads_for(int L, int n, const std::vector<int>& rad) {
    int t = 32;
    for (int R : rad) {
        const int B = kEPT / R;
        const long long nb = (long long)L * n / R;
        t = std::max<long long>(t, (nb + B - 1) / B);
    }
    return (t + 31) / 32 * 32;
}

// Tile shape of one axis pass: L lines of length n, rows of >= 128/256 B for
// coalescing, tile <= 64 KB of shared memory, <= 512 threads.
bool plan_pass(int n, int esize, bool strided, long long nlines, PassPlan& pp, std::string& why) {
    std::vector<int> rad;
    if (!factor_radices(n, rad)) {
        why = "axis length " + std::to_string(n) + " is not of the form 2^a 3^b 5^c";
        return false;
    }
    if (n > kMaxAxis) {
        why = "axis length " + std::to_string(n) + " exceeds " + std::to_string(kMaxAxis);
        return false;
    }
    int L = strided ? 256 / esize : 128 / esize;
    while ((long long)L * n < 2048 && L < 256) L *= 2;
    const int pitch = strided ? n : (n % 2 == 0 ? n + 1 : n);
    while (L > 1 && (size_t)L * pitch * esize > 64 * 1024) L /= 2;
    while (L > 1 && L / 2 >= nlines) L /= 2;
    int T = threads_for(L, n, rad);
    while (T > 512 && L > 1) {
        L /= 2;
        T = threads_for(L, n, rad);
    }
    if (T > 512) {
        why = "no tile shape for axis length " + std::to_string(n);
        return false;
    }
    Geo& g = pp.g;
    g = Geo{};
    g.n = n;
    g.L = L;
    g.lshift = 0;
    while ((1 << g.lshift) < L) ++g.lshift;
    g.nthreads = T;
    g.ls = strided ? 1 : pitch;
    g.es = strided ? L : 1;
    g.nst = (int)rad.size();
    int Ns = 1;
    for (int p = 0; p < g.nst; ++p) {
        g.rad[p] = rad[p];
        g.Ns[p] = Ns;
        g.twstride[p] = n / (Ns * rad[p]);
        g.fNs[p] = make_fastdiv((uint32_t)Ns);
        Ns *= rad[p];
    }
    g.fn = make_fastdiv((uint32_t)n);
    pp.nlines = nlines;
    pp.grid = (unsigned)((nlines + L - 1) / L);
    pp.smem = (size_t)L * pitch * esize;
    if (strided) pp.smem = ((pp.smem + 15) & ~(size_t)15) + (size_t)L * (16 + 16 + 8);
    return true;
}

}  // namespace

namespace sesk {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace sesk

struct ses_solver {
    int dev = 0;
    ses_precision prec = SES_C128;
    int esize = 16;
    double box[6] = {0, 1, 0, 1, 0, 1};
    int n[3] = {1, 1, 1};
    long long N = 0;
    double dt = 0.0, mass = 1.0;
    bool with_tables = true;

    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t cap = nullptr;  // private capture stream for graphs
    cudaEvent_t ev = nullptr;

    void* psi = nullptr;
    void* scratch = nullptr;
    void* vtab = nullptr;
    double* V = nullptr;
    void* tw[3] = {nullptr, nullptr, nullptr};
    double* kv[3] = {nullptr, nullptr, nullptr};
    cx<double>* kd[3] = {nullptr, nullptr, nullptr};
    double* mask1[3] = {nullptr, nullptr, nullptr};
    float* mask1f[3] = {nullptr, nullptr, nullptr};
    cx<float>* kdf[3] = {nullptr, nullptr, nullptr};
    double* maskfull = nullptr;
    bool has_mask = false;

    PassPlan pp[3];
    void* stw[3] = {nullptr, nullptr, nullptr};   // compiled-plan stage twiddles (hi)
    void* stwl[3] = {nullptr, nullptr, nullptr};  // FP32 remainders (lo)
    int last_axis = 0;  // highest axis with n > 1 (0 for 1D / single point)

    double* partials = nullptr;
    size_t partial_rows = 0;
    double* dsums = nullptr;
    double* hsums = nullptr;  // pinned

    cudaGraphExec_t body[2] = {nullptr, nullptr};
    size_t bytes = 0;

    // pipelined passes: TMA descriptors of psi / scratch along y and z, per variant
    static constexpr int kMaxVar = 4;
    CUtensorMap tmap[2][3][kMaxVar];
    bool tmap_ok[2][3][kMaxVar] = {};
    unsigned* derr = nullptr;  // device error word written by bounded waits
    unsigned* herr = nullptr;  // pinned host copy
    int sms = 148;
    bool pipelined = true;
    bool pdl = true;  // single-field passes launched with programmatic stream serialization
    long long wait_limit = 0;      // failure-detection hook: bounded-wait limit of pipelined passes (0: ~2 s)
    uint32_t extra_tx = 0;         // failure-detection hook: bytes each tile barrier expects beyond its copies
    int xsel = 0;                  // pipelined contiguous-pass variant (-1: register path)
    int ssel[3] = {0, 0, 0};       // pipelined strided-pass variant per axis (-1: register path)
    // two-sweep 3D step (plane pass with the y transforms, then the z pass) when
    // the x-y plane fits in shared memory: the compiled plane pass (nullptr: not
    // available for this grid) and whether steps use it
    const void* plane = nullptr;
    bool use_plane = false;
    ses_batch_s* batch = nullptr;  // batch this handle belongs to (its stream is the batch's)
    // long 1D line (nx > 4096, ny = nz = 1) stored as n[0] x n[1] = N1 x N2 and
    // transformed in four steps; box[0..1] and N keep the physical line
    bool long1d = false;
    bool imag = false;       // imaginary-time handle: real weight tables, no absorber
    void* kfull = nullptr;   // kinetic delta per stored k-space element
    void* tw4 = nullptr;     // W_N^{n1 k2} per element (complex64: hi part)
    void* tw4l = nullptr;    // complex64: lo part
    ses_observables* dobs = nullptr;  // ses_gpu_observe_async: observables finished on the device
};

namespace {

// Physical axis length (the layout axes of a long line differ from it).
int phys_n(const ses_solver* h, int a) { return h->long1d ? (a == 0 ? (int)h->N : 1) : h->n[a]; }

// Device buffers of a handle come from the stream-ordered allocator on the
// handle's current stream (every later use of them is ordered after it), and go
// back to it with cudaFreeAsync: creating and destroying handles while other
// work runs (serving) never synchronises the device, as cudaMalloc / cudaFree can.
ses_status dalloc(ses_solver* h, void** p, size_t bytes) {
    cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(SES_ENOMEM, "cudaMallocAsync(" + std::to_string(bytes) + " B) failed: " +
                                    cudaGetErrorString(e));
    }
    h->bytes += bytes;
    return SES_OK;
}

// Small page-locked host buffers (observable sums, error words), carved once from
// 64 KiB chunks and recycled: unlike cudaFreeHost, returning one needs no device
// synchronisation.  Slots are 256 bytes; chunks live until the process exits.
class PinnedSlab {
  public:
    static constexpr size_t kSlot = 256, kChunk = 64 * 1024;
    void* get() {
        std::lock_guard<std::mutex> lk(mu_);
        if (free_.empty()) {
            void* c = nullptr;
            if (cudaMallocHost(&c, kChunk) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            for (size_t o = 0; o < kChunk; o += kSlot) free_.push_back(static_cast<char*>(c) + o);
        }
        void* p = free_.back();
        free_.pop_back();
        return p;
    }
    void put(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        free_.push_back(p);
    }

  private:
    std::mutex mu_;
    std::vector<void*> free_;
};

PinnedSlab& pinned_slab() {
    static PinnedSlab slab;
    return slab;
}

void drop_graphs(ses_solver* h) {
    for (auto& g : h->body) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

void release(ses_solver* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);  // the handle's queued work is done
    drop_graphs(h);
    // back to the stream-ordered allocator (no device-wide synchronisation)
    cudaStream_t fs = h->own ? h->own : h->stream;
    auto dfree = [&](void* p) {
        if (p) cudaFreeAsync(p, fs);
    };
    void* ptrs[] = {h->psi, h->scratch, h->vtab, h->V, h->maskfull, h->partials, h->dsums, h->kfull, h->tw4, h->tw4l,
                    h->dobs, h->derr};
    for (void* p : ptrs) dfree(p);
    for (int a = 0; a < 3; ++a) {
        dfree(h->tw[a]);
        dfree(h->kv[a]);
        dfree(h->kd[a]);
        dfree(h->mask1[a]);
        dfree(h->mask1f[a]);
        dfree(h->kdf[a]);
        dfree(h->stw[a]);
        dfree(h->stwl[a]);
    }
    pinned_slab().put(h->hsums);
    pinned_slab().put(h->herr);
    if (h->ev) cudaEventDestroy(h->ev);
    if (h->cap) cudaStreamDestroy(h->cap);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
}

template <typename K>
void set_smem_attr(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

// Bounded wait on everything queued so far on the handle's stream.
ses_status wait_bounded(ses_solver* h, int timeout_ms) {
    if (timeout_ms <= 0) timeout_ms = 10000;
    if (h->derr) SES_CU(cudaMemcpyAsync(h->herr, h->derr, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    SES_CU(cudaEventRecord(h->ev, h->stream));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(h->ev);
        if (q == cudaSuccess) {
            if (h->herr && *h->herr) {
                *h->herr = 0;
                cudaMemsetAsync(h->derr, 0, sizeof(unsigned), h->stream);
                return fail(SES_ETIMEDOUT, "a pipelined pass gave up waiting for its tile loads");
            }
            return SES_OK;
        }
        if (q != cudaErrorNotReady)
            return fail(SES_EDEVICE, std::string("device error: ") + cudaGetErrorString(q));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms > timeout_ms)
            return fail(SES_ETIMEDOUT, "wait exceeded " + std::to_string(timeout_ms) + " ms");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

template <typename T>
PassArgs<T> make_args(const ses_solver* h, int axis, const void* src, void* dst) {
    PassArgs<T> a{};
    a.src = reinterpret_cast<const cx<T>*>(src);
    a.dst = reinterpret_cast<cx<T>*>(dst);
    a.g = h->pp[axis].g;
    a.axis = axis;
    a.nx = h->n[0];
    a.ny = h->n[1];
    a.nz = h->n[2];
    a.nlines = h->pp[axis].nlines;
    const long long nx = h->n[0], ny = h->n[1];
    if (axis == 0) {
        a.nu = a.nlines;
        a.sw = 0;
        a.se = 1;
    } else if (axis == 1) {
        a.nu = nx;
        a.sw = nx * ny;
        a.se = nx;
    } else {
        a.nu = nx * ny;
        a.sw = 0;
        a.se = nx * ny;
    }
    a.fnu = make_fastdiv((uint32_t)a.nu);
    a.fny = make_fastdiv((uint32_t)ny);
    a.fnx = make_fastdiv((uint32_t)nx);
    a.tw = reinterpret_cast<const cx<T>*>(h->tw[axis]);
    a.stw = reinterpret_cast<const cx<T>*>(h->stw[axis]);
    a.stwl = reinterpret_cast<const cx<T>*>(h->stwl[axis]);
    a.out_scale = 1.0;
    Tables& tb = a.tb;
    tb.vtab = h->vtab;
    for (int q = 0; q < 3; ++q) {
        tb.mask1[q] = h->mask1[q];
        tb.kd[q] = h->kd[q];
        tb.kv[q] = h->kv[q];
        tb.mask1f[q] = h->mask1f[q];
        tb.kdf[q] = h->kdf[q];
    }
    tb.maskfull = h->maskfull;
    tb.inv_mass = 1.0 / h->mass;
    tb.kscale = 1.0 / (double)h->N;
    tb.kfull = h->kfull;
    tb.tw4 = h->tw4;
    tb.tw4l = h->tw4l;
    tb.long_n2 = h->long1d ? h->n[1] : 0;
    a.partials = h->partials;
    return a;
}

template <typename T>
using XKernel = void (*)(const PassArgs<T>);

template <typename T>
XKernel<T> xkernel(int mode) {
    switch (mode) {
        case XM_FWD: return xpass_kernel<T, XM_FWD>;
        case XM_INV: return xpass_kernel<T, XM_INV>;
        case XM_START: return xpass_kernel<T, XM_START>;
        case XM_MID: return xpass_kernel<T, XM_MID>;
        case XM_END: return xpass_kernel<T, XM_END>;
        case XM_1D: return xpass_kernel<T, XM_1D>;
        default: return xpass_kernel<T, XM_REDUCE>;
    }
}

template <typename T>
XKernel<T> skernel(int mode) {
    switch (mode) {
        case SM_FWD: return spass_kernel<T, SM_FWD>;
        case SM_INV: return spass_kernel<T, SM_INV>;
        case SM_FUSED: return spass_kernel<T, SM_FUSED>;
        default: return spass_kernel<T, SM_REDUCE>;
    }
}

// Launch of a pass kernel (single-field or batched), with programmatic stream
// serialization when the handle allows it (the kernel starts while the previous
// kernel of the stream drains and waits in pdl_wait before touching any field).
template <typename... KArgs, typename... Args>
cudaError_t launch_pass(bool pdl, void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem,
                        cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);  // also recorded for cudaGetLastError
}

template <typename T>
ses_status launch(const ses_solver* h, int axis, int mode, const PassArgs<T>& a, cudaStream_t s) {
    const PassPlan& pp = h->pp[axis];
    if (pp.cp) {
        const PlanEntry<T>* e = reinterpret_cast<const PlanEntry<T>*>(pp.cp);
        const int n = h->n[axis];
        const int tl = n / e->e;
        bool done = false;
        const int xs = h->xsel, ss = h->ssel[axis];
        if (h->pipelined && axis == 0 && xs >= 0 && xs < (int)e->xv.size() && e->xv[xs].k[mode] &&
            e->xv[xs].bps[mode] > 0) {
            const auto& v = e->xv[xs];
            PipeArgs pa{};
            pa.ntiles = (int)((pp.nlines + v.lpc - 1) / v.lpc);
            pa.err = h->derr;
            pa.wait_limit = h->wait_limit;
            pa.extra_tx = h->extra_tx;
            const int grid = std::min(pa.ntiles, h->sms * v.bps[mode]);
            launch_pass(h->pdl, v.k[mode], (unsigned)grid, 32u * v.warps, v.smem[mode], s, a, pa);
            done = true;
        } else if (h->pipelined && axis != 0 && ss >= 0 && ss < (int)e->sv.size() && e->sv[ss].k[mode] &&
                   e->sv[ss].bps[mode] > 0) {
            const auto& v = e->sv[ss];
            const int buf = a.src == reinterpret_cast<const cx<T>*>(h->psi) ? 0
                            : (a.src == reinterpret_cast<const cx<T>*>(h->scratch) ? 1 : -1);
            if (buf >= 0 && ss < ses_solver::kMaxVar && h->tmap_ok[buf][axis][ss] && a.src == a.dst &&
                (axis == 2 || h->n[0] % v.ls == 0)) {
                PipeArgs pa{};
                pa.ntiles = (int)((pp.nlines + v.ls - 1) / v.ls);
                pa.kind = axis == 1 ? 0 : 1;
                pa.rows_per_box = n > 256 ? 256 : n;
                pa.nbox = n / pa.rows_per_box;
                pa.err = h->derr;
                pa.wait_limit = h->wait_limit;
                pa.extra_tx = h->extra_tx;
                const int grid = std::min(pa.ntiles, h->sms * v.bps[mode]);
                launch_pass(h->pdl, v.k[mode], (unsigned)grid, (unsigned)(v.ls * tl), v.smem, s, a,
                            h->tmap[buf][axis][ss], pa);
                done = true;
            }
        }
        if (!done) {
            PassKernel<T> k = axis == 0 ? e->xk[mode] : e->sk[mode];
            launch_pass(h->pdl, k, pp.cgrid, pp.cblock, pp.csmem, s, a);
        }
    } else {
        XKernel<T> k = axis == 0 ? xkernel<T>(mode) : skernel<T>(mode);
        launch_pass(h->pdl, k, pp.grid, (unsigned)pp.g.nthreads, pp.smem, s, a);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(SES_EDEVICE, std::string("pass launch: ") + cudaGetErrorString(e));
    return SES_OK;
}

struct XProg {
    int mode = XM_FWD;
    int d_load = DG_NONE, d_mid = DG_NONE, d_store = DG_NONE;
    int m_load = 0, m_mid = 0, m_store = 0;
    double out_scale = 1.0;
    double kick = 0.0;                  // dipole kick theta at this pass's potential site
    const double* kick_axis = nullptr;  // polarization (3 doubles)
};

template <typename T>
ses_status pass_x(const ses_solver* h, const void* src, void* dst, const XProg& p, cudaStream_t s) {
    PassArgs<T> a = make_args<T>(h, 0, src, dst);
    a.d_load = p.d_load;
    a.d_mid = p.d_mid;
    a.d_store = p.d_store;
    a.m_load = p.m_load;
    a.m_mid = p.m_mid;
    a.m_store = p.m_store;
    a.out_scale = p.out_scale;
    if (p.kick != 0.0) {  // driven step: the run-time-plan x pass carries the dipole kick
        a.tb.kick = p.kick;
        for (int q = 0; q < 3; ++q) {
            a.tb.kax[q] = p.kick_axis[q];
            a.tb.korg[q] = h->box[2 * q];
            a.tb.kh[q] = (h->box[2 * q + 1] - h->box[2 * q]) / phys_n(h, q);
        }
        const PassPlan& pp = h->pp[0];
        xkernel<T>(p.mode)<<<pp.grid, pp.g.nthreads, pp.smem, s>>>(a);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(SES_EDEVICE, std::string("driven x pass launch: ") + cudaGetErrorString(e));
        return SES_OK;
    }
    return launch<T>(h, 0, p.mode, a, s);
}

template <typename T>
ses_status pass_s(const ses_solver* h, int axis, const void* src, void* dst, int mode, double scale_,
                  cudaStream_t s) {
    PassArgs<T> a = make_args<T>(h, axis, src, dst);
    a.out_scale = scale_;
    return launch<T>(h, axis, mode, a, s);
}

// Plane pass of the two-sweep 3D step on `field` (PlaneMode `mode`, diagonal
// program of p): the x pass's arguments carry the field, tables and program,
// the y pass's the y stage twiddles and the inverse y pass's scale (1).
template <typename T>
ses_status pass_plane(const ses_solver* h, int mode, const XProg& p, void* field, cudaStream_t s) {
    const PlaneEntry<T>* e = reinterpret_cast<const PlaneEntry<T>*>(h->plane);
    if (!e) return fail(SES_EINVAL, "no plane pass for this grid");
    PassArgs<T> ax = make_args<T>(h, 0, field, field);
    ax.d_load = p.d_load;
    ax.d_mid = p.d_mid;
    ax.d_store = p.d_store;
    ax.m_load = p.m_load;
    ax.m_mid = p.m_mid;
    ax.m_store = p.m_store;
    PassArgs<T> ay = make_args<T>(h, 1, field, field);
    ay.out_scale = 1.0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(h->n[2] * e->cs));  // a cluster of e->cs CTAs per z-plane
    cfg.blockDim = dim3((unsigned)e->nt);
    cfg.dynamicSmemBytes = e->smem;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    int na = 0;
    if (e->cs > 1) {
        at[na].id = cudaLaunchAttributeClusterDimension;
        at[na].val.clusterDim.x = (unsigned)e->cs;
        at[na].val.clusterDim.y = 1;
        at[na].val.clusterDim.z = 1;
        ++na;
    }
    if (h->pdl) {
        at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    cfg.attrs = at;
    cfg.numAttrs = na;
    const cudaError_t err = cudaLaunchKernelEx(&cfg, e->k[mode], ax, ay);
    if (err != cudaSuccess) return fail(SES_EDEVICE, std::string("plane pass launch: ") + cudaGetErrorString(err));
    return SES_OK;
}

// Strided pass of a long line (SM_TW_*), with its potential/mask program.
template <typename T>
ses_status pass_tw(const ses_solver* h, const void* src, void* dst, int mode, const XProg& p, cudaStream_t s) {
    PassArgs<T> a = make_args<T>(h, 1, src, dst);
    a.d_load = p.d_load;
    a.d_mid = p.d_mid;
    a.d_store = p.d_store;
    a.m_load = p.m_load;
    a.m_mid = p.m_mid;
    a.m_store = p.m_store;
    return launch<T>(h, 1, mode, a, s);
}

// x pass of a long line: fwd, kinetic (per-element table), inv.
template <typename T>
ses_status pass_long_x(const ses_solver* h, cudaStream_t s) {
    XProg p;
    p.mode = XM_1D;
    return pass_x<T>(h, h->psi, h->psi, p, s);
}

template <typename T>
void set_attrs_prec() {
    for (int m = XM_FWD; m <= XM_REDUCE; ++m) set_smem_attr(xkernel<T>(m));
    for (int m = SM_FWD; m <= SM_REDUCE; ++m) set_smem_attr(skernel<T>(m));
}

void init_kernel_attrs() {  // once per process; handles may be created from several threads
    static std::once_flag once;
    std::call_once(once, [] {
        set_attrs_prec<float>();
        set_attrs_prec<double>();
    });
}

// y/z part of one step: fwd y, fused z, inv y (3D) or fused y (2D) or fused z.
template <typename T>
ses_status mid_axes(const ses_solver* h, cudaStream_t s) {
    if (h->last_axis == 2) {
        if (h->n[1] > 1) SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_FWD, 1.0, s));
        SES_TRY(pass_s<T>(h, 2, h->psi, h->psi, SM_FUSED, 1.0, s));
        if (h->n[1] > 1) SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_INV, 1.0, s));
    } else if (h->last_axis == 1) {
        SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_FUSED, 1.0, s));
    }
    return SES_OK;
}

// One interior unit of the merged Strang batch.
template <typename T>
ses_status interior_unit(const ses_solver* h, bool mask, cudaStream_t s) {
    XProg p;
    if (h->long1d) {  // [* conj W, inv y, V (M), fwd y, * W] [fwd x, K/N, inv x]
        p.d_mid = DG_FULL;
        p.m_mid = mask;
        SES_TRY(pass_tw<T>(h, h->psi, h->psi, SM_TW_MID, p, s));
        return pass_long_x<T>(h, s);
    }
    if (h->last_axis == 0) {  // 1D: [V M, fwd, K/N, inv]
        p.mode = XM_1D;
        p.d_load = DG_FULL;
        p.m_load = mask;
        return pass_x<T>(h, h->psi, h->psi, p, s);
    }
    if (h->use_plane) {  // [inv y, inv x, V (M), fwd x, fwd y] [fwd z, K/N, inv z]
        p.d_mid = DG_FULL;
        p.m_mid = mask;
        SES_TRY(pass_plane<T>(h, PL_MID, p, h->psi, s));
        return pass_s<T>(h, 2, h->psi, h->psi, SM_FUSED, 1.0, s);
    }
    p.mode = XM_MID;
    p.d_mid = DG_FULL;
    p.m_mid = mask;
    SES_TRY(pass_x<T>(h, h->psi, h->psi, p, s));
    return mid_axes<T>(h, s);
}

template <typename T>
ses_status ensure_body(ses_solver* h, bool mask) {
    cudaGraphExec_t& ex = h->body[mask ? 1 : 0];
    if (ex) return SES_OK;
    if (!h->cap) SES_CU(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
    SES_CU(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
    ses_status st = SES_OK;
    for (int u = 0; u < kBodyUnroll && st == SES_OK; ++u) st = interior_unit<T>(h, mask, h->cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->cap, &graph);
    if (st != SES_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(SES_EDEVICE, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t ie = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        ex = nullptr;
        return fail(SES_EDEVICE, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    return SES_OK;
}

template <typename T>
ses_status enqueue_steps(ses_solver* h, int S, bool mask) {
    cudaStream_t s = h->stream;
    if (h->long1d) {
        // [Vh, fwd y, * W] [x: fwd, K/N, inv] {[* conj W, inv y, V (M), fwd y, * W] [x]} ... [* conj W, inv y, Vh (M)]
        XProg first;
        first.d_load = DG_HALF;
        SES_TRY(pass_tw<T>(h, h->psi, h->psi, SM_TW_START, first, s));
        SES_TRY(pass_long_x<T>(h, s));
        int interior = S - 1;
        if (interior >= kBodyUnroll) SES_TRY(ensure_body<T>(h, mask));
        while (interior >= kBodyUnroll) {
            SES_CU(cudaGraphLaunch(h->body[mask ? 1 : 0], s));
            interior -= kBodyUnroll;
        }
        for (; interior > 0; --interior) SES_TRY(interior_unit<T>(h, mask, s));
        XProg last;
        last.d_store = DG_HALF;
        last.m_store = mask;
        return pass_tw<T>(h, h->psi, h->psi, SM_TW_END, last, s);
    }
    if (h->last_axis == 0) {
        // 1D batch: [Vh] U [V M] U ... U [Vh M], each step one fused x pass
        XProg first;
        first.mode = XM_1D;
        first.d_load = DG_HALF;
        if (S == 1) {
            first.d_store = DG_HALF;
            first.m_store = mask;
        }
        SES_TRY(pass_x<T>(h, h->psi, h->psi, first, s));
        if (S == 1) return SES_OK;
        int interior = S - 2;
        if (interior >= kBodyUnroll) SES_TRY(ensure_body<T>(h, mask));
        while (interior >= kBodyUnroll) {
            SES_CU(cudaGraphLaunch(h->body[mask ? 1 : 0], s));
            interior -= kBodyUnroll;
        }
        for (; interior > 0; --interior) SES_TRY(interior_unit<T>(h, mask, s));
        XProg lastp;
        lastp.mode = XM_1D;
        lastp.d_load = DG_FULL;
        lastp.m_load = mask;
        lastp.d_store = DG_HALF;
        lastp.m_store = mask;
        return pass_x<T>(h, h->psi, h->psi, lastp, s);
    }
    // 3D / 2D: [V/2, fwd x] [y, z] {[inv x, V (M), fwd x] [y, z]} ... [inv x, V/2 (M)];
    // two-sweep 3D: [V/2, fwd x, fwd y] [z] {[inv y, inv x, V (M), fwd x, fwd y] [z]} ... [inv y, inv x, V/2 (M)]
    XProg start;
    start.mode = XM_START;
    start.d_load = DG_HALF;
    if (h->use_plane) {
        SES_TRY(pass_plane<T>(h, PL_START, start, h->psi, s));
        SES_TRY(pass_s<T>(h, 2, h->psi, h->psi, SM_FUSED, 1.0, s));
    } else {
        SES_TRY(pass_x<T>(h, h->psi, h->psi, start, s));
        SES_TRY(mid_axes<T>(h, s));
    }
    int interior = S - 1;
    if (interior >= kBodyUnroll) SES_TRY(ensure_body<T>(h, mask));
    while (interior >= kBodyUnroll) {
        SES_CU(cudaGraphLaunch(h->body[mask ? 1 : 0], s));
        interior -= kBodyUnroll;
    }
    for (; interior > 0; --interior) SES_TRY(interior_unit<T>(h, mask, s));
    XProg end;
    end.mode = XM_END;
    end.d_store = DG_HALF;
    end.m_store = mask;
    if (h->use_plane) return pass_plane<T>(h, PL_END, end, h->psi, s);
    return pass_x<T>(h, h->psi, h->psi, end, s);
}

// Dipole-driven steps (drive.ixx:50-65): kick(t) . step . kick(t + dt) with
// kick theta(t) = amplitude cos(omega t) dt/2; the kicks are diagonal like the
// potential, so they ride on the x passes that apply it (the kick ending step s
// and the one starting step s + 1 as one phase).  Direct launches: the phases
// change every step.
template <typename T>
ses_status enqueue_driven(ses_solver* h, int S, bool mask, const double* axis, double amp, double omega,
                          double t0) {
    cudaStream_t s = h->stream;
    const double dt = h->dt;
    auto theta = [&](double t) { return amp * std::cos(omega * t) * 0.5 * dt; };
    XProg start;
    start.mode = XM_START;
    start.d_load = DG_HALF;
    start.kick = theta(t0);
    start.kick_axis = axis;
    SES_TRY(pass_x<T>(h, h->psi, h->psi, start, s));
    SES_TRY(mid_axes<T>(h, s));
    for (int k = 1; k < S; ++k) {
        const double t_prev = t0 + (k - 1) * dt, t = t0 + k * dt;
        XProg mid;
        mid.mode = XM_MID;
        mid.d_mid = DG_FULL;
        mid.m_mid = mask;
        mid.kick = theta(t_prev + dt) + theta(t);
        mid.kick_axis = axis;
        SES_TRY(pass_x<T>(h, h->psi, h->psi, mid, s));
        SES_TRY(mid_axes<T>(h, s));
    }
    XProg end;
    end.mode = XM_END;
    end.d_store = DG_HALF;
    end.m_store = mask;
    end.kick = theta(t0 + (S - 1) * dt + dt);
    end.kick_axis = axis;
    return pass_x<T>(h, h->psi, h->psi, end, s);
}

// Natural-order transform of a long 1D line x[n1 + N1 n2] (fft(std::vector<cd>&),
// core/src/fft.ixx:75-98).  Four steps: the strided pass transforms over n2 and
// multiplies by W_N^{n1 k2}, the contiguous pass transforms over n1, leaving
// X[k2 + N2 k1] at k1 + N1 k2; a transpose through the scratch field puts it in
// natural order.  The inverse conjugates around the forward transform
// (fft.ixx:89-98): conj(fft(conj(X))) / N.
template <typename T>
ses_status enqueue_fft_long(ses_solver* h, int inverse) {
    cudaStream_t s = h->stream;
    cx<T>* psi = reinterpret_cast<cx<T>*>(h->psi);
    const unsigned eb = (unsigned)std::min<long long>((h->N + 255) / 256, (long long)h->sms * 8);
    if (inverse) scale_kernel<T><<<eb, 256, 0, s>>>(psi, h->N, 1.0, 1);
    XProg none;
    SES_TRY(pass_tw<T>(h, h->psi, h->psi, SM_TW_START, none, s));
    XProg fwd;
    fwd.mode = XM_FWD;
    SES_TRY(pass_x<T>(h, h->psi, h->psi, fwd, s));
    const int n1 = h->n[0], n2 = h->n[1];
    transpose_kernel<T><<<dim3((unsigned)(n1 + 31) / 32, (unsigned)(n2 + 31) / 32), dim3(32, 8), 0, s>>>(
        psi, reinterpret_cast<cx<T>*>(h->scratch), n2, n1);
    SES_CU(cudaGetLastError());
    SES_CU(cudaMemcpyAsync(h->psi, h->scratch, (size_t)h->N * sizeof(cx<T>), cudaMemcpyDeviceToDevice, s));
    if (inverse) scale_kernel<T><<<eb, 256, 0, s>>>(psi, h->N, 1.0 / (double)h->N, 1);
    SES_CU(cudaGetLastError());
    return SES_OK;
}

template <typename T>
ses_status enqueue_fft3(ses_solver* h, void* data, int inverse) {
    cudaStream_t s = h->stream;
    if (h->long1d) return enqueue_fft_long<T>(h, inverse);
    if (!inverse) {
        XProg p;
        p.mode = XM_FWD;
        SES_TRY(pass_x<T>(h, data, data, p, s));
        if (h->n[1] > 1) SES_TRY(pass_s<T>(h, 1, data, data, SM_FWD, 1.0, s));
        if (h->n[2] > 1) SES_TRY(pass_s<T>(h, 2, data, data, SM_FWD, 1.0, s));
        return SES_OK;
    }
    if (h->n[2] > 1) SES_TRY(pass_s<T>(h, 2, data, data, SM_INV, 1.0, s));
    if (h->n[1] > 1) SES_TRY(pass_s<T>(h, 1, data, data, SM_INV, 1.0, s));
    XProg p;
    p.mode = XM_INV;
    p.out_scale = 1.0 / (double)h->N;
    return pass_x<T>(h, data, data, p, s);
}

ObsArgs obs_args(const ses_solver* h, double xlo, double xhi);

// Imaginary time: psi /= sqrt(sum |psi|^2 dV) on the device (the sum stays in dsums[0]).
template <typename T>
ses_status enqueue_renormalize(ses_solver* h) {
    cudaStream_t s = h->stream;
    const ObsArgs o = obs_args(h, -1e300, 1e300);
    obs_real_kernel<T><<<kObsBlocks, 256, 0, s>>>(reinterpret_cast<const cx<T>*>(h->psi), h->V, o, h->partials);
    finalize_kernel<<<1, 32, 0, s>>>(h->partials, kObsBlocks, kRedR, h->dsums);
    const double dv = o.hx * o.hy * o.hz;
    const unsigned gb = (unsigned)std::min<long long>((h->N + 255) / 256, 148 * 16);
    renormalize_kernel<T><<<gb, 256, 0, s>>>(reinterpret_cast<cx<T>*>(h->psi), h->N, h->dsums, dv);
    SES_CU(cudaGetLastError());
    return SES_OK;
}

ObsArgs obs_args(const ses_solver* h, double xlo, double xhi) {
    ObsArgs o{};
    o.N = h->N;
    o.nx = phys_n(h, 0);
    o.ny = phys_n(h, 1);
    o.fnx = make_fastdiv((uint32_t)o.nx);
    o.fny = make_fastdiv((uint32_t)o.ny);
    o.x0 = h->box[0];
    o.hx = (h->box[1] - h->box[0]) / phys_n(h, 0);
    o.y0 = h->box[2];
    o.hy = (h->box[3] - h->box[2]) / phys_n(h, 1);
    o.z0 = h->box[4];
    o.hz = (h->box[5] - h->box[4]) / phys_n(h, 2);
    o.xlo = xlo;
    o.xhi = xhi;
    return o;
}

template <typename T>
ses_status enqueue_observe(ses_solver* h, double xlo, double xhi) {
    cudaStream_t s = h->stream;
    ObsArgs o{};
    o.N = h->N;
    o.nx = phys_n(h, 0);
    o.ny = phys_n(h, 1);
    o.fnx = make_fastdiv((uint32_t)o.nx);
    o.fny = make_fastdiv((uint32_t)o.ny);
    o.x0 = h->box[0];
    o.hx = (h->box[1] - h->box[0]) / phys_n(h, 0);
    o.y0 = h->box[2];
    o.hy = (h->box[3] - h->box[2]) / phys_n(h, 1);
    o.z0 = h->box[4];
    o.hz = (h->box[5] - h->box[4]) / phys_n(h, 2);
    o.xlo = xlo;
    o.xhi = xhi;
    obs_real_kernel<T><<<kObsBlocks, 256, 0, s>>>(reinterpret_cast<const cx<T>*>(h->psi), h->V, o,
                                                  h->partials);
    finalize_kernel<<<1, 32, 0, s>>>(h->partials, kObsBlocks, kRedR, h->dsums);
    SES_CU(cudaGetLastError());
    // k-space: phi = FFT(psi) into the scratch field, reduced in the last pass
    unsigned rows = 0;
    if (h->long1d) {  // k-space copy: [fwd y, * W] into scratch, then [fwd x] reduced
        XProg none;
        SES_TRY(pass_tw<T>(h, h->psi, h->scratch, SM_TW_START, none, s));
        XProg p;
        p.mode = XM_REDUCE;
        SES_TRY(pass_x<T>(h, h->scratch, h->scratch, p, s));
        rows = h->pp[0].cgrid;
    } else if (h->last_axis == 0) {
        XProg p;
        p.mode = XM_REDUCE;
        SES_TRY(pass_x<T>(h, h->psi, h->scratch, p, s));
        rows = h->pp[0].cp ? h->pp[0].cgrid : h->pp[0].grid;
    } else {
        XProg p;
        p.mode = XM_FWD;
        SES_TRY(pass_x<T>(h, h->psi, h->scratch, p, s));
        if (h->last_axis == 2 && h->n[1] > 1)
            SES_TRY(pass_s<T>(h, 1, h->scratch, h->scratch, SM_FWD, 1.0, s));
        SES_TRY(pass_s<T>(h, h->last_axis, h->scratch, h->scratch, SM_REDUCE, 1.0, s));
        rows = h->pp[h->last_axis].cp ? h->pp[h->last_axis].cgrid : h->pp[h->last_axis].grid;
    }
    finalize_kernel<<<1, 32, 0, s>>>(h->partials, (int)rows, kRedK, h->dsums + kRedR);
    SES_CU(cudaGetLastError());
    SES_CU(cudaMemcpyAsync(h->hsums, h->dsums, (kRedR + kRedK) * sizeof(double),
                           cudaMemcpyDeviceToHost, s));
    return SES_OK;
}

// Per-pass timing of one batch (launch kinds: 0 x-mid, 1 y-fwd, 2 fused,
// 3 y-inv, 4 x-start, 5 x-end), events on the handle's stream.
template <typename T>
ses_status profile_batch(ses_solver* h, int S, bool mask, double* out) {
    cudaStream_t s = h->stream;
    std::vector<std::pair<int, cudaEvent_t>> marks;  // kind of the launch that follows
    auto mark = [&](int kind) -> ses_status {
        cudaEvent_t e;
        SES_CU(cudaEventCreate(&e));
        SES_CU(cudaEventRecord(e, s));
        marks.push_back({kind, e});
        return SES_OK;
    };
    ses_status st = SES_OK;
    auto run = [&]() -> ses_status {
        if (h->last_axis == 0) {
            for (int k = 0; k < S; ++k) {
                XProg p;
                p.mode = XM_1D;
                p.d_load = k == 0 ? DG_HALF : DG_FULL;
                p.m_load = k == 0 ? 0 : mask;
                if (k == S - 1) {
                    p.d_store = DG_HALF;
                    p.m_store = mask;
                }
                SES_TRY(mark(k == 0 ? 4 : (k == S - 1 ? 5 : 0)));
                SES_TRY(pass_x<T>(h, h->psi, h->psi, p, s));
            }
            return mark(-1);
        }
        auto mids = [&]() -> ses_status {
            if (h->last_axis == 2) {
                if (h->n[1] > 1) {
                    SES_TRY(mark(1));
                    SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_FWD, 1.0, s));
                }
                SES_TRY(mark(2));
                SES_TRY(pass_s<T>(h, 2, h->psi, h->psi, SM_FUSED, 1.0, s));
                if (h->n[1] > 1) {
                    SES_TRY(mark(3));
                    SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_INV, 1.0, s));
                }
            } else {
                SES_TRY(mark(2));
                SES_TRY(pass_s<T>(h, 1, h->psi, h->psi, SM_FUSED, 1.0, s));
            }
            return SES_OK;
        };
        // two-sweep steps: the plane passes count as x passes (kinds 4, 0, 5), the
        // z pass as the fused pass; the y kinds stay empty
        auto xpass = [&](const XProg& p, int pmode) -> ses_status {
            return h->use_plane ? pass_plane<T>(h, pmode, p, h->psi, s) : pass_x<T>(h, h->psi, h->psi, p, s);
        };
        auto rest = [&]() -> ses_status {
            if (!h->use_plane) return mids();
            SES_TRY(mark(2));
            return pass_s<T>(h, 2, h->psi, h->psi, SM_FUSED, 1.0, s);
        };
        XProg start;
        start.mode = XM_START;
        start.d_load = DG_HALF;
        SES_TRY(mark(4));
        SES_TRY(xpass(start, PL_START));
        SES_TRY(rest());
        for (int k = 1; k < S; ++k) {
            XProg p;
            p.mode = XM_MID;
            p.d_mid = DG_FULL;
            p.m_mid = mask;
            SES_TRY(mark(0));
            SES_TRY(xpass(p, PL_MID));
            SES_TRY(rest());
        }
        XProg end;
        end.mode = XM_END;
        end.d_store = DG_HALF;
        end.m_store = mask;
        SES_TRY(mark(5));
        SES_TRY(xpass(end, PL_END));
        return mark(-1);
    };
    st = run();
    if (st == SES_OK) st = wait_bounded(h, 60000);
    double sum[6] = {0, 0, 0, 0, 0, 0};
    int cnt[6] = {0, 0, 0, 0, 0, 0};
    if (st == SES_OK) {
        for (size_t i = 0; i + 1 < marks.size(); ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, marks[i].second, marks[i + 1].second) != cudaSuccess) {
                st = fail(SES_EDEVICE, "event timing failed");
                break;
            }
            sum[marks[i].first] += ms;
            cnt[marks[i].first] += 1;
        }
        float total = 0.f;
        if (st == SES_OK && marks.size() >= 2)
            cudaEventElapsedTime(&total, marks.front().second, marks.back().second);
        for (int k = 0; k < 6; ++k) out[k] = cnt[k] ? sum[k] / cnt[k] : 0.0;
        out[6] = total;
        out[7] = (double)(marks.size() - 1);
    }
    for (auto& m : marks) cudaEventDestroy(m.second);
    return st;
}

// ---------------------------------------------------------------------------
// Tile-variant selection and autotuning
// ---------------------------------------------------------------------------
std::string tune_cache_path() {
    if (const char* p = std::getenv("SES_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/ses_b200/autotune.txt";
}

std::string tune_key(const ses_solver* h, int axis) {
    std::ostringstream k;
    const char* role = axis == 0 ? "x" : (axis == h->last_axis ? "fused" : "s");
    k << "sm" << h->sms << ":" << (h->prec == SES_C128 ? "c128" : "c64") << ":" << role << ":"
      << h->n[axis] << ":" << h->pp[axis].nlines;
    return k.str();
}

// The cache file's entries, re-read only when its path, size or modification time
// changes (batches look them up at every membership change).
std::map<std::string, int> read_tune_cache() {
    static std::mutex mu;
    static std::string last_path;
    static long long last_mtime = -1, last_size = -1;
    static std::map<std::string, int> last;
    const std::string path = tune_cache_path();
    struct stat st{};
    const bool exists = stat(path.c_str(), &st) == 0;
    const long long mtime = exists ? (long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec : -1;
    const long long size = exists ? (long long)st.st_size : -1;
    std::lock_guard<std::mutex> lk(mu);
    if (path == last_path && mtime == last_mtime && size == last_size) return last;
    std::map<std::string, int> m;
    if (exists) {
        std::ifstream f(path);
        std::string key;
        int v;
        while (f >> key >> v) m[key] = v;
    }
    last_path = path;
    last_mtime = mtime;
    last_size = size;
    last = m;
    return m;
}

void write_tune_cache(const std::map<std::string, int>& add) {
    std::map<std::string, int> m = read_tune_cache();
    for (const auto& kv : add) m[kv.first] = kv.second;
    const std::string path = tune_cache_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        std::string dir = path.substr(0, slash);
        std::string cmd;
        for (size_t i = 1; i <= dir.size(); ++i)  // mkdir -p without a shell
            if (i == dir.size() || dir[i] == '/') {
                const std::string sub = dir.substr(0, i);
                mkdir(sub.c_str(), 0755);
            }
    }
    std::ofstream f(path, std::ios::trunc);
    for (const auto& kv : m) f << kv.first << " " << kv.second << "\n";
}

template <typename T>
int variant_count(const ses_solver* h, int axis) {
    const PlanEntry<T>* e = reinterpret_cast<const PlanEntry<T>*>(h->pp[axis].cp);
    if (!e) return 0;
    return axis == 0 ? (int)e->xv.size() : (int)std::min<size_t>(e->sv.size(), ses_solver::kMaxVar);
}

std::string plane_tune_key(const ses_solver* h) {
    std::ostringstream k;
    k << "sm" << h->sms << ":" << (h->prec == SES_C128 ? "c128" : "c64") << ":plane:" << h->n[0] << "x"
      << h->n[1] << "x" << h->n[2];
    return k.str();
}

// Plane passes of a 3D grid whose x and y axes run compiled plans they were built with.
template <typename T>
std::vector<const PlaneEntry<T>*> handle_planes(const ses_solver* h) {
    if (h->long1d || h->last_axis != 2 || h->n[1] < 2) return {};
    return plane_candidates<T>(h->n[0], h->n[1], reinterpret_cast<const PlanEntry<T>*>(h->pp[0].cp),
                               reinterpret_cast<const PlanEntry<T>*>(h->pp[1].cp));
}

// Step form by CTAs per plane: 0 = four axis passes, cs > 0 = the plane pass of
// that many CTAs per plane (false when the grid has none).
template <typename T>
bool select_plane(ses_solver* h, int cs) {
    h->plane = nullptr;
    h->use_plane = false;
    if (cs <= 0) return true;
    for (const PlaneEntry<T>* e : handle_planes<T>(h))
        if (e->cs == cs) {
            h->plane = e;
            h->use_plane = true;
            return true;
        }
    return false;
}

// Default step form of a grid with plane passes, from B200 measurements of
// single-handle n^3 steps (us per step: four axis passes / plane on 1 CTA / on a
// cluster of 2): complex128 32: 8.2 / 6.9 / 7.7, 48: 12.6 / 12.8 / 11.8,
// 64: 14.6 / 13.1 / 11.8 (the one-CTA plane leaves 84 of 148 SMs idle on 64
// planes); complex64 32: 9.7 / 5.9 / 7.4, 48: 12.8 / 8.5 / 9.7, 64: 12.8 / 10.5 /
// 10.3, 96: 25.9 / 21.5 / 22.6, 128: 47.1 / 36.4 / --.
template <typename T>
int default_plane_cs(const ses_solver* h) {
    auto planes = handle_planes<T>(h);
    if (planes.empty()) return 0;
    const int want = sizeof(T) == 8 && h->n[0] >= 48 ? 2 : 1;
    for (auto* e : planes)
        if (e->cs == want) return want;
    return 0;  // other variants only when the autotuner or SES_PLANE picks them
}

int plane_cs(const ses_solver* h) {
    if (!h->use_plane || !h->plane) return 0;
    return h->prec == SES_C128 ? reinterpret_cast<const PlaneEntry<double>*>(h->plane)->cs
                               : reinterpret_cast<const PlaneEntry<float>*>(h->plane)->cs;
}

void apply_plane_choice(ses_solver* h, int cs) {
    if (h->prec == SES_C128) select_plane<double>(h, cs);
    else select_plane<float>(h, cs);
}

bool has_planes(const ses_solver* h) {
    return h->prec == SES_C128 ? !handle_planes<double>(h).empty() : !handle_planes<float>(h).empty();
}

// Selections at creation: cache, then environment overrides SES_XVAR / SES_SVAR / SES_PLANE.
void apply_selection(ses_solver* h) {
    apply_plane_choice(h, h->prec == SES_C128 ? default_plane_cs<double>(h) : default_plane_cs<float>(h));
    const std::map<std::string, int> cache = read_tune_cache();
    for (int a = 0; a < 3; ++a) {
        auto it = cache.find(tune_key(h, a));
        if (it == cache.end()) continue;
        if (a == 0) h->xsel = it->second;
        else h->ssel[a] = it->second;
    }
    if (has_planes(h)) {  // cached choice, then SES_PLANE (CTAs per plane; 0 = four axis passes)
        auto it = cache.find(plane_tune_key(h));
        if (it != cache.end()) apply_plane_choice(h, it->second);
        if (const char* e = std::getenv("SES_PLANE")) apply_plane_choice(h, std::atoi(e));
    }
    if (const char* e = std::getenv("SES_XVAR")) h->xsel = std::atoi(e);
    if (const char* e = std::getenv("SES_PDL")) h->pdl = std::atoi(e) != 0;
    if (const char* e = std::getenv("SES_SVAR")) h->ssel[1] = h->ssel[2] = std::atoi(e);
}

// Mean ms of `reps` calls of one() on the handle's stream after 2 untimed calls.
template <class F>
ses_status time_reps(ses_solver* h, F& one, int reps, float* ms) {
    cudaStream_t s = h->stream;
    for (int i = 0; i < 2; ++i) SES_TRY(one());
    cudaEvent_t e0, e1;
    SES_CU(cudaEventCreate(&e0));
    SES_CU(cudaEventCreate(&e1));
    cudaEventRecord(e0, s);
    ses_status st = SES_OK;
    for (int i = 0; i < reps && st == SES_OK; ++i) st = one();
    cudaEventRecord(e1, s);
    if (st == SES_OK) st = wait_bounded(h, 60000);
    float t = 0.f;
    if (st == SES_OK) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    return st;
}

// Mean ms of `reps` launches of the axis's step pass on the scratch field.
template <typename T>
ses_status time_axis_pass(ses_solver* h, int axis, int reps, float* ms) {
    cudaStream_t s = h->stream;
    auto one = [&]() -> ses_status {
        if (axis == 0) {
            XProg p;
            if (h->last_axis == 0) {
                p.mode = XM_FWD;  // 1D handles run XM_1D, which has no pipelined variant
            } else {
                p.mode = XM_MID;
                p.d_mid = DG_FULL;
                p.m_mid = h->has_mask;
            }
            return pass_x<T>(h, h->scratch, h->scratch, p, s);
        }
        return pass_s<T>(h, axis, h->scratch, h->scratch, axis == h->last_axis ? SM_FUSED : SM_FWD, 1.0, s);
    };
    return time_reps(h, one, reps, ms);
}

// Mean ms of `reps` interior steps on the scratch field in the handle's current
// step form (four axis passes, or plane pass + z pass).
template <typename T>
ses_status time_step_form(ses_solver* h, int reps, float* ms) {
    cudaStream_t s = h->stream;
    void* f = h->scratch;
    auto one = [&]() -> ses_status {
        XProg p;
        p.mode = XM_MID;
        p.d_mid = DG_FULL;
        p.m_mid = h->has_mask;
        if (h->use_plane) {
            SES_TRY(pass_plane<T>(h, PL_MID, p, f, s));
            return pass_s<T>(h, 2, f, f, SM_FUSED, 1.0, s);
        }
        SES_TRY(pass_x<T>(h, f, f, p, s));
        SES_TRY(pass_s<T>(h, 1, f, f, SM_FWD, 1.0, s));
        SES_TRY(pass_s<T>(h, 2, f, f, SM_FUSED, 1.0, s));
        return pass_s<T>(h, 1, f, f, SM_INV, 1.0, s);
    };
    return time_reps(h, one, reps, ms);
}

template <typename T>
ses_status autotune_impl(ses_solver* h, int flags) {
    std::map<std::string, int> chosen;
    const bool saved_pipe = h->pipelined;
    h->pipelined = true;
    for (int axis = 0; axis < 3; ++axis) {
        if (h->n[axis] < 2 || !h->pp[axis].cp) continue;
        if (axis > 0 && axis != h->last_axis && axis != 1) continue;
        const int nv = variant_count<T>(h, axis);
        int best = -1;
        float best_ms = 1e30f;
        for (int c = -1; c < nv; ++c) {
            if (axis == 0) h->xsel = c;
            else h->ssel[axis] = c;
            float ms = 0.f;
            SES_TRY(time_axis_pass<T>(h, axis, 5, &ms));
            if (ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
        if (axis == 0) h->xsel = best;
        else h->ssel[axis] = best;
        chosen[tune_key(h, axis)] = best;
    }
    const auto planes = handle_planes<T>(h);
    if (!planes.empty()) {  // step form: four axis passes, or a plane pass (by CTAs per plane) + z pass
        select_plane<T>(h, 0);
        float best_ms = 0.f;
        SES_TRY(time_step_form<T>(h, 10, &best_ms));
        int best = 0;
        for (const PlaneEntry<T>* e : planes) {
            select_plane<T>(h, e->cs);
            float ms = 0.f;
            SES_TRY(time_step_form<T>(h, 10, &ms));
            if (ms < best_ms) {
                best_ms = ms;
                best = e->cs;
            }
        }
        select_plane<T>(h, best);
        chosen[plane_tune_key(h)] = best;
    }
    h->pipelined = saved_pipe;
    drop_graphs(h);
    if (flags & 1) write_tune_cache(chosen);
    return SES_OK;
}

template <typename T>
std::string plan_info_t(const ses_solver* h) {
    std::ostringstream o;
    if (h->long1d) o << "line of " << h->N << " as " << h->n[0] << " x " << h->n[1] << " (four-step): ";
    const char* names[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
        o << names[a] << ":" << h->n[a];
        const PlanEntry<T>* e = reinterpret_cast<const PlanEntry<T>*>(h->pp[a].cp);
        if (h->n[a] < 2) {
            o << " (untransformed)";
        } else if (!e) {
            o << " run-time plan (" << h->pp[a].g.nst << " stages)";
        } else {
            o << " compiled " << e->r0;
            if (e->r1 > 1) o << "x" << e->r1;
            if (e->r2 > 1) o << "x" << e->r2;
            o << " E=" << e->e;
            const int sel = a == 0 ? h->xsel : h->ssel[a];
            const int nv = a == 0 ? (int)e->xv.size() : (int)e->sv.size();
            if (!h->pipelined || sel < 0 || sel >= nv) {
                o << " register-path";
            } else if (a == 0) {
                o << " pipelined warps=" << e->xv[sel].warps << " ring=" << e->xv[sel].nbuf << " (variant "
                  << sel << ")";
            } else {
                o << " pipelined TMA lines=" << e->sv[sel].ls << " ring=" << e->sv[sel].nbuf << " (variant "
                  << sel << ")";
            }
        }
        if (a < 2) o << "; ";
    }
    if (has_planes(h)) {
        const int cs = plane_cs(h);
        o << "; step: ";
        if (cs == 0) o << "four axis passes";
        else o << "two sweeps (x-y plane pass on " << cs << (cs == 1 ? " CTA" : " CTAs") << " per plane, z pass)";
    }
    return o.str();
}

ses_status check_handle(ses_handle h) {
    if (!h) return fail(SES_EINVAL, "null handle");
    return SES_OK;
}

template <typename T>
ses_status build_tables(ses_solver* h) {
    const long long N = h->N;
    const int tb = 256;
    const unsigned gb = (unsigned)std::min<long long>((N + tb - 1) / tb, 148 * 32);
    if (h->imag) {
        if (h->prec == SES_C128)
            build_vtab_imag_c128<<<gb, tb, 0, h->stream>>>(h->V, reinterpret_cast<cx<double>*>(h->vtab), N, h->dt);
        else
            build_vtab_imag_c64<<<gb, tb, 0, h->stream>>>(h->V, reinterpret_cast<cx<float>*>(h->vtab), N, h->dt);
        SES_CU(cudaGetLastError());
        return SES_OK;
    }
    if (h->prec == SES_C128)
        build_vtab_c128<<<gb, tb, 0, h->stream>>>(h->V, reinterpret_cast<cx<double>*>(h->vtab), N,
                                                   h->dt);
    else
        build_vtab_c64<<<gb, tb, 0, h->stream>>>(h->V, reinterpret_cast<cx<float>*>(h->vtab), N,
                                                  h->dt);
    SES_CU(cudaGetLastError());
    return SES_OK;
}

void attach_compiled_plan(ses_solver* h, int axis) {
    PassPlan& pp = h->pp[axis];
    const int n = h->n[axis];
    pp.cp = nullptr;
    if (n < 2) return;
    int e = 0, ls = 0, xw = 4;
    const int kind = axis == 0 ? 1 : 2;
    if (h->prec == SES_C128) {
        if (const PlanEntry<double>* p = find_plan<double>(n, kind)) {
            pp.cp = p;
            e = p->e;
            ls = p->ls;
            xw = p->xw;
        }
    } else if (const PlanEntry<float>* p = find_plan<float>(n, kind)) {
        pp.cp = p;
        e = p->e;
        ls = p->ls;
        xw = p->xw;
    }
    if (!pp.cp) return;
    const int tl = n / e;
    if (axis == 0) {
        const long long lpc = (long long)xw * (32 / tl);
        pp.cgrid = (unsigned)((pp.nlines + lpc - 1) / lpc);
        pp.cblock = 32 * xw;
        pp.csmem = 0;
    } else {
        pp.cgrid = (unsigned)((pp.nlines + ls - 1) / ls);
        pp.cblock = (unsigned)(ls * tl);
        pp.csmem = (size_t)n * ls * h->esize;
    }
}

ses_status upload_stage_twiddles(ses_solver* h) {
    for (int a = 0; a < 3; ++a) {
        const PassPlan& pp = h->pp[a];
        if (!pp.cp) continue;
        int r0, r1, r2;
        if (h->prec == SES_C128) {
            const auto* p = reinterpret_cast<const PlanEntry<double>*>(pp.cp);
            r0 = p->r0; r1 = p->r1; r2 = p->r2;
        } else {
            const auto* p = reinterpret_cast<const PlanEntry<float>*>(pp.cp);
            r0 = p->r0; r1 = p->r1; r2 = p->r2;
        }
        const std::vector<double> t = stage_twiddles(h->n[a], r0, r1, r2);
        const size_t cnt = t.size() / 2;
        if (h->prec == SES_C128) {
            SES_TRY(dalloc(h, &h->stw[a], cnt * sizeof(cx<double>)));
            SES_CU(cudaMemcpyAsync(h->stw[a], t.data(), cnt * sizeof(cx<double>), cudaMemcpyHostToDevice, h->stream));
        } else {
            std::vector<float> hi(2 * cnt), lo(2 * cnt);
            for (size_t i = 0; i < 2 * cnt; ++i) {
                hi[i] = (float)t[i];
                lo[i] = (float)(t[i] - (double)hi[i]);
            }
            SES_TRY(dalloc(h, &h->stw[a], cnt * sizeof(cx<float>)));
            SES_TRY(dalloc(h, &h->stwl[a], cnt * sizeof(cx<float>)));
            SES_CU(cudaMemcpyAsync(h->stw[a], hi.data(), cnt * sizeof(cx<float>), cudaMemcpyHostToDevice, h->stream));
            SES_CU(cudaMemcpyAsync(h->stwl[a], lo.data(), cnt * sizeof(cx<float>), cudaMemcpyHostToDevice, h->stream));
        }
    }
    return SES_OK;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
    });
    return fn;
}

// TMA descriptors for the strided passes over `base` (psi or scratch), one per
// pipelined variant (the box width is the variant's tile width L):
// y pass: 3D {nx, ny, nz} boxes {L, rows, 1}; z pass: 2D {nx*ny, nz} boxes {L, rows};
// elements addressed as 8-byte words (complex128 = 2 words).
template <typename T>
void build_tmaps_t(ses_solver* h, int buf, void* base, EncodeTiledFn enc) {
    for (int axis = 1; axis < 3; ++axis) {
        const PassPlan& pp = h->pp[axis];
        if (!pp.cp || h->n[axis] < 2) continue;
        const auto* e = reinterpret_cast<const PlanEntry<T>*>(pp.cp);
        const int n = h->n[axis];
        const cuuint32_t rows = (cuuint32_t)(n > 256 ? 256 : n);
        if (n % (int)rows) continue;
        const cuuint64_t ew = (cuuint64_t)(h->esize / 8);
        const cuuint64_t nx = h->n[0], ny = h->n[1], nz = h->n[2];
        for (int k = 0; k < (int)e->sv.size() && k < ses_solver::kMaxVar; ++k) {
            const int ls = e->sv[k].ls;
            CUresult r;
            if (axis == 1) {
                if (nx % (cuuint64_t)ls) continue;  // a tile must not cross z
                const cuuint64_t dims[3] = {nx * ew, ny, nz};
                const cuuint64_t strides[2] = {nx * h->esize, nx * ny * h->esize};
                const cuuint32_t box[3] = {(cuuint32_t)(ls * ew), rows, 1};
                const cuuint32_t es[3] = {1, 1, 1};
                r = enc(&h->tmap[buf][axis][k], CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            } else {
                const cuuint64_t dims[2] = {nx * ny * ew, nz};
                const cuuint64_t strides[1] = {nx * ny * h->esize};
                const cuuint32_t box[2] = {(cuuint32_t)(ls * ew), rows};
                const cuuint32_t es[2] = {1, 1};
                r = enc(&h->tmap[buf][axis][k], CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            }
            h->tmap_ok[buf][axis][k] = (r == CUDA_SUCCESS);
        }
    }
}

void build_tmaps(ses_solver* h, int buf, void* base) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return;
    if (h->prec == SES_C128) build_tmaps_t<double>(h, buf, base, enc);
    else build_tmaps_t<float>(h, buf, base, enc);
}

ses_status create_impl(const ses_grid_desc* grid, ses_precision prec, double dt, double mass,
                       const double* V, const double* psi0, bool with_tables, ses_handle* out,
                       bool imag = false) {
    if (!grid || !out) return fail(SES_EINVAL, "null grid or output pointer");
    *out = nullptr;
    if (prec != SES_C128 && prec != SES_C64) return fail(SES_EINVAL, "unknown precision");
    const ses_axis ax[3] = {grid->x, grid->y, grid->z};
    for (int a = 0; a < 3; ++a) {
        if (ax[a].n < 1) return fail(SES_EINVAL, "axis length must be >= 1");
        if (!(ax[a].xmax > ax[a].xmin)) return fail(SES_EINVAL, "axis needs xmax > xmin");
    }
    const long long N = (long long)ax[0].n * ax[1].n * ax[2].n;
    if (N >= (1ll << 31)) return fail(SES_EINVAL, "grid exceeds 2^31 points");
    if (with_tables) {
        if (!V) return fail(SES_EINVAL, "potential pointer is null");
        if (!(mass > 0.0)) return fail(SES_EINVAL, "mass must be > 0");
        if (!std::isfinite(dt)) return fail(SES_EINVAL, "dt must be finite");
    }
    init_kernel_attrs();

    // A 1D line longer than one CTA's transform (N > 4096) runs as N1 x N2 with
    // compiled plans for both factors, N1 >= N2 as balanced as possible.
    int long_n1 = 0, long_n2 = 0;
    if (ax[1].n == 1 && ax[2].n == 1 && ax[0].n > 4096) {
        const std::vector<int> lens = {16, 32, 48, 64, 96, 128, 160, 256, 512, 1024};
        for (int n1 : lens) {
            if (ax[0].n % n1) continue;
            const int n2 = ax[0].n / n1;
            if (n2 > n1) continue;
            // N1 runs on the contiguous passes, N2 on the strided ones
            const bool ok = prec == SES_C128 ? (find_plan<double>(n1, 1) && find_plan<double>(n2, 2))
                                             : (find_plan<float>(n1, 1) && find_plan<float>(n2, 2));
            if (ok) {
                long_n1 = n1;
                long_n2 = n2;
                break;
            }
        }
        if (imag)
            return fail(SES_EINVAL, "imaginary time supports lines up to 4096 points");
        if (!long_n1)
            return fail(SES_EINVAL, "1D line of " + std::to_string(ax[0].n) +
                                        " points: lines above 4096 need N = N1 x N2 with both factors in "
                                        "{16,32,48,64,96,128,160,256,512,1024}");
    }

    ses_solver* h = new ses_solver();
    h->prec = prec;
    h->esize = prec == SES_C128 ? 16 : 8;
    h->N = N;
    h->dt = dt;
    h->mass = mass;
    h->with_tables = with_tables;
    h->imag = imag;
    for (int a = 0; a < 3; ++a) {
        h->n[a] = ax[a].n;
        h->box[2 * a] = ax[a].xmin;
        h->box[2 * a + 1] = ax[a].xmax;
    }
    if (long_n1) {
        h->long1d = true;
        h->n[0] = long_n1;
        h->n[1] = long_n2;
    }
    cudaGetDevice(&h->dev);
    h->last_axis = h->n[2] > 1 ? 2 : (h->n[1] > 1 ? 1 : 0);

    auto bail = [&](ses_status s) {
        release(h);
        return s;
    };
    const long long nlines[3] = {(long long)h->n[1] * h->n[2], (long long)h->n[0] * h->n[2],
                                 (long long)h->n[0] * h->n[1]};
    size_t rows = kObsBlocks;
    for (int a = 0; a < 3; ++a) {
        std::string why;
        if (!plan_pass(h->n[a], h->esize, a != 0, nlines[a], h->pp[a], why))
            return bail(fail(SES_EINVAL, why));
        rows = std::max<size_t>(rows, h->pp[a].grid);
        attach_compiled_plan(h, a);
        rows = std::max<size_t>(rows, h->pp[a].cgrid);
    }
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail(SES_EDEVICE, "stream/event creation failed"));
    }
    h->stream = h->own;

    ses_status st;
    if ((st = dalloc(h, &h->psi, N * h->esize)) != SES_OK) return bail(st);
    // scratch: the k-space copy for observables, and the staging area for
    // complex128 halves on C64 upload/readback ((N+1)/2 * 16 B <= N*8 + 16 B)
    if ((st = dalloc(h, &h->scratch, N * h->esize + 16)) != SES_OK) return bail(st);
    h->partial_rows = rows;
    if ((st = dalloc(h, (void**)&h->partials, rows * kRedR * sizeof(double))) != SES_OK) return bail(st);
    if ((st = dalloc(h, (void**)&h->dsums, 32 * sizeof(double))) != SES_OK) return bail(st);
    static_assert(32 * sizeof(double) <= PinnedSlab::kSlot, "observable sums fit a pinned slot");
    if (!(h->hsums = static_cast<double*>(pinned_slab().get())))
        return bail(fail(SES_ENOMEM, "pinned host allocation failed"));
    for (int a = 0; a < 3; ++a) {
        // wavenumber / kinetic tables follow the physical axis (a long line's x
        // tables cover the whole line); FFT twiddles follow the layout axis
        const int n = std::max(h->n[a], phys_n(h, a));
        const int nl = h->n[a];
        if ((st = dalloc(h, &h->tw[a], (size_t)nl * h->esize)) != SES_OK) return bail(st);
        if ((st = dalloc(h, (void**)&h->kv[a], (size_t)n * sizeof(double))) != SES_OK) return bail(st);
        if ((st = dalloc(h, (void**)&h->kd[a], (size_t)n * sizeof(cx<double>))) != SES_OK) return bail(st);
        const unsigned gb = (unsigned)((n + 255) / 256);
        if (prec == SES_C128)
            build_twiddles<double><<<gb, 256, 0, h->stream>>>(nl, reinterpret_cast<cx<double>*>(h->tw[a]));
        else
            build_twiddles<float><<<gb, 256, 0, h->stream>>>(nl, reinterpret_cast<cx<float>*>(h->tw[a]));
        build_axis_tables<<<gb, 256, 0, h->stream>>>(h->box[2 * a], h->box[2 * a + 1], n,
                                                     with_tables ? dt : 0.0,
                                                     with_tables ? mass : 1.0, h->kv[a], h->kd[a]);
        if (imag) build_axis_tables_imag<<<gb, 256, 0, h->stream>>>(n, dt, mass, h->kv[a], h->kd[a]);
        if ((st = dalloc(h, (void**)&h->kdf[a], (size_t)n * sizeof(cx<float>))) != SES_OK) return bail(st);
        convert_kernel<double, float><<<gb, 256, 0, h->stream>>>(h->kd[a], h->kdf[a], n);
    }
    if (h->long1d) {
        if ((st = dalloc(h, &h->kfull, N * h->esize)) != SES_OK) return bail(st);
        if ((st = dalloc(h, &h->tw4, N * h->esize)) != SES_OK) return bail(st);
        if (prec == SES_C64 && (st = dalloc(h, &h->tw4l, N * h->esize)) != SES_OK) return bail(st);
        const unsigned gb = (unsigned)std::min<long long>((N + 255) / 256, 148 * 16);
        const double dtk = with_tables ? dt : 0.0, mk_ = with_tables ? mass : 1.0;
        if (prec == SES_C128)
            build_long_tables<double><<<gb, 256, 0, h->stream>>>(h->kv[0], h->n[0], h->n[1], dtk, mk_,
                                                                 (cx<double>*)h->kfull, (cx<double>*)h->tw4, nullptr);
        else
            build_long_tables<float><<<gb, 256, 0, h->stream>>>(h->kv[0], h->n[0], h->n[1], dtk, mk_,
                                                                (cx<float>*)h->kfull, (cx<float>*)h->tw4,
                                                                (cx<float>*)h->tw4l);
    }
    if (cudaGetLastError() != cudaSuccess) return bail(fail(SES_EDEVICE, "axis table build failed"));
    if ((st = upload_stage_twiddles(h)) != SES_OK) return bail(st);
    if ((st = dalloc(h, (void**)&h->derr, sizeof(unsigned))) != SES_OK) return bail(st);
    if (!(h->herr = static_cast<unsigned*>(pinned_slab().get())))
        return bail(fail(SES_ENOMEM, "pinned host allocation failed"));
    *h->herr = 0;
    if (cudaMemsetAsync(h->derr, 0, sizeof(unsigned), h->stream) != cudaSuccess)
        return bail(fail(SES_EDEVICE, "memset failed"));
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->dev);
    if (const char* env = std::getenv("SES_PIPELINED")) h->pipelined = std::atoi(env) != 0;
    build_tmaps(h, 0, h->psi);
    build_tmaps(h, 1, h->scratch);
    apply_selection(h);
    if (with_tables) {
        if ((st = dalloc(h, (void**)&h->V, N * sizeof(double))) != SES_OK) return bail(st);
        if ((st = dalloc(h, &h->vtab, N * h->esize)) != SES_OK) return bail(st);
        if (cudaMemcpyAsync(h->V, V, N * sizeof(double), cudaMemcpyHostToDevice, h->stream) !=
            cudaSuccess)
            return bail(fail(SES_EDEVICE, "potential upload failed"));
        st = prec == SES_C128 ? build_tables<double>(h) : build_tables<float>(h);
        if (st != SES_OK) return bail(st);
    }
    if (psi0) {
        if ((st = ses_gpu_write_psi(h, psi0)) != SES_OK) return bail(st);
    } else {
        if (cudaMemsetAsync(h->psi, 0, N * h->esize, h->stream) != cudaSuccess)
            return bail(fail(SES_EDEVICE, "memset failed"));
    }
    if ((st = wait_bounded(h, 0)) != SES_OK) return bail(st);
    *out = h;
    return SES_OK;
}

// Observables from the sums enqueue_observe copied to the host (after a wait).
// finish_observe on the device, for ses_gpu_observe_async: the same operations
// in the same order, with round-to-nearest intrinsics so that no multiply-add is
// contracted (the values equal the host's bit for bit).
__global__ void finish_observe_kernel(const double* __restrict__ sums, double dv, ses_observables* out) {
    if (threadIdx.x != 0) return;
    const double* r = sums;
    const double* k = sums + kRedR;
    auto ratio = [](double num, double den) { return den > 0.0 ? __ddiv_rn(num, den) : 0.0; };
    ses_observables o;
    o.norm = __dmul_rn(r[0], dv);
    o.energy_v = ratio(r[1], r[0]);
    o.energy_t = ratio(k[1], k[0]);
    o.energy = __dadd_rn(o.energy_v, o.energy_t);
    o.p_range = __dmul_rn(r[2], dv);
    for (int a = 0; a < 3; ++a) {
        o.mean_pos[a] = ratio(r[3 + a], r[0]);
        const double var = __dsub_rn(ratio(r[6 + a], r[0]), __dmul_rn(o.mean_pos[a], o.mean_pos[a]));
        o.sigma_pos[a] = __dsqrt_rn(fmax(0.0, var));
        o.mean_mom[a] = ratio(k[2 + a], k[0]);
    }
    *out = o;
}

void finish_observe(const ses_solver* h, ses_observables* out) {
    const double* r = h->hsums;
    const double* k = h->hsums + kRedR;
    const double dv = ((h->box[1] - h->box[0]) / phys_n(h, 0)) * ((h->box[3] - h->box[2]) / phys_n(h, 1)) *
                      ((h->box[5] - h->box[4]) / phys_n(h, 2));
    auto ratio = [](double num, double den) { return den > 0.0 ? num / den : 0.0; };
    out->norm = r[0] * dv;
    out->energy_v = ratio(r[1], r[0]);
    out->energy_t = ratio(k[1], k[0]);
    out->energy = out->energy_v + out->energy_t;
    out->p_range = r[2] * dv;
    for (int a = 0; a < 3; ++a) {
        out->mean_pos[a] = ratio(r[3 + a], r[0]);
        const double var = ratio(r[6 + a], r[0]) - out->mean_pos[a] * out->mean_pos[a];
        out->sigma_pos[a] = std::sqrt(std::max(0.0, var));
        out->mean_mom[a] = ratio(k[2 + a], k[0]);
    }
}


// ---------------------------------------------------------------------------
// Batches: many handles advanced together.  Members with the same shape and
// precision form a class; each pass of a step is ONE launch per class
// (xbatch_kernel / sbatch_kernel walking instance x line tiles, grid sized to
// the resident CTAs).  Every class runs its whole step sequence on its own
// stream, forked from and joined back to the batch stream, so classes of
// different sizes overlap on the GPU; interior steps are CUDA graphs per class.
// ---------------------------------------------------------------------------
enum BatchProg {
    BP_XSTART,  // [Vh, fwd x]
    BP_XMID,    // [inv x, V (M), fwd x]
    BP_XEND,    // [inv x, Vh (M)]
    BP_1DFIRST, // 1D [Vh, fwd, K/N, inv]
    BP_1DONE,   // 1D [Vh, fwd, K/N, inv, Vh (M)]
    BP_1DMID,   // 1D [V (M), fwd, K/N, inv]
    BP_1DLAST,  // 1D [V (M), fwd, K/N, inv, Vh (M)]
    BP_NX,
    BP_MID0 = BP_NX,  // strided passes of the step, in order
    BP_LSTART = BP_NX + 3,  // long line: [Vh, fwd y, * W]
    BP_LX,                  // long line: [fwd x, K/N, inv x]
    BP_LMID,                // long line: [* conj W, inv y, V (M), fwd y, * W]
    BP_LEND,                // long line: [* conj W, inv y, Vh (M)]
    BP_COUNT
};

// Axis, mode and potential/mask program of a long-line program.
void long_prog(int prog, bool mask, int* axis, int* mode, XProg* p) {
    *p = XProg();
    switch (prog) {
        case BP_LSTART: *axis = 1; *mode = SM_TW_START; p->d_load = DG_HALF; break;
        case BP_LX: *axis = 0; *mode = XM_1D; break;
        case BP_LMID: *axis = 1; *mode = SM_TW_MID; p->d_mid = DG_FULL; p->m_mid = mask; break;
        default: *axis = 1; *mode = SM_TW_END; p->d_store = DG_HALF; p->m_store = mask; break;
    }
}

XProg batch_xprog(int prog, bool mask) {
    XProg p;
    switch (prog) {
        case BP_XSTART: p.mode = XM_START; p.d_load = DG_HALF; break;
        case BP_XMID: p.mode = XM_MID; p.d_mid = DG_FULL; p.m_mid = mask; break;
        case BP_XEND: p.mode = XM_END; p.d_store = DG_HALF; p.m_store = mask; break;
        case BP_1DFIRST: p.mode = XM_1D; p.d_load = DG_HALF; break;
        case BP_1DONE:
            p.mode = XM_1D; p.d_load = DG_HALF; p.d_store = DG_HALF; p.m_store = mask;
            break;
        case BP_1DMID: p.mode = XM_1D; p.d_load = DG_FULL; p.m_load = mask; break;
        default:
            p.mode = XM_1D; p.d_load = DG_FULL; p.m_load = mask; p.d_store = DG_HALF; p.m_store = mask;
            break;
    }
    return p;
}

struct BatchClass {
    ses_precision prec = SES_C64;
    int n[3] = {1, 1, 1};
    std::vector<ses_solver*> mem;
    bool batched = false;  // every pass of the step has a batched kernel
    int nmid = 0;
    int mid_axis[3] = {0, 0, 0}, mid_mode[3] = {0, 0, 0};
    size_t esz = 0;        // sizeof(PassArgs<T>)
    void* dargs = nullptr; // [prog][mask][member] PassArgs<T>
    size_t dcap = 0;
    // pipelined (TMA-fed) batched variants: -1 = register-path batched kernels
    int xvar = -1;
    int svar[3] = {-1, -1, -1};
    CUtensorMap* dmaps = nullptr;  // [strided pass q][member] tensor maps of the members' psi
    size_t mcap = 0;
    cudaStream_t cs = nullptr, cap = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t body[2] = {nullptr, nullptr};
    bool dirty = true;
    // pinned staging of the argument / tensor-map uploads, two buffers used in
    // turn; staged[i] is recorded after the copies out of hstage[i], so a buffer
    // is rewritten only once the copy that read it has run
    unsigned char* hstage[2] = {nullptr, nullptr};
    size_t hcap[2] = {0, 0};
    cudaEvent_t staged[2] = {nullptr, nullptr};
    int stage_i = 0;
    // two-sweep step of a 3D class (batched plane pass + z pass; nullptr: four passes)
    const void* plane = nullptr;
};

}  // namespace

struct ses_batch_s {
    int dev = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    cudaEvent_t fork = nullptr, ev = nullptr;
    unsigned* derr = nullptr;  // device error word of the pipelined batched passes
    unsigned* herr = nullptr;  // pinned host copy
    std::vector<ses_solver*> members;  // in add order
    std::vector<BatchClass*> classes;
    std::map<std::string, int> sel;    // autotuned variant per class pass (batch_tune_key)
    int sms = 148;
    // graphs replaced while launches of them may still be queued: destroyed once
    // the event recorded on the batch stream at their replacement has completed
    std::vector<std::pair<cudaEvent_t, cudaGraphExec_t>> retired;
};

namespace {

// Host wait (polling, bounded) for an event; false on timeout or device error.
bool event_wait(cudaEvent_t e, int timeout_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) return true;
        if (q != cudaErrorNotReady) return false;
        if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) return false;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

// A class graph that queued launches may still use: destroyed later (reap).
void retire_graph(ses_batch_s* b, cudaGraphExec_t g) {
    if (!g) return;
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(e, b->stream) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(b->stream);  // cannot order it: wait, then destroy now
        if (e) cudaEventDestroy(e);
        cudaGraphExecDestroy(g);
        return;
    }
    b->retired.emplace_back(e, g);
}

// Destroy the retired graphs whose launches have all completed (all: the batch is idle).
void reap(ses_batch_s* b, bool all) {
    for (size_t i = 0; i < b->retired.size();) {
        auto& r = b->retired[i];
        if (all || cudaEventQuery(r.first) == cudaSuccess) {
            cudaGraphExecDestroy(r.second);
            cudaEventDestroy(r.first);
            b->retired.erase(b->retired.begin() + (long)i);
        } else {
            ++i;
        }
    }
    cudaGetLastError();  // a not-ready query leaves no error to report
}

void drop_class(ses_batch_s* b, BatchClass* c) {
    for (auto& g : c->body) {
        retire_graph(b, g);
        g = nullptr;
    }
    for (int i = 0; i < 2; ++i) {
        if (c->staged[i]) {
            event_wait(c->staged[i], 60000);
            cudaEventDestroy(c->staged[i]);
        }
        if (c->hstage[i]) cudaFreeHost(c->hstage[i]);
    }
    if (c->dargs) cudaFree(c->dargs);  // waits for the device: no queued launch reads them any more
    if (c->dmaps) cudaFree(c->dmaps);
    if (c->done) cudaEventDestroy(c->done);
    if (c->cap) cudaStreamDestroy(c->cap);
    if (c->cs) cudaStreamDestroy(c->cs);
    delete c;
}

ses_status batch_wait(ses_batch_s* b, int timeout_ms) {
    if (timeout_ms <= 0) timeout_ms = 10000;
    SES_CU(cudaMemcpyAsync(b->herr, b->derr, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
    SES_CU(cudaEventRecord(b->ev, b->stream));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(b->ev);
        if (q == cudaSuccess) {
            reap(b, false);
            if (*b->herr) {
                *b->herr = 0;
                cudaMemsetAsync(b->derr, 0, sizeof(unsigned), b->stream);
                return fail(SES_ETIMEDOUT, "a pipelined batched pass gave up waiting for its tile loads");
            }
            return SES_OK;
        }
        if (q != cudaErrorNotReady)
            return fail(SES_EDEVICE, std::string("device error: ") + cudaGetErrorString(q));
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - t0)
                            .count();
        if (ms > timeout_ms) return fail(SES_ETIMEDOUT, "wait exceeded " + std::to_string(timeout_ms) + " ms");
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

template <typename T>
bool class_has_batch_kernels(const BatchClass& c) {
    const ses_solver* h = c.mem[0];
    if (h->long1d) {  // four-step programs: contiguous XM_1D and the strided SM_TW_* passes
        const auto* ex = reinterpret_cast<const PlanEntry<T>*>(h->pp[0].cp);
        const auto* ey = reinterpret_cast<const PlanEntry<T>*>(h->pp[1].cp);
        return ex && ey && ex->xb[XM_1D] && ey->sb[SM_TW_START] && ey->sb[SM_TW_MID] && ey->sb[SM_TW_END];
    }
    for (int a = 0; a < 3; ++a) {
        if (h->n[a] < 2 && a > 0) continue;
        if (h->n[a] < 2) return false;  // a 1-point x axis has no compiled plan
        const auto* e = reinterpret_cast<const PlanEntry<T>*>(h->pp[a].cp);
        if (!e) return false;
    }
    return true;
}

// Cache key of a class pass: prog 0 = x pass between steps, 1 + q = strided pass q.
std::string batch_tune_key(const ses_batch_s* b, const BatchClass& c, int prog) {
    std::ostringstream k;
    k << "sm" << b->sms << ":" << (c.prec == SES_C128 ? "c128" : "c64") << ":batch-"
      << (prog == 0 ? std::string("x") : "s" + std::to_string(prog - 1)) << ":" << c.n[0] << "x" << c.n[1]
      << "x" << c.n[2];
    return k.str();
}

template <typename T>
bool xvar_ok(const BatchClass& c, int k) {
    const auto* ex = reinterpret_cast<const PlanEntry<T>*>(c.mem[0]->pp[0].cp);
    if (k < 0 || k >= (int)ex->xv.size()) return false;
    const auto& v = ex->xv[k];
    for (int m : {XM_START, XM_MID, XM_END})
        if (!v.kb[m] || v.bbps[m] <= 0) return false;
    return true;
}

template <typename T>
bool svar_ok(const BatchClass& c, int q, int k, int buf) {
    const ses_solver* h0 = c.mem[0];
    const int a = c.mid_axis[q];
    const auto* es = reinterpret_cast<const PlanEntry<T>*>(h0->pp[a].cp);
    if (k < 0 || k >= (int)es->sv.size() || k >= ses_solver::kMaxVar) return false;
    const auto& v = es->sv[k];
    if (!v.kb[c.mid_mode[q]] || v.bbps[c.mid_mode[q]] <= 0) return false;
    if (a == 1 && h0->n[0] % v.ls) return false;
    for (const ses_solver* h : c.mem)
        if (!h->tmap_ok[buf][a][k]) return false;
    return true;
}

// Variant per class pass: the batch's autotuned choice, else the on-disk cache,
// else the first member's selection; -1 = register-path batched kernel.
template <typename T>
void class_select(const ses_batch_s* b, BatchClass& c) {
    const ses_solver* h0 = c.mem[0];
    c.xvar = -1;
    for (int q = 0; q < 3; ++q) c.svar[q] = -1;
    if (!h0->pipelined || h0->last_axis == 0) return;
    const std::map<std::string, int> cache = read_tune_cache();
    auto pick = [&](int prog, int fallback) {
        const std::string key = batch_tune_key(b, c, prog);
        auto it = b->sel.find(key);
        if (it != b->sel.end()) return it->second;
        auto jt = cache.find(key);
        if (jt != cache.end()) return jt->second;
        return fallback;
    };
    const int xs = pick(0, h0->xsel);
    if (xvar_ok<T>(c, xs)) c.xvar = xs;
    for (int q = 0; q < c.nmid; ++q) {
        const int ss = pick(1 + q, h0->ssel[c.mid_axis[q]]);
        if (svar_ok<T>(c, q, ss, 0)) c.svar[q] = ss;
    }
}

// Tensor maps [q][member] of the members' psi (buf 0) or scratch (buf 1) for
// the class's selected strided variants, into a device table grown as needed.
ses_status class_maps(const BatchClass& c, int buf, CUtensorMap*& dmaps, size_t& cap) {
    const size_t nm = c.mem.size();
    bool any = false;
    for (int q = 0; q < c.nmid; ++q) any = any || c.svar[q] >= 0;
    if (!any) return SES_OK;
    std::vector<CUtensorMap> maps((size_t)3 * nm);
    for (int q = 0; q < c.nmid; ++q)
        if (c.svar[q] >= 0)
            for (size_t i = 0; i < nm; ++i) maps[(size_t)q * nm + i] = c.mem[i]->tmap[buf][c.mid_axis[q]][c.svar[q]];
    const size_t mb = maps.size() * sizeof(CUtensorMap);
    if (mb > cap) {
        if (dmaps) cudaFree(dmaps);
        dmaps = nullptr;
        cap = 0;
        if (cudaMalloc(&dmaps, mb) != cudaSuccess) {
            cudaGetLastError();
            return fail(SES_ENOMEM, "batch tensor map table allocation failed");
        }
        cap = mb;
    }
    SES_CU(cudaMemcpy(dmaps, maps.data(), mb, cudaMemcpyHostToDevice));
    return SES_OK;
}

// Members of a class share one copy of every table whose contents are equal,
// so the batched passes keep one set in L1/L2 instead of one per instance:
// the stage twiddles (same plan) always, and an axis's wavenumber / kinetic
// tables when the axis extent, dt and mass are equal.
template <typename T>
void share_tables(const BatchClass& c, size_t i, PassArgs<T>& a) {
    const ses_solver* h0 = c.mem[0];
    const ses_solver* h = c.mem[i];
    a.stw = reinterpret_cast<const cx<T>*>(h0->stw[a.axis]);
    a.stwl = reinterpret_cast<const cx<T>*>(h0->stwl[a.axis]);
    for (int ax = 0; ax < 3; ++ax)
        for (size_t j = 0; j < i; ++j) {
            const ses_solver* g = c.mem[j];
            if (g->box[2 * ax + 1] - g->box[2 * ax] == h->box[2 * ax + 1] - h->box[2 * ax] && g->dt == h->dt &&
                g->mass == h->mass) {
                a.tb.kd[ax] = g->kd[ax];
                a.tb.kdf[ax] = g->kdf[ax];
                a.tb.kv[ax] = g->kv[ax];
                break;
            }
        }
}

std::string batch_plane_key(const ses_batch_s* b, const BatchClass& c) {
    std::ostringstream k;
    k << "sm" << b->sms << ":" << (c.prec == SES_C128 ? "c128" : "c64") << ":batch-plane:" << c.n[0] << "x"
      << c.n[1] << "x" << c.n[2];
    return k.str();
}

// The batched plane pass of a 3D class (one CTA per plane, built for the class's
// x and y plans), when the step form is two sweeps: by the class's shape and
// precision only -- the batch's tuned choice, else the tune cache, else
// SES_BATCH_PLANE (1: two sweeps), else four passes -- so a member steps the same
// way alone and in any mix.
template <typename T>
const PlaneEntry<T>* class_plane_entry(const BatchClass& c) {
    const ses_solver* h0 = c.mem[0];
    if (!c.batched || h0->long1d || h0->last_axis != 2 || h0->n[1] < 2 || c.nmid != 3) return nullptr;
    const PlaneEntry<T>* pe = nullptr;
    for (const PlaneEntry<T>* e : plane_candidates<T>(h0->n[0], h0->n[1],
                                                      reinterpret_cast<const PlanEntry<T>*>(h0->pp[0].cp),
                                                      reinterpret_cast<const PlanEntry<T>*>(h0->pp[1].cp)))
        if (e->cs == 1 && e->kb[PL_MID]) pe = e;
    return pe;
}

template <typename T>
const void* class_plane(const ses_batch_s* b, const BatchClass& c) {
    const PlaneEntry<T>* pe = class_plane_entry<T>(c);
    if (!pe) return nullptr;
    int use = 0;
    const std::string key = batch_plane_key(b, c);
    auto it = b->sel.find(key);
    if (it != b->sel.end()) {
        use = it->second;
    } else {
        const std::map<std::string, int> cache = read_tune_cache();
        auto jt = cache.find(key);
        if (jt != cache.end()) use = jt->second;
        else if (const char* env = std::getenv("SES_BATCH_PLANE")) use = std::atoi(env);
    }
    return use ? pe : nullptr;
}

template <typename T>
ses_status class_upload(const ses_batch_s* b, BatchClass& c) {
    const size_t nm = c.mem.size();
    const ses_solver* h0 = c.mem[0];
    c.nmid = 0;
    if (h0->last_axis == 2) {
        if (h0->n[1] > 1) { c.mid_axis[c.nmid] = 1; c.mid_mode[c.nmid++] = SM_FWD; }
        c.mid_axis[c.nmid] = 2; c.mid_mode[c.nmid++] = SM_FUSED;
        if (h0->n[1] > 1) { c.mid_axis[c.nmid] = 1; c.mid_mode[c.nmid++] = SM_INV; }
    } else if (h0->last_axis == 1) {
        c.mid_axis[0] = 1; c.mid_mode[0] = SM_FUSED; c.nmid = 1;
    }
    c.batched = class_has_batch_kernels<T>(c);
    if (!c.batched) return SES_OK;
    c.esz = sizeof(PassArgs<T>);
    std::vector<PassArgs<T>> host((size_t)BP_COUNT * 2 * nm);
    for (int prog = 0; prog < BP_COUNT; ++prog)
        for (int mask = 0; mask < 2; ++mask)
            for (size_t i = 0; i < nm; ++i) {
                const ses_solver* h = c.mem[i];
                const bool m = mask && h->has_mask;
                PassArgs<T>& a = host[((size_t)prog * 2 + mask) * nm + i];
                if (prog < BP_NX) {
                    const XProg p = batch_xprog(prog, m);
                    a = make_args<T>(h, 0, h->psi, h->psi);
                    a.d_load = p.d_load; a.d_mid = p.d_mid; a.d_store = p.d_store;
                    a.m_load = p.m_load; a.m_mid = p.m_mid; a.m_store = p.m_store;
                    a.out_scale = p.out_scale;
                } else if (prog >= BP_LSTART) {
                    int ax, md;
                    XProg p;
                    long_prog(prog, m, &ax, &md, &p);
                    a = make_args<T>(h, ax, h->psi, h->psi);
                    a.d_load = p.d_load; a.d_mid = p.d_mid; a.d_store = p.d_store;
                    a.m_load = p.m_load; a.m_mid = p.m_mid; a.m_store = p.m_store;
                } else if (prog - BP_MID0 < c.nmid) {
                    a = make_args<T>(h, c.mid_axis[prog - BP_MID0], h->psi, h->psi);
                } else {
                    a = make_args<T>(h, 0, h->psi, h->psi);  // unused slot
                }
                share_tables(c, i, a);
            }
    class_select<T>(b, c);
    c.plane = class_plane<T>(b, c);
    // tensor maps [q][member] of the members' psi for the selected strided variants
    std::vector<CUtensorMap> maps;
    bool any = false;
    for (int q = 0; q < c.nmid; ++q) any = any || c.svar[q] >= 0;
    if (any) {
        maps.resize((size_t)3 * nm);
        for (int q = 0; q < c.nmid; ++q)
            if (c.svar[q] >= 0)
                for (size_t i = 0; i < nm; ++i) maps[(size_t)q * nm + i] = c.mem[i]->tmap[0][c.mid_axis[q]][c.svar[q]];
    }
    const size_t bytes = host.size() * sizeof(PassArgs<T>);
    const size_t mb = maps.size() * sizeof(CUtensorMap);
    // device tables grow with headroom; a reallocation waits for the device (cudaFree)
    auto grow = [&](void** d, size_t& cap, size_t need, const char* what) -> ses_status {
        if (need <= cap) return SES_OK;
        if (*d) cudaFree(*d);
        *d = nullptr;
        cap = 0;
        const size_t want = need + need / 2;
        if (cudaMalloc(d, want) != cudaSuccess) {
            cudaGetLastError();
            return fail(SES_ENOMEM, std::string("batch ") + what + " table allocation failed");
        }
        cap = want;
        return SES_OK;
    };
    SES_TRY(grow(&c.dargs, c.dcap, bytes, "argument"));
    if (mb) SES_TRY(grow(reinterpret_cast<void**>(&c.dmaps), c.mcap, mb, "tensor map"));
    // stage in pinned memory and copy in stream order: the copies run after every
    // launch queued so far on the batch stream (they read the old contents), so
    // no host wait is needed; the staging buffer is reused two uploads later
    const int si = c.stage_i;
    c.stage_i ^= 1;
    if (!c.staged[si]) SES_CU(cudaEventCreateWithFlags(&c.staged[si], cudaEventDisableTiming));
    else if (!event_wait(c.staged[si], 600000)) return fail(SES_ETIMEDOUT, "batch argument staging wait expired");
    const size_t sb = bytes + ((mb + 63) / 64) * 64 + 64;
    if (sb > c.hcap[si]) {
        if (c.hstage[si]) cudaFreeHost(c.hstage[si]);
        c.hstage[si] = nullptr;
        c.hcap[si] = 0;
        if (cudaMallocHost(reinterpret_cast<void**>(&c.hstage[si]), sb + sb / 2) != cudaSuccess) {
            cudaGetLastError();
            return fail(SES_ENOMEM, "pinned staging allocation failed");
        }
        c.hcap[si] = sb + sb / 2;
    }
    const size_t moff = ((bytes + 63) / 64) * 64;
    std::memcpy(c.hstage[si], host.data(), bytes);
    if (mb) std::memcpy(c.hstage[si] + moff, maps.data(), mb);
    SES_CU(cudaMemcpyAsync(c.dargs, c.hstage[si], bytes, cudaMemcpyHostToDevice, b->stream));
    if (mb) SES_CU(cudaMemcpyAsync(c.dmaps, c.hstage[si] + moff, mb, cudaMemcpyHostToDevice, b->stream));
    SES_CU(cudaEventRecord(c.staged[si], b->stream));
    return SES_OK;
}

// One batched pass of program `prog` over every member of the class.
// args_ovr / maps_ovr (autotuning): the pass's per-member arguments and the
// tensor-map table to use instead of the class's own.
// Batched plane pass (PlaneMode pmode) over every member of class c: the x
// program's arguments carry each member's field, tables and diagonal program,
// the y forward pass's the y stage twiddles and the inverse y scale (1).
template <typename T>
ses_status class_launch_plane(const ses_batch_s* b, const BatchClass& c, int pmode, bool mask, cudaStream_t s,
                              const void* plane = nullptr, const PassArgs<T>* axs = nullptr,
                              const PassArgs<T>* ays = nullptr) {
    const auto* e = reinterpret_cast<const PlaneEntry<T>*>(plane ? plane : c.plane);
    const ses_solver* h0 = c.mem[0];
    const size_t nm = c.mem.size();
    const int xprog = pmode == PL_START ? BP_XSTART : (pmode == PL_MID ? BP_XMID : BP_XEND);
    const PassArgs<T>* base = reinterpret_cast<const PassArgs<T>*>(c.dargs);
    if (!axs) axs = base + ((size_t)xprog * 2 + (mask ? 1 : 0)) * nm;
    if (!ays) ays = base + ((size_t)BP_MID0 * 2 + (mask ? 1 : 0)) * nm;
    const unsigned nz = (unsigned)h0->n[2];
    if ((unsigned long long)nz * nm >= (1ull << 31))
        return fail(SES_EINVAL, "batch class too large: instances x planes must stay below 2^31");
    BatchWork w{};
    w.bpi = nz;
    w.total = (uint32_t)(nz * nm);
    w.fbpi = make_fastdiv(w.bpi);
    const unsigned grid = std::min<unsigned>(w.total, (unsigned)(b->sms * std::max(1, e->kb_bps)));
    launch_pass(h0->pdl, e->kb[pmode], grid, (unsigned)e->nt, e->smem, s, axs, ays, w);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(SES_EDEVICE, std::string("batched plane pass launch: ") + cudaGetErrorString(err));
    return SES_OK;
}

template <typename T>
ses_status class_launch(const ses_batch_s* b, const BatchClass& c, int prog, bool mask, cudaStream_t s,
                        const PassArgs<T>* args_ovr = nullptr, const CUtensorMap* maps_ovr = nullptr) {
    const ses_solver* h0 = c.mem[0];
    if (c.plane && !args_ovr) {  // two-sweep class: x programs are plane passes, the y passes are inside them
        if (prog == BP_XSTART) return class_launch_plane<T>(b, c, PL_START, mask, s);
        if (prog == BP_XMID) return class_launch_plane<T>(b, c, PL_MID, mask, s);
        if (prog == BP_XEND) return class_launch_plane<T>(b, c, PL_END, mask, s);
        if (prog == BP_MID0 || prog == BP_MID0 + 2) return SES_OK;
    }
    int axis = prog < BP_NX ? 0 : (prog >= BP_LSTART ? 1 : c.mid_axis[prog - BP_MID0]);
    int mode = prog < BP_NX ? batch_xprog(prog, mask).mode : (prog >= BP_LSTART ? 0 : c.mid_mode[prog - BP_MID0]);
    if (prog >= BP_LSTART) {
        XProg unused;
        long_prog(prog, mask, &axis, &mode, &unused);
    }
    const PassPlan& pp = h0->pp[axis];
    const auto* e = reinterpret_cast<const PlanEntry<T>*>(pp.cp);
    const size_t nm = c.mem.size();
    const PassArgs<T>* args =
        args_ovr ? args_ovr : reinterpret_cast<const PassArgs<T>*>(c.dargs) + ((size_t)prog * 2 + (mask ? 1 : 0)) * nm;
    const CUtensorMap* maps = maps_ovr ? maps_ovr : c.dmaps;
    const int q = prog - BP_MID0;
    if (prog < BP_LSTART && (axis == 0 ? c.xvar >= 0 && (mode == XM_START || mode == XM_MID || mode == XM_END)
                                       : c.svar[q] >= 0)) {
        const int n = h0->n[axis];
        PipeArgs pa{};
        pa.err = b->derr;
        BatchWork w{};
        if (axis == 0) {
            const auto& v = e->xv[c.xvar];
            w.bpi = (uint32_t)((pp.nlines + v.lpc - 1) / v.lpc);
        } else {
            const auto& v = e->sv[c.svar[q]];
            w.bpi = (uint32_t)((pp.nlines + v.ls - 1) / v.ls);
            pa.kind = axis == 1 ? 0 : 1;
            pa.rows_per_box = n > 256 ? 256 : n;
            pa.nbox = n / pa.rows_per_box;
        }
        if ((unsigned long long)w.bpi * nm >= (1ull << 31))
            return fail(SES_EINVAL, "batch class too large: instances x tiles must stay below 2^31");
        w.total = (uint32_t)(w.bpi * nm);
        w.fbpi = make_fastdiv(w.bpi);
        pa.ntiles = (int)w.total;
        if (axis == 0) {
            const auto& v = e->xv[c.xvar];
            const unsigned grid = std::min<unsigned>(w.total, (unsigned)(b->sms * v.bbps[mode]));
            launch_pass(h0->pdl, v.kb[mode], grid, 32u * v.warps, v.smemb[mode], s, args, w, pa);
        } else {
            const auto& v = e->sv[c.svar[q]];
            const unsigned grid = std::min<unsigned>(w.total, (unsigned)(b->sms * v.bbps[mode]));
            launch_pass(h0->pdl, v.kb[mode], grid, (unsigned)(v.ls * (n / e->e)), v.smem, s, args,
                        maps + (size_t)q * nm, w, pa);
        }
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess)
            return fail(SES_EDEVICE, std::string("batched pipelined pass launch: ") + cudaGetErrorString(err));
        return SES_OK;
    }
    if ((unsigned long long)pp.cgrid * nm >= (1ull << 31))
        return fail(SES_EINVAL, "batch class too large: instances x tiles must stay below 2^31");
    BatchWork w{};
    w.bpi = pp.cgrid;
    w.total = (uint32_t)(pp.cgrid * nm);
    w.fbpi = make_fastdiv(w.bpi);
    if (axis == 0) {
        const int bps = std::max(1, e->xb_bps[mode]);
        const unsigned grid = std::min<unsigned>(w.total, (unsigned)(b->sms * bps));
        launch_pass(h0->pdl, e->xb[mode], grid, pp.cblock, e->xbsm, s, args, w);
    } else {
        const int bps = std::max(1, e->sb_bps[mode]);
        const unsigned grid = std::min<unsigned>(w.total, (unsigned)(b->sms * bps));
        launch_pass(h0->pdl, e->sb[mode], grid, pp.cblock, pp.csmem + e->twb, s, args, w);
    }
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(SES_EDEVICE, std::string("batched pass launch: ") + cudaGetErrorString(err));
    return SES_OK;
}

template <typename T>
ses_status class_unit(const ses_batch_s* b, const BatchClass& c, bool mask, cudaStream_t s) {
    if (c.mem[0]->long1d) {
        SES_TRY(class_launch<T>(b, c, BP_LMID, mask, s));
        return class_launch<T>(b, c, BP_LX, mask, s);
    }
    if (c.mem[0]->last_axis == 0) return class_launch<T>(b, c, BP_1DMID, mask, s);
    SES_TRY(class_launch<T>(b, c, BP_XMID, mask, s));
    for (int q = 0; q < c.nmid; ++q) SES_TRY(class_launch<T>(b, c, BP_MID0 + q, mask, s));
    return SES_OK;
}

template <typename T>
ses_status class_body(const ses_batch_s* b, BatchClass& c, bool mask) {
    cudaGraphExec_t& ex = c.body[mask ? 1 : 0];
    if (ex) return SES_OK;
    if (!c.cap) SES_CU(cudaStreamCreateWithFlags(&c.cap, cudaStreamNonBlocking));
    SES_CU(cudaStreamBeginCapture(c.cap, cudaStreamCaptureModeThreadLocal));
    ses_status st = SES_OK;
    for (int u = 0; u < kBodyUnroll && st == SES_OK; ++u) st = class_unit<T>(b, c, mask, c.cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c.cap, &graph);
    if (st != SES_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return fail(SES_EDEVICE, std::string("graph capture: ") + cudaGetErrorString(e));
    const cudaError_t ie = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        ex = nullptr;
        return fail(SES_EDEVICE, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    return SES_OK;
}

// S merged Strang steps of every member of a batched class, on stream s.
template <typename T>
ses_status class_steps(const ses_batch_s* b, BatchClass& c, int S, bool mask, cudaStream_t s) {
    const bool one_d = c.mem[0]->last_axis == 0;
    const bool long1d = c.mem[0]->long1d;
    int interior;
    if (long1d) {
        SES_TRY(class_launch<T>(b, c, BP_LSTART, mask, s));
        SES_TRY(class_launch<T>(b, c, BP_LX, mask, s));
        interior = S - 1;
    } else if (one_d) {
        if (S == 1) return class_launch<T>(b, c, BP_1DONE, mask, s);
        SES_TRY(class_launch<T>(b, c, BP_1DFIRST, mask, s));
        interior = S - 2;
    } else {
        SES_TRY(class_launch<T>(b, c, BP_XSTART, mask, s));
        for (int q = 0; q < c.nmid; ++q) SES_TRY(class_launch<T>(b, c, BP_MID0 + q, mask, s));
        interior = S - 1;
    }
    if (interior >= kBodyUnroll) SES_TRY(class_body<T>(b, c, mask));
    while (interior >= kBodyUnroll) {
        SES_CU(cudaGraphLaunch(c.body[mask ? 1 : 0], s));
        interior -= kBodyUnroll;
    }
    for (; interior > 0; --interior) SES_TRY(class_unit<T>(b, c, mask, s));
    return class_launch<T>(b, c, long1d ? BP_LEND : (one_d ? BP_1DLAST : BP_XEND), mask, s);
}

// Regroup members into classes and refresh the argument tables of changed ones.
ses_status batch_refresh(ses_batch_s* b) {
    bool any_dirty = false;
    for (BatchClass* c : b->classes) any_dirty |= c->dirty;
    if (!any_dirty) return SES_OK;
    // the new tables are uploaded in stream order (class_upload); launches queued
    // before read the old ones, so nothing waits here
    reap(b, false);
    for (BatchClass* c : b->classes) {
        if (!c->dirty || c->mem.empty()) continue;
        for (auto& g : c->body) {
            retire_graph(b, g);
            g = nullptr;
        }
        SES_TRY(c->prec == SES_C128 ? class_upload<double>(b, *c) : class_upload<float>(b, *c));
        if (!c->cs) SES_CU(cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking));
        if (!c->done) SES_CU(cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming));
        c->dirty = false;
    }
    return SES_OK;
}

BatchClass* find_class(ses_batch_s* b, const ses_solver* h) {
    for (BatchClass* c : b->classes)
        if (c->prec == h->prec && c->n[0] == h->n[0] && c->n[1] == h->n[1] && c->n[2] == h->n[2]) return c;
    return nullptr;
}

// Times every variant of each class pass on the members' scratch fields (psi is
// not touched) and keeps the fastest in b->sel.
template <typename T>
ses_status class_autotune(ses_batch_s* b, BatchClass& c, std::map<std::string, int>& chosen) {
    const size_t nm = c.mem.size();
    const ses_solver* h0 = c.mem[0];
    if (!c.batched || h0->last_axis == 0 || h0->long1d) return SES_OK;
    std::vector<PassArgs<T>> host(nm * (1 + (size_t)c.nmid));
    for (size_t i = 0; i < nm; ++i) {
        const ses_solver* h = c.mem[i];
        PassArgs<T>& a = host[i];
        const XProg p = batch_xprog(BP_XMID, h->has_mask);
        a = make_args<T>(h, 0, h->scratch, h->scratch);
        a.d_mid = p.d_mid;
        a.m_mid = p.m_mid;
        for (int q = 0; q < c.nmid; ++q) host[(1 + (size_t)q) * nm + i] = make_args<T>(h, c.mid_axis[q], h->scratch, h->scratch);
    }
    PassArgs<T>* dargs = nullptr;
    CUtensorMap* dmaps = nullptr;
    size_t mcap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ses_status st = SES_OK;
    auto cleanup = [&]() {
        if (dargs) cudaFree(dargs);
        if (dmaps) cudaFree(dmaps);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    if (cudaMalloc(&dargs, host.size() * sizeof(PassArgs<T>)) != cudaSuccess ||
        cudaMemcpy(dargs, host.data(), host.size() * sizeof(PassArgs<T>), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return fail(SES_ENOMEM, "batch autotune buffers");
    }
    const int saved_x = c.xvar;
    int saved_s[3] = {c.svar[0], c.svar[1], c.svar[2]};
    const void* saved_plane = c.plane;  // the four-pass variants are tuned with the four-pass step
    c.plane = nullptr;
    auto time_prog = [&](int prog, float* ms) -> ses_status {
        const PassArgs<T>* a = dargs + (prog == BP_XMID ? 0 : (size_t)(1 + prog - BP_MID0) * nm);
        SES_TRY(class_maps(c, 1, dmaps, mcap));
        SES_TRY(class_launch<T>(b, c, prog, true, b->stream, a, dmaps));
        SES_CU(cudaEventRecord(e0, b->stream));
        for (int r = 0; r < 3; ++r) SES_TRY(class_launch<T>(b, c, prog, true, b->stream, a, dmaps));
        SES_CU(cudaEventRecord(e1, b->stream));
        SES_TRY(batch_wait(b, 60000));
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        *ms = t / 3;
        return SES_OK;
    };
    // x pass between steps
    {
        const auto* ex = reinterpret_cast<const PlanEntry<T>*>(h0->pp[0].cp);
        int best = -1;
        float best_ms = 1e30f;
        for (int k = -1; k < (int)ex->xv.size() && st == SES_OK; ++k) {
            if (k >= 0 && !xvar_ok<T>(c, k)) continue;
            c.xvar = k;
            float ms = 0.f;
            st = time_prog(BP_XMID, &ms);
            if (st == SES_OK && ms < best_ms) {
                best_ms = ms;
                best = k;
            }
        }
        c.xvar = saved_x;
        if (st == SES_OK) chosen[batch_tune_key(b, c, 0)] = best;
    }
    for (int q = 0; q < c.nmid && st == SES_OK; ++q) {
        const auto* es = reinterpret_cast<const PlanEntry<T>*>(h0->pp[c.mid_axis[q]].cp);
        int best = -1;
        float best_ms = 1e30f;
        for (int k = -1; k < (int)es->sv.size() && st == SES_OK; ++k) {
            if (k >= 0 && !(svar_ok<T>(c, q, k, 1) && svar_ok<T>(c, q, k, 0))) continue;
            c.svar[q] = k;
            float ms = 0.f;
            st = time_prog(BP_MID0 + q, &ms);
            if (st == SES_OK && ms < best_ms) {
                best_ms = ms;
                best = k;
            }
        }
        c.svar[q] = saved_s[q];
        if (st == SES_OK) chosen[batch_tune_key(b, c, 1 + q)] = best;
    }
    // step form: an interior step as four passes (with the variants just chosen)
    // or as the plane pass and the z pass
    const PlaneEntry<T>* pe = class_plane_entry<T>(c);
    if (st == SES_OK && pe) {
        const int sx = c.xvar, s0 = c.svar[0], s1 = c.svar[1], s2 = c.svar[2];
        c.xvar = chosen[batch_tune_key(b, c, 0)];
        for (int q = 0; q < 3; ++q) c.svar[q] = chosen[batch_tune_key(b, c, 1 + q)];
        auto time_unit = [&](bool plane, float* ms) -> ses_status {
            SES_TRY(class_maps(c, 1, dmaps, mcap));
            auto unit = [&]() -> ses_status {
                if (plane) SES_TRY(class_launch_plane<T>(b, c, PL_MID, true, b->stream, pe, dargs, dargs + nm));
                else SES_TRY(class_launch<T>(b, c, BP_XMID, true, b->stream, dargs, dmaps));
                for (int q = 0; q < c.nmid; ++q) {
                    if (plane && q != 1) continue;  // the y passes run inside the plane pass
                    SES_TRY(class_launch<T>(b, c, BP_MID0 + q, true, b->stream, dargs + (size_t)(1 + q) * nm, dmaps));
                }
                return SES_OK;
            };
            SES_TRY(unit());
            SES_CU(cudaEventRecord(e0, b->stream));
            for (int r = 0; r < 3; ++r) SES_TRY(unit());
            SES_CU(cudaEventRecord(e1, b->stream));
            SES_TRY(batch_wait(b, 60000));
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            *ms = t / 3;
            return SES_OK;
        };
        float four = 0.f, two = 0.f;
        st = time_unit(false, &four);
        if (st == SES_OK) st = time_unit(true, &two);
        if (st == SES_OK) chosen[batch_plane_key(b, c)] = two < four ? 1 : 0;
        c.xvar = sx;
        c.svar[0] = s0;
        c.svar[1] = s1;
        c.svar[2] = s2;
    }
    c.plane = saved_plane;
    cleanup();
    return st;
}

ses_status batch_remove_impl(ses_batch_s* b, ses_solver* h) {
    auto it = std::find(b->members.begin(), b->members.end(), h);
    if (it == b->members.end()) return fail(SES_ENOTFOUND, "handle is not a member of this batch");
    // the handle's own stream waits for everything queued on the batch so far
    // (its steps included): no host wait
    SES_CU(cudaEventRecord(h->ev, b->stream));
    SES_CU(cudaStreamWaitEvent(h->own, h->ev, 0));
    b->members.erase(it);
    BatchClass* c = find_class(b, h);
    if (c) {
        c->mem.erase(std::find(c->mem.begin(), c->mem.end(), h));
        c->dirty = true;
        if (c->mem.empty()) {
            b->classes.erase(std::find(b->classes.begin(), b->classes.end(), c));
            drop_class(b, c);
        }
    }
    h->batch = nullptr;
    h->stream = h->own;
    return SES_OK;
}

}  // namespace

// Host <-> device copies of one field on stream s, queued without waiting:
// complex128 directly; complex64 staged in halves through the scratch field
// (rounded on upload, widened on readback).
ses_status enqueue_write_psi(ses_solver* h, const double* psi_in, cudaStream_t s) {
    const size_t N = (size_t)h->N;
    if (h->prec == SES_C128) {
        SES_CU(cudaMemcpyAsync(h->psi, psi_in, N * 16, cudaMemcpyHostToDevice, s));
        return SES_OK;
    }
    const size_t half = (N + 1) / 2;
    for (size_t off = 0; off < N; off += half) {
        const size_t cnt = std::min(half, N - off);
        SES_CU(cudaMemcpyAsync(h->scratch, psi_in + 2 * off, cnt * 16, cudaMemcpyHostToDevice, s));
        const unsigned gb = (unsigned)std::min<size_t>((cnt + 255) / 256, 148 * 32);
        convert_kernel<double, float><<<gb, 256, 0, s>>>(reinterpret_cast<const cx<double>*>(h->scratch),
                                                          reinterpret_cast<cx<float>*>(h->psi) + off,
                                                          (long long)cnt);
        SES_CU(cudaGetLastError());
    }
    return SES_OK;
}

ses_status enqueue_read_psi(ses_solver* h, double* psi_out, cudaStream_t s) {
    const size_t N = (size_t)h->N;
    if (h->prec == SES_C128) {
        SES_CU(cudaMemcpyAsync(psi_out, h->psi, N * 16, cudaMemcpyDeviceToHost, s));
        return SES_OK;
    }
    const size_t half = (N + 1) / 2;
    for (size_t off = 0; off < N; off += half) {
        const size_t cnt = std::min(half, N - off);
        const unsigned gb = (unsigned)std::min<size_t>((cnt + 255) / 256, 148 * 32);
        convert_kernel<float, double><<<gb, 256, 0, s>>>(reinterpret_cast<const cx<float>*>(h->psi) + off,
                                                          reinterpret_cast<cx<double>*>(h->scratch),
                                                          (long long)cnt);
        SES_CU(cudaGetLastError());
        SES_CU(cudaMemcpyAsync(psi_out + 2 * off, h->scratch, cnt * 16, cudaMemcpyDeviceToHost, s));
    }
    return SES_OK;
}

extern "C" {

const char* ses_version(void) { return "ses-b200 0.1 (sm_100a)"; }

const char* ses_last_error(void) { return g_err.c_str(); }

ses_status ses_device_count(int* out) {
    if (!out) return fail(SES_EINVAL, "null output");
    int c = 0;
    const cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = 0;
        return fail(SES_EDEVICE, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    *out = c;
    return SES_OK;
}

ses_status ses_gpu_create(const ses_grid_desc* grid, ses_precision prec, double dt, double mass,
                          const double* V, const double* psi0, ses_handle* out) {
    return create_impl(grid, prec, dt, mass, V, psi0, true, out);
}

ses_status ses_gpu_create_imag(const ses_grid_desc* grid, ses_precision prec, double dtau, double mass,
                               const double* V, const double* psi0, ses_handle* out) {
    if (!(dtau > 0.0)) return fail(SES_EINVAL, "dtau must be > 0");
    return create_impl(grid, prec, dtau, mass, V, psi0, true, out, true);
}

ses_status ses_gpu_relax(ses_handle h, int nsteps, int renorm_every, double* energy) {
    SES_TRY(check_handle(h));
    if (!h->imag) return fail(SES_EINVAL, "handle was not created for imaginary time (ses_gpu_create_imag)");
    if (nsteps < 1) return fail(SES_EINVAL, "nsteps must be >= 1");
    const int R = renorm_every > 0 ? renorm_every : 1;
    int done = 0, last = 1;
    while (done < nsteps) {
        last = std::min(R, nsteps - done);
        SES_TRY(h->prec == SES_C128 ? enqueue_steps<double>(h, last, false) : enqueue_steps<float>(h, last, false));
        SES_TRY(h->prec == SES_C128 ? enqueue_renormalize<double>(h) : enqueue_renormalize<float>(h));
        done += last;
    }
    if (!energy) return SES_OK;
    SES_CU(cudaMemcpyAsync(h->hsums, h->dsums, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    SES_TRY(wait_bounded(h, 0));
    const ObsArgs o = obs_args(h, 0.0, 0.0);
    const double n2 = h->hsums[0] * o.hx * o.hy * o.hz;  // norm^2 after the last `last` steps
    *energy = -std::log(n2) / (2.0 * last * h->dt);
    return SES_OK;
}

ses_status ses_gpu_destroy(ses_handle h) {
    SES_TRY(check_handle(h));
    if (h->batch) SES_TRY(batch_remove_impl(h->batch, h));
    release(h);
    return SES_OK;
}

ses_status ses_gpu_set_potential(ses_handle h, const double* V) {
    SES_TRY(check_handle(h));
    if (!V) return fail(SES_EINVAL, "potential pointer is null");
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no phase tables");
    SES_CU(cudaMemcpyAsync(h->V, V, h->N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    SES_TRY(h->prec == SES_C128 ? build_tables<double>(h) : build_tables<float>(h));
    return wait_bounded(h, 0);
}

ses_status ses_gpu_set_absorber_separable(ses_handle h, const double* mx, const double* my,
                                          const double* mz) {
    SES_TRY(check_handle(h));
    const double* m[3] = {mx, my, mz};
    if (!mx || !my || !mz) return fail(SES_EINVAL, "null mask profile");
    if (h->long1d) {  // stored in full: the layout axes are not the line's axis
        std::vector<double> full((size_t)h->N);
        for (long long i = 0; i < h->N; ++i) full[(size_t)i] = (mx[i] * my[0]) * mz[0];
        return ses_gpu_set_absorber(h, full.data());
    }
    SES_TRY(wait_bounded(h, 0));
    drop_graphs(h);
    if (h->maskfull) {
        cudaFree(h->maskfull);
        h->maskfull = nullptr;
    }
    for (int a = 0; a < 3; ++a) {
        if (!h->mask1[a]) SES_TRY(dalloc(h, (void**)&h->mask1[a], (size_t)h->n[a] * sizeof(double)));
        if (!h->mask1f[a]) SES_TRY(dalloc(h, (void**)&h->mask1f[a], (size_t)h->n[a] * sizeof(float)));
        SES_CU(cudaMemcpyAsync(h->mask1[a], m[a], (size_t)h->n[a] * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        std::vector<float> mf(m[a], m[a] + h->n[a]);
        SES_CU(cudaMemcpyAsync(h->mask1f[a], mf.data(), (size_t)h->n[a] * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    }
    h->has_mask = true;
    return SES_OK;
}

ses_status ses_gpu_set_absorber(ses_handle h, const double* mask) {
    SES_TRY(check_handle(h));
    SES_TRY(wait_bounded(h, 0));
    drop_graphs(h);
    if (!mask) {
        h->has_mask = false;
        return SES_OK;
    }
    // Detect an exact per-axis product mask[i,j,k] == (mx[i]*my[j])*mz[k]:
    // profiles read off the axis lines through the cell of largest mask value.
    const int nx = h->n[0], ny = h->n[1], nz = h->n[2];
    const bool try_separable = !h->long1d;
    long long best = 0;
    for (long long f = 1; f < h->N; ++f)
        if (mask[f] > mask[best]) best = f;
    const int bi = (int)(best % nx), bj = (int)((best / nx) % ny), bk = (int)(best / ((long long)nx * ny));
    bool separable = try_separable && mask[best] == 1.0;
    std::vector<double> mx(nx), my(ny), mz(nz);
    if (separable) {
        for (int i = 0; i < nx; ++i) mx[i] = mask[i + (long long)nx * (bj + (long long)ny * bk)];
        for (int j = 0; j < ny; ++j) my[j] = mask[bi + (long long)nx * (j + (long long)ny * bk)];
        for (int k = 0; k < nz; ++k) mz[k] = mask[bi + (long long)nx * (bj + (long long)ny * k)];
        for (int k = 0; k < nz && separable; ++k)
            for (int j = 0; j < ny && separable; ++j)
                for (int i = 0; i < nx; ++i)
                    if (mx[i] * my[j] * mz[k] != mask[i + (long long)nx * (j + (long long)ny * k)]) {
                        separable = false;
                        break;
                    }
    }
    if (separable) return ses_gpu_set_absorber_separable(h, mx.data(), my.data(), mz.data());
    for (int a = 0; a < 3; ++a) {
        if (h->mask1[a]) cudaFree(h->mask1[a]);
        if (h->mask1f[a]) cudaFree(h->mask1f[a]);
        h->mask1[a] = nullptr;
        h->mask1f[a] = nullptr;
    }
    if (!h->maskfull) SES_TRY(dalloc(h, (void**)&h->maskfull, h->N * sizeof(double)));
    SES_CU(cudaMemcpyAsync(h->maskfull, mask, h->N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->has_mask = true;
    return SES_OK;
}

ses_status ses_gpu_step(ses_handle h, int nsteps, int absorb) {
    SES_TRY(check_handle(h));
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no phase tables");
    if (nsteps < 0) return fail(SES_EINVAL, "nsteps must be >= 0");
    if (nsteps == 0) return SES_OK;
    const bool mask = absorb != 0 && h->has_mask;
    return h->prec == SES_C128 ? enqueue_steps<double>(h, nsteps, mask)
                               : enqueue_steps<float>(h, nsteps, mask);
}

ses_status ses_gpu_step_driven(ses_handle h, int nsteps, int absorb, const double* axis, double amplitude,
                               double omega, double t0) {
    SES_TRY(check_handle(h));
    if (!h->with_tables || h->imag) return fail(SES_EINVAL, "handle has no real-time phase tables");
    if (!axis) return fail(SES_EINVAL, "null polarization axis");
    if (h->last_axis == 0 || h->long1d) return fail(SES_EINVAL, "the dipole drive steps 2D and 3D grids");
    if (nsteps < 0) return fail(SES_EINVAL, "nsteps must be >= 0");
    if (nsteps == 0) return SES_OK;
    const bool mask = absorb != 0 && h->has_mask;
    return h->prec == SES_C128 ? enqueue_driven<double>(h, nsteps, mask, axis, amplitude, omega, t0)
                               : enqueue_driven<float>(h, nsteps, mask, axis, amplitude, omega, t0);
}

ses_status ses_gpu_fft3(ses_handle h, int direction) {
    SES_TRY(check_handle(h));
    if (direction != 0 && direction != 1) return fail(SES_EINVAL, "direction must be 0 or 1");
    return h->prec == SES_C128 ? enqueue_fft3<double>(h, h->psi, direction)
                               : enqueue_fft3<float>(h, h->psi, direction);
}

ses_status ses_gpu_tables(ses_handle h, double* half_v, double* kin) {
    SES_TRY(check_handle(h));
    if (h->imag) return fail(SES_EINVAL, "imaginary-time handle: its tables are real weights, not phases");
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no phase tables");
    if (!half_v && !kin) return SES_OK;
    void *dh = nullptr, *dk = nullptr;
    ses_status st = SES_OK;
    const size_t bytes = h->N * sizeof(cx<double>);
    if (half_v && (st = dalloc(h, &dh, bytes)) != SES_OK) return st;
    if (kin && (st = dalloc(h, &dk, bytes)) != SES_OK) {
        cudaFree(dh);
        return st;
    }
    const unsigned gb = (unsigned)std::min<long long>((h->N + 255) / 256, 148 * 32);
    build_full_tables<<<gb, 256, 0, h->stream>>>(h->V, h->kv[0], h->kv[1], h->kv[2], phys_n(h, 0), phys_n(h, 1),
                                                 h->N, h->dt, h->mass, (cx<double>*)dh, (cx<double>*)dk);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && dh) e = cudaMemcpyAsync(half_v, dh, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && dk) e = cudaMemcpyAsync(kin, dk, bytes, cudaMemcpyDeviceToHost, h->stream);
    st = e == cudaSuccess ? wait_bounded(h, 0) : fail(SES_EDEVICE, cudaGetErrorString(e));
    if (dh) {
        cudaFree(dh);
        h->bytes -= bytes;
    }
    if (dk) {
        cudaFree(dk);
        h->bytes -= bytes;
    }
    return st;
}

ses_status ses_gpu_dt(ses_handle h, double* dt) {
    SES_TRY(check_handle(h));
    if (!dt) return fail(SES_EINVAL, "null output");
    *dt = h->dt;
    return SES_OK;
}

ses_status ses_gpu_observe(ses_handle h, double xlo, double xhi, ses_observables* out) {
    SES_TRY(check_handle(h));
    if (!out) return fail(SES_EINVAL, "null output");
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no potential");
    SES_TRY(h->prec == SES_C128 ? enqueue_observe<double>(h, xlo, xhi)
                                : enqueue_observe<float>(h, xlo, xhi));
    SES_TRY(wait_bounded(h, 0));
    finish_observe(h, out);
    return SES_OK;
}

ses_status ses_gpu_observe_async(ses_handle h, double xlo, double xhi, ses_observables* out) {
    SES_TRY(check_handle(h));
    if (!out) return fail(SES_EINVAL, "null output");
    if (!h->dobs) SES_TRY(dalloc(h, reinterpret_cast<void**>(&h->dobs), sizeof(ses_observables)));
    SES_TRY(h->prec == SES_C128 ? enqueue_observe<double>(h, xlo, xhi) : enqueue_observe<float>(h, xlo, xhi));
    const double dv = ((h->box[1] - h->box[0]) / phys_n(h, 0)) * ((h->box[3] - h->box[2]) / phys_n(h, 1)) *
                      ((h->box[5] - h->box[4]) / phys_n(h, 2));
    finish_observe_kernel<<<1, 32, 0, h->stream>>>(h->dsums, dv, h->dobs);
    SES_CU(cudaGetLastError());
    SES_CU(cudaMemcpyAsync(out, h->dobs, sizeof(ses_observables), cudaMemcpyDeviceToHost, h->stream));
    return SES_OK;
}

ses_status ses_gpu_write_psi(ses_handle h, const double* psi_in) {
    SES_TRY(check_handle(h));
    if (!psi_in) return fail(SES_EINVAL, "null psi");
    SES_TRY(enqueue_write_psi(h, psi_in, h->stream));
    return wait_bounded(h, 0);
}

ses_status ses_gpu_read_psi(ses_handle h, double* psi_out) {
    SES_TRY(check_handle(h));
    if (!psi_out) return fail(SES_EINVAL, "null psi");
    SES_TRY(enqueue_read_psi(h, psi_out, h->stream));
    return wait_bounded(h, 0);
}

// Snapshot wire format: a 128-byte header, then psi in the handle's own precision
// (interleaved float or double pairs, x fastest, as Engine::readback/upload_state).
namespace {
struct SnapHeader {
    char magic[8];       // "SESPSI1"
    int32_t prec;        // ses_precision
    int32_t n[3];
    double box[6];
    double dt, mass;
    int64_t steps;       // caller's step counter
    char pad[128 - 8 - 4 - 12 - 48 - 16 - 8];
};
static_assert(sizeof(SnapHeader) == 128, "snapshot header is 128 bytes");
}  // namespace

ses_status ses_gpu_snapshot(ses_handle h, int64_t steps, void* out, size_t cap, size_t* bytes) {
    SES_TRY(check_handle(h));
    const size_t need = sizeof(SnapHeader) + (size_t)h->N * h->esize;
    if (bytes) *bytes = need;
    if (!out) return SES_OK;  // size query
    if (cap < need) return fail(SES_EINVAL, "snapshot buffer too small: " + std::to_string(need) + " bytes needed");
    SnapHeader hd{};
    std::memcpy(hd.magic, "SESPSI1", 8);
    hd.prec = h->prec;
    for (int a = 0; a < 3; ++a) hd.n[a] = phys_n(h, a);
    for (int a = 0; a < 6; ++a) hd.box[a] = h->box[a];
    hd.dt = h->dt;
    hd.mass = h->mass;
    hd.steps = steps;
    std::memcpy(out, &hd, sizeof(hd));
    SES_CU(cudaMemcpyAsync(static_cast<char*>(out) + sizeof(hd), h->psi, (size_t)h->N * h->esize,
                           cudaMemcpyDeviceToHost, h->stream));
    return wait_bounded(h, 0);
}

ses_status ses_gpu_restore(ses_handle h, const void* snap, size_t bytes, int64_t* steps) {
    SES_TRY(check_handle(h));
    if (!snap || bytes < sizeof(SnapHeader)) return fail(SES_EINVAL, "not a snapshot");
    SnapHeader hd;
    std::memcpy(&hd, snap, sizeof(hd));
    if (std::memcmp(hd.magic, "SESPSI1", 8) != 0) return fail(SES_EINVAL, "not a snapshot (bad magic)");
    if (hd.prec != h->prec) return fail(SES_EINVAL, "snapshot precision differs from the handle's");
    for (int a = 0; a < 3; ++a)
        if (hd.n[a] != phys_n(h, a)) return fail(SES_EINVAL, "snapshot grid differs from the handle's");
    if (bytes < sizeof(SnapHeader) + (size_t)h->N * h->esize) return fail(SES_EINVAL, "snapshot is truncated");
    if (steps) *steps = hd.steps;
    SES_CU(cudaMemcpyAsync(h->psi, static_cast<const char*>(snap) + sizeof(hd), (size_t)h->N * h->esize,
                           cudaMemcpyHostToDevice, h->stream));
    return wait_bounded(h, 0);
}

ses_status ses_gpu_density_slice(ses_handle h, int axis, int index, float* out) {
    SES_TRY(check_handle(h));
    if (!out) return fail(SES_EINVAL, "null output");
    if (axis < 0 || axis > 2) return fail(SES_EINVAL, "axis must be 0, 1 or 2");
    const int nx = phys_n(h, 0), ny = phys_n(h, 1), nz = phys_n(h, 2);
    const int na[3] = {nx, ny, nz};
    if (index < 0 || index >= na[axis]) return fail(SES_EINVAL, "slice index out of range");
    const long long cnt = (long long)(axis == 0 ? ny : nx) * (axis == 2 ? ny : nz);
    float* d = reinterpret_cast<float*>(h->scratch);  // N * esize bytes >= cnt floats
    const unsigned gb = (unsigned)std::min<long long>((cnt + 255) / 256, 148 * 8);
    if (h->prec == SES_C128)
        density_slice_kernel<double><<<gb, 256, 0, h->stream>>>(reinterpret_cast<const cx<double>*>(h->psi), nx, ny,
                                                                nz, axis, index, d);
    else
        density_slice_kernel<float><<<gb, 256, 0, h->stream>>>(reinterpret_cast<const cx<float>*>(h->psi), nx, ny,
                                                               nz, axis, index, d);
    SES_CU(cudaGetLastError());
    SES_CU(cudaMemcpyAsync(out, d, (size_t)cnt * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return wait_bounded(h, 0);
}

ses_status ses_gpu_sync(ses_handle h, int timeout_ms) {
    SES_TRY(check_handle(h));
    return wait_bounded(h, timeout_ms);
}

ses_status ses_gpu_set_stream(ses_handle h, void* cuda_stream) {
    SES_TRY(check_handle(h));
    if (h->batch) return fail(SES_EBUSY, "handle belongs to a batch; set the batch's stream instead");
    SES_TRY(wait_bounded(h, 0));
    h->stream = cuda_stream ? reinterpret_cast<cudaStream_t>(cuda_stream) : h->own;
    return SES_OK;
}

ses_status ses_gpu_psi_device(ses_handle h, void** dptr, size_t* bytes) {
    SES_TRY(check_handle(h));
    if (dptr) *dptr = h->psi;
    if (bytes) *bytes = (size_t)h->N * h->esize;
    return SES_OK;
}

ses_status ses_gpu_profile_step(ses_handle h, int nsteps, int absorb, double* pass_ms) {
    SES_TRY(check_handle(h));
    if (!pass_ms) return fail(SES_EINVAL, "null output");
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no phase tables");
    if (nsteps < 1) return fail(SES_EINVAL, "nsteps must be >= 1");
    if (h->long1d) return fail(SES_EINVAL, "per-pass profile is not available for long 1D lines");
    for (int k = 0; k < 8; ++k) pass_ms[k] = 0.0;
    const bool mask = absorb != 0 && h->has_mask;
    return h->prec == SES_C128 ? profile_batch<double>(h, nsteps, mask, pass_ms)
                               : profile_batch<float>(h, nsteps, mask, pass_ms);
}

ses_status ses_gpu_autotune(ses_handle h, int flags) {
    SES_TRY(check_handle(h));
    SES_TRY(wait_bounded(h, 0));
    if (h->long1d) return SES_OK;  // long lines run the register-path kernels only
    return h->prec == SES_C128 ? autotune_impl<double>(h, flags) : autotune_impl<float>(h, flags);
}

ses_status ses_gpu_plan_info(ses_handle h, char* buf, size_t len) {
    SES_TRY(check_handle(h));
    if (!buf || len == 0) return fail(SES_EINVAL, "null buffer");
    const std::string info = h->prec == SES_C128 ? plan_info_t<double>(h) : plan_info_t<float>(h);
    std::snprintf(buf, len, "%s", info.c_str());
    return SES_OK;
}

ses_status ses_gpu_footprint(ses_handle h, size_t* bytes) {
    SES_TRY(check_handle(h));
    if (!bytes) return fail(SES_EINVAL, "null output");
    *bytes = h->bytes;
    return SES_OK;
}

ses_status ses_gpu_norm_and_peak(ses_handle h, double* norm, double* peak) {
    SES_TRY(check_handle(h));
    if (!norm && !peak) return fail(SES_EINVAL, "null outputs");
    cudaStream_t s = h->stream;
    if (h->prec == SES_C128)
        norm_peak_kernel<double><<<kNormPeakBlocks, 256, 0, s>>>(reinterpret_cast<const cx<double>*>(h->psi), h->N,
                                                                 h->partials);
    else
        norm_peak_kernel<float><<<kNormPeakBlocks, 256, 0, s>>>(reinterpret_cast<const cx<float>*>(h->psi), h->N,
                                                                h->partials);
    norm_peak_finalize<<<1, 32, 0, s>>>(h->partials, kNormPeakBlocks, h->dsums);
    SES_CU(cudaGetLastError());
    SES_CU(cudaMemcpyAsync(h->hsums, h->dsums, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SES_TRY(wait_bounded(h, 0));
    const double dv = ((h->box[1] - h->box[0]) / phys_n(h, 0)) * ((h->box[3] - h->box[2]) / phys_n(h, 1)) *
                      ((h->box[5] - h->box[4]) / phys_n(h, 2));
    if (norm) *norm = h->hsums[0] * dv;
    if (peak) *peak = h->hsums[1];
    return SES_OK;
}

ses_status ses_gpu_scale(ses_handle h, double factor) {
    SES_TRY(check_handle(h));
    if (!std::isfinite(factor)) return fail(SES_EINVAL, "scale factor must be finite");
    const unsigned eb = (unsigned)std::min<long long>((h->N + 255) / 256, (long long)h->sms * 8);
    if (h->prec == SES_C128)
        scale_kernel<double><<<eb, 256, 0, h->stream>>>(reinterpret_cast<cx<double>*>(h->psi), h->N, factor, 0);
    else
        scale_kernel<float><<<eb, 256, 0, h->stream>>>(reinterpret_cast<cx<float>*>(h->psi), h->N, factor, 0);
    SES_CU(cudaGetLastError());
    return SES_OK;
}

ses_status ses_gpu_set_wait_limit(ses_handle h, int64_t wait_cycles, uint32_t extra_tx_bytes) {
    SES_TRY(check_handle(h));
    if (wait_cycles < 0) return fail(SES_EINVAL, "wait_cycles must be >= 0");
    if (extra_tx_bytes > 4096) return fail(SES_EINVAL, "extra_tx_bytes must be <= 4096");
    SES_TRY(wait_bounded(h, 0));  // launches already queued keep their limits
    h->wait_limit = wait_cycles;
    h->extra_tx = extra_tx_bytes;
    drop_graphs(h);               // captured launches carry the old values
    return SES_OK;
}

ses_status ses_gpu_prepare(ses_handle h, int absorb) {
    SES_TRY(check_handle(h));
    return h->prec == SES_C128 ? ensure_body<double>(h, absorb != 0) : ensure_body<float>(h, absorb != 0);
}

ses_status ses_fft3_host(const int32_t* n, ses_precision prec, double* data, int inverse) {
    if (!n || !data) return fail(SES_EINVAL, "null argument");
    ses_grid_desc g{};
    g.x = ses_axis{0.0, 1.0, n[0]};
    g.y = ses_axis{0.0, 1.0, n[1]};
    g.z = ses_axis{0.0, 1.0, n[2]};
    ses_handle h = nullptr;
    SES_TRY(create_impl(&g, prec, 0.0, 1.0, nullptr, data, false, &h));
    ses_status st = ses_gpu_fft3(h, inverse ? 1 : 0);
    if (st == SES_OK) st = ses_gpu_read_psi(h, data);
    release(h);
    return st;
}


// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------
static ses_status check_batch(ses_batch b) {
    if (!b) return fail(SES_EINVAL, "null batch");
    return SES_OK;
}

ses_status ses_batch_create(ses_batch* out) {
    if (!out) return fail(SES_EINVAL, "null output");
    *out = nullptr;
    ses_batch_s* b = new ses_batch_s();
    cudaGetDevice(&b->dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->dev);
    if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (b->fork) cudaEventDestroy(b->fork);
        if (b->own) cudaStreamDestroy(b->own);
        delete b;
        return fail(SES_EDEVICE, "batch stream creation failed (no device?)");
    }
    if (cudaMalloc(&b->derr, sizeof(unsigned)) != cudaSuccess ||
        cudaMallocHost(&b->herr, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(b->derr, 0, sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        if (b->derr) cudaFree(b->derr);
        cudaEventDestroy(b->ev);
        cudaEventDestroy(b->fork);
        cudaStreamDestroy(b->own);
        delete b;
        return fail(SES_ENOMEM, "batch error word allocation failed");
    }
    *b->herr = 0;
    b->stream = b->own;
    *out = b;
    return SES_OK;
}

ses_status ses_batch_destroy(ses_batch b) {
    SES_TRY(check_batch(b));
    const ses_status st = batch_wait(b, 0);
    for (ses_solver* h : b->members) {
        h->batch = nullptr;
        h->stream = h->own;
    }
    for (BatchClass* c : b->classes) drop_class(b, c);
    cudaStreamSynchronize(b->stream);
    reap(b, true);
    if (b->derr) cudaFree(b->derr);
    if (b->herr) cudaFreeHost(b->herr);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return st;
}

ses_status ses_batch_add(ses_batch b, ses_handle h) {
    SES_TRY(check_batch(b));
    SES_TRY(check_handle(h));
    if (h->batch) return fail(SES_EBUSY, "handle already belongs to a batch");
    if (!h->with_tables) return fail(SES_EINVAL, "handle has no phase tables");
    if (h->dev != b->dev) return fail(SES_EINVAL, "handle and batch are on different devices");
    // the batch stream waits for the handle's queued work (uploads, table builds): no host wait
    SES_CU(cudaEventRecord(h->ev, h->stream));
    SES_CU(cudaStreamWaitEvent(b->stream, h->ev, 0));
    h->batch = b;
    h->stream = b->stream;
    b->members.push_back(h);
    BatchClass* c = find_class(b, h);
    if (!c) {
        c = new BatchClass();
        c->prec = h->prec;
        for (int a = 0; a < 3; ++a) c->n[a] = h->n[a];
        b->classes.push_back(c);
    }
    c->mem.push_back(h);
    c->dirty = true;
    return SES_OK;
}

ses_status ses_batch_remove(ses_batch b, ses_handle h) {
    SES_TRY(check_batch(b));
    SES_TRY(check_handle(h));
    if (h->batch != b) return fail(SES_ENOTFOUND, "handle is not a member of this batch");
    return batch_remove_impl(b, h);
}

ses_status ses_batch_step(ses_batch b, int nsteps, int absorb) {
    SES_TRY(check_batch(b));
    if (nsteps < 0) return fail(SES_EINVAL, "nsteps must be >= 0");
    if (nsteps == 0 || b->members.empty()) return SES_OK;
    SES_TRY(batch_refresh(b));
    const bool mask = absorb != 0;
    SES_CU(cudaEventRecord(b->fork, b->stream));
    for (BatchClass* c : b->classes) {
        if (!c->batched) {  // no batched kernels for this shape: each member steps on the batch stream
            for (ses_solver* h : c->mem) SES_TRY(ses_gpu_step(h, nsteps, absorb));
            continue;
        }
        SES_CU(cudaStreamWaitEvent(c->cs, b->fork, 0));
        SES_TRY(c->prec == SES_C128 ? class_steps<double>(b, *c, nsteps, mask, c->cs)
                                    : class_steps<float>(b, *c, nsteps, mask, c->cs));
        SES_CU(cudaEventRecord(c->done, c->cs));
        SES_CU(cudaStreamWaitEvent(b->stream, c->done, 0));
    }
    return SES_OK;
}

ses_status ses_batch_prepare(ses_batch b, int absorb) {
    SES_TRY(check_batch(b));
    if (b->members.empty()) return SES_OK;
    SES_TRY(batch_refresh(b));
    for (BatchClass* c : b->classes) {
        if (c->mem.empty()) continue;
        if (!c->batched) {
            for (ses_solver* h : c->mem) SES_TRY(ses_gpu_prepare(h, absorb));
            continue;
        }
        SES_TRY(c->prec == SES_C128 ? class_body<double>(b, *c, absorb != 0) : class_body<float>(b, *c, absorb != 0));
    }
    return SES_OK;
}

ses_status ses_batch_observe(ses_batch b, double xlo, double xhi, ses_observables* out, int count) {
    SES_TRY(check_batch(b));
    if (!out && count) return fail(SES_EINVAL, "null output");
    if (count != (int)b->members.size())
        return fail(SES_EINVAL, "count must equal the number of members (" +
                                    std::to_string(b->members.size()) + ")");
    for (ses_solver* h : b->members)
        SES_TRY(h->prec == SES_C128 ? enqueue_observe<double>(h, xlo, xhi) : enqueue_observe<float>(h, xlo, xhi));
    SES_TRY(batch_wait(b, 0));
    for (int i = 0; i < count; ++i) finish_observe(b->members[i], &out[i]);
    return SES_OK;
}

ses_status ses_batch_run(ses_batch b, const double* const* psi_in, int nsteps, int absorb, double xlo,
                         double xhi, ses_observables* obs, double* const* psi_out, int count, int timeout_ms) {
    SES_TRY(check_batch(b));
    if (nsteps < 0) return fail(SES_EINVAL, "nsteps must be >= 0");
    if (count != (int)b->members.size())
        return fail(SES_EINVAL, "count must equal the number of members (" +
                                    std::to_string(b->members.size()) + ")");
    SES_TRY(batch_refresh(b));
    std::map<const ses_solver*, int> index;
    for (int i = 0; i < count; ++i) index[b->members[i]] = i;
    // largest class first.  The copies of the class streams share the PCIe link
    // (the copy engines interleave them), so the classes finish their uploads at
    // about the same time and their readbacks queue at the end; chaining the
    // uploads class by class, starting a smaller class first and holding the
    // smallest classes' steps back to overlap the largest one's readback did not
    // shorten the call (measured on B200 with the batched sweep, 0.76-0.77 s either way)
    std::vector<BatchClass*> order(b->classes.begin(), b->classes.end());
    std::stable_sort(order.begin(), order.end(), [](const BatchClass* x, const BatchClass* y) {
        return (double)x->mem.size() * x->n[0] * x->n[1] * x->n[2] > (double)y->mem.size() * y->n[0] * y->n[1] * y->n[2];
    });
    const bool mask = absorb != 0;
    SES_CU(cudaEventRecord(b->fork, b->stream));
    for (BatchClass* c : order) {
        if (c->mem.empty()) continue;
        const cudaStream_t s = c->batched ? c->cs : b->stream;
        if (c->batched) SES_CU(cudaStreamWaitEvent(s, b->fork, 0));
        for (ses_solver* h : c->mem) h->stream = s;  // the member-level enqueues below go to s
        auto queue = [&]() -> ses_status {
            if (psi_in)
                for (ses_solver* h : c->mem)
                    if (const double* p = psi_in[index[h]]) SES_TRY(enqueue_write_psi(h, p, s));
            if (nsteps > 0) {
                if (c->batched)
                    SES_TRY(c->prec == SES_C128 ? class_steps<double>(b, *c, nsteps, mask, s)
                                                : class_steps<float>(b, *c, nsteps, mask, s));
                else
                    for (ses_solver* h : c->mem) SES_TRY(ses_gpu_step(h, nsteps, absorb));
            }
            if (obs)
                for (ses_solver* h : c->mem)
                    SES_TRY(h->prec == SES_C128 ? enqueue_observe<double>(h, xlo, xhi)
                                                : enqueue_observe<float>(h, xlo, xhi));
            if (psi_out)
                for (ses_solver* h : c->mem)
                    if (double* p = psi_out[index[h]]) SES_TRY(enqueue_read_psi(h, p, s));
            return SES_OK;
        };
        const ses_status st = queue();
        for (ses_solver* h : c->mem) h->stream = b->stream;
        if (c->batched) {
            SES_CU(cudaEventRecord(c->done, s));
            SES_CU(cudaStreamWaitEvent(b->stream, c->done, 0));
        }
        if (st != SES_OK) return st;
    }
    SES_TRY(batch_wait(b, timeout_ms > 0 ? timeout_ms : 60000));
    if (obs)
        for (int i = 0; i < count; ++i) finish_observe(b->members[i], &obs[i]);
    return SES_OK;
}

ses_status ses_batch_autotune(ses_batch b, int flags) {
    SES_TRY(check_batch(b));
    SES_TRY(batch_refresh(b));
    std::map<std::string, int> chosen;
    for (BatchClass* c : b->classes)
        SES_TRY(c->prec == SES_C128 ? class_autotune<double>(b, *c, chosen) : class_autotune<float>(b, *c, chosen));
    for (const auto& kv : chosen) b->sel[kv.first] = kv.second;
    for (BatchClass* c : b->classes) c->dirty = true;  // re-select, re-upload maps, re-capture graphs
    if (flags & 1) write_tune_cache(chosen);
    return batch_refresh(b);
}

ses_status ses_batch_info(ses_batch b, char* buf, size_t len) {
    SES_TRY(check_batch(b));
    if (!buf || len == 0) return fail(SES_EINVAL, "null buffer");
    SES_TRY(batch_refresh(b));
    std::ostringstream o;
    for (size_t i = 0; i < b->classes.size(); ++i) {
        const BatchClass* c = b->classes[i];
        o << (i ? "; " : "") << c->n[0] << "x" << c->n[1] << "x" << c->n[2] << " "
          << (c->prec == SES_C128 ? "c128" : "c64") << " members=" << c->mem.size();
        if (!c->batched) {
            o << " member-by-member";
            continue;
        }
        if (c->plane) {  // two sweeps: the plane pass replaces the x and y passes
            o << " plane";
            o << " s1=" << (c->svar[1] >= 0 ? "pipe" + std::to_string(c->svar[1]) : std::string("reg"));
            continue;
        }
        o << " x=" << (c->xvar >= 0 ? "pipe" + std::to_string(c->xvar) : std::string("reg"));
        for (int q = 0; q < c->nmid; ++q)
            o << " s" << q << "=" << (c->svar[q] >= 0 ? "pipe" + std::to_string(c->svar[q]) : std::string("reg"));
    }
    const std::string t = o.str();
    std::snprintf(buf, len, "%s", t.c_str());
    return SES_OK;
}

ses_status ses_batch_observe_some(ses_batch b, const ses_handle* hs, int count, const double* xlo,
                                  const double* xhi, ses_observables* out) {
    SES_TRY(check_batch(b));
    if (count < 0 || (count > 0 && (!hs || !xlo || !xhi || !out))) return fail(SES_EINVAL, "null argument");
    for (int i = 0; i < count; ++i)
        if (!hs[i] || hs[i]->batch != b) return fail(SES_EINVAL, "handle is not a member of this batch");
    for (int i = 0; i < count; ++i) {
        ses_solver* h = hs[i];
        SES_TRY(h->prec == SES_C128 ? enqueue_observe<double>(h, xlo[i], xhi[i]) : enqueue_observe<float>(h, xlo[i], xhi[i]));
    }
    SES_TRY(batch_wait(b, 0));
    for (int i = 0; i < count; ++i) finish_observe(hs[i], &out[i]);
    return SES_OK;
}

ses_status ses_batch_sync(ses_batch b, int timeout_ms) {
    SES_TRY(check_batch(b));
    return batch_wait(b, timeout_ms);
}

ses_status ses_batch_set_stream(ses_batch b, void* cuda_stream) {
    SES_TRY(check_batch(b));
    SES_TRY(batch_wait(b, 0));
    b->stream = cuda_stream ? reinterpret_cast<cudaStream_t>(cuda_stream) : b->own;
    for (ses_solver* h : b->members) h->stream = b->stream;
    return SES_OK;
}

ses_status ses_batch_members(ses_batch b, int* members, int* classes) {
    SES_TRY(check_batch(b));
    if (members) *members = (int)b->members.size();
    if (classes) *classes = (int)b->classes.size();
    return SES_OK;
}

ses_status ses_batch_profile(ses_batch b, int nsteps, int absorb, double* ms, int count) {
    SES_TRY(check_batch(b));
    if (nsteps < 1) return fail(SES_EINVAL, "nsteps must be >= 1");
    if (!ms || count < (int)b->classes.size() * 5)
        return fail(SES_EINVAL, "output needs 5 values per class");
    SES_TRY(batch_refresh(b));
    const bool mask = absorb != 0;
    for (size_t ci = 0; ci < b->classes.size(); ++ci) {
        BatchClass* c = b->classes[ci];
        double* o = ms + 5 * ci;
        for (int q = 0; q < 5; ++q) o[q] = 0.0;
        if (!c->batched || c->mem[0]->long1d) continue;
        const bool one_d = c->mem[0]->last_axis == 0;
        std::vector<int> progs;
        progs.push_back(one_d ? (int)BP_1DMID : (int)BP_XMID);
        if (!one_d)
            for (int q = 0; q < c->nmid; ++q) progs.push_back(BP_MID0 + q);
        std::vector<cudaEvent_t> ev((size_t)nsteps * progs.size() + 1);
        for (auto& e : ev) SES_CU(cudaEventCreate(&e));
        size_t k = 0;
        auto run = [&](int prog) {
            return c->prec == SES_C128 ? class_launch<double>(b, *c, prog, mask, b->stream)
                                       : class_launch<float>(b, *c, prog, mask, b->stream);
        };
        // untimed batch start, so that the fields stay a valid Strang batch
        ses_status st = run(one_d ? (int)BP_1DFIRST : (int)BP_XSTART);
        if (!one_d)
            for (int q = 0; q < c->nmid && st == SES_OK; ++q) st = run(BP_MID0 + q);
        if (st == SES_OK) SES_CU(cudaEventRecord(ev[k++], b->stream));
        for (int s = 0; s < nsteps && st == SES_OK; ++s)
            for (int prog : progs) {
                st = c->prec == SES_C128 ? class_launch<double>(b, *c, prog, mask, b->stream)
                                         : class_launch<float>(b, *c, prog, mask, b->stream);
                if (st != SES_OK) break;
                cudaEventRecord(ev[k++], b->stream);
            }
        if (st == SES_OK) st = run(one_d ? (int)BP_1DLAST : (int)BP_XEND);
        if (st == SES_OK) st = batch_wait(b, 0);
        if (st == SES_OK) {
            for (int s = 0; s < nsteps; ++s)
                for (size_t p = 0; p < progs.size(); ++p) {
                    const size_t i = 1 + (size_t)s * progs.size() + p;
                    float t = 0.f;
                    cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
                    o[p] += t / nsteps;
                    o[4] += t / nsteps;
                }
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (st != SES_OK) return st;
    }
    return SES_OK;
}

}  // extern "C"
